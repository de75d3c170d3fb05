// Chain-aggregation multigrid (CAMG) preconditioned conjugate gradient for the
// DEA systems (device).
//
// Why: in a CNT resistor network the element resistors along one CNT conduct
// 1e4-1e9 times better than the tunnelling junctions between CNTs, so after the
// chain block-Jacobi has equilibrated every CNT the remaining error is "one
// potential per CNT", a graph Laplacian over CNTs with junction conductances
// spanning five orders of magnitude.  One-level preconditioners take thousands
// of iterations on it; a coarse space with one unknown per chain block removes
// it.  The hierarchy:
//
//   level 0   the free-node system; smoother: the chain blocks (explicit
//             tridiagonal inverses), damped by kOmega0 so 2 M^-1 - A stays
//             positive definite on floating islands (bipartite trees of CNTs
//             that no prescribed node reaches, where the undamped block smoother
//             would make the V-cycle singular)
//   level 1   one unknown per chain block (aggregate = block)
//   level l+1 pairwise aggregates of level l: three rounds of handshake
//             matching on the strongest coupling |a_ij| (ties: smaller j), then
//             every unmatched row joins the pair of its strongest neighbour
//   coarsest  <= kMgDenseMax rows: dense inverse (Gauss-Jordan in shared
//             memory, 1e-8 diagonal regularisation, variables with a vanishing
//             pivot dropped); otherwise an l1-Jacobi step
//
// Coarse operators are Galerkin products P^T A P with piecewise-constant P: one
// thread per aggregate gathers its members' cross-aggregate couplings, sorts
// them stably by coarse column and sums each run in order (deterministic, no
// host synchronisation inside a level).  Their diagonals come from summed row
// sums, diag_J = sum_{I in J} rowsum_I - sum_{J' != J} A_JJ', so the large
// intra-aggregate conductances never cancel in floating point and an aggregate
// with no outside coupling gets an exact zero row.  Levels >= 1 are smoothed by
// l1-Jacobi (1 / (|d| + sum |a|)), which makes the symmetric V(1,1)-cycle an SPD
// preconditioner.
//
// The solve is one persistent cooperative launch.  Level-0 rows are split over
// CTAs at block boundaries (the block smoother only reads rows of its own CTA);
// coarse levels are spread over all threads.  Per CG iteration the grid barriers
// are: 1 after the pre-smoother and r.r, one per restriction, one after the
// coarse solve, one per prolongation above level 1, one after the post-smoother
// and r.z, one after p.q.  The stopping rule, FP64 true-residual replacement and
// the first-iteration behaviour are those of the one-level kernel (solver.cu).
#include <algorithm>
#include <cmath>
#include <vector>

#include "solver.cuh"
#include "trace.cuh"

namespace cicy {

namespace {

constexpr int kMgThreads = 256;
constexpr int kMgClusterThreads = 1024;
constexpr int kMgClusterCtas = 16;            // non-portable cluster size
constexpr int kMgClusterMaxRows = 20000;  // above this the grid-wide variant (more threads per row) is faster on B200
constexpr int kMgMaxRestarts = 24;
constexpr double kOmega0 = 0.95;

int grid_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)b;
}

// ---------------------------------------------------------------------------
// Setup kernels

__global__ void k_block_of_row(int n, const int32_t* __restrict__ is_start, const int32_t* __restrict__ start_scan,
                               int32_t* __restrict__ agg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        agg[i] = start_scan[i] + is_start[i] - 1;
}

// Row sums of the level-0 matrix (diagonal included); a row sum at rounding level
// of its diagonal is an unconnected (floating) row: exactly 0.
__global__ void k_rowsum0(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                          double* __restrict__ rs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0, d = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            s += v[k];
            if (ci[k] == i) d = v[k];
        }
        rs[i] = (fabs(s) <= 1e-13 * fabs(d)) ? 0.0 : s;
    }
}

// Strongest neighbour of each row (|a_ij| largest, ties: smaller j); with
// free_only, among unmatched rows and only for unmatched rows.
__global__ void k_strongest(int n, int free_only, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                            const double* __restrict__ v, const int32_t* __restrict__ mate, int32_t* __restrict__ best) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int bj = -1;
        if (!(free_only && mate[i] >= 0)) {
            double bs = -1.0;
            for (int k = rp[i]; k < rp[i + 1]; k++) {
                const int j = ci[k];
                if (free_only && mate[j] >= 0) continue;
                const double s = fabs(v[k]);
                if (s > bs || (s == bs && j < bj)) {
                    bs = s;
                    bj = j;
                }
            }
        }
        best[i] = bj;
    }
}

__global__ void k_handshake(int n, const int32_t* __restrict__ best, int32_t* __restrict__ mate) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int j = best[i];
        if (mate[i] < 0 && j >= 0 && best[j] == i) mate[i] = j;
    }
}

__global__ void k_pair_rep(int n, const int32_t* __restrict__ mate, int32_t* __restrict__ rep) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        rep[i] = mate[i] >= 0 ? min(i, mate[i]) : i;
}

// Unmatched rows join the pair of their strongest neighbour (pairs' representatives
// are never rewritten here, so reading rep[j] is race-free).
__global__ void k_join(int n, const int32_t* __restrict__ mate, const int32_t* __restrict__ best, int32_t* __restrict__ rep) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int j = best[i];
        if (mate[i] < 0 && j >= 0 && mate[j] >= 0) rep[i] = rep[j];
    }
}

__global__ void k_is_rep(int n, const int32_t* __restrict__ rep, int32_t* __restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flag[i] = rep[i] == i ? 1 : 0;
}

__global__ void k_agg_ids(int n, const int32_t* __restrict__ rep, const int32_t* __restrict__ id, int32_t* __restrict__ agg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) agg[i] = id[rep[i]];
}

__global__ void k_fill_neg(int n, int32_t* __restrict__ a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = -1;
}

// Dense coarsest matrix (M zeroed before), then its inverse in place by Gauss-Jordan
// without pivoting (SPD up to floating islands).
__global__ void k_dense_coarse(int nc, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                               const double* __restrict__ diag, double* __restrict__ M) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        for (int k = rp[i]; k < rp[i + 1]; k++) M[(size_t)i * nc + ci[k]] = v[k];
        M[(size_t)i * nc + i] = diag[i];
    }
}

// Blocked in-place Gauss-Jordan (32 pivots per block).  For pivot block b with the others o:
// one warp inverts the Schur-complemented diagonal block D = S_bb pivot by pivot (dropping a
// variable whose pivot vanishes: its row and column of D^-1 are zero), then the CTA applies the
// block step S_bo <- D^-1 S_bo, S_ob <- -S_ob D^-1, S_oo <- S_oo - S_ob D^-1 S_bo, S_bb <- D^-1:
// the unblocked elimination's result with 4 barriers per block instead of 2 per pivot.
constexpr int kGjBlock = 32;
constexpr int kGjDS = kGjBlock + 1;  // row stride of a diagonal block in shared memory

// The CTA's kGjThreads (512) threads: D <- D^-1 in place (32 x 32, row stride kGjDS; a smaller
// block is padded with the identity, which stays decoupled); a variable whose pivot is not
// above thr is dropped (its row and column of D^-1 are zero).  Thread t holds column t % 32 of
// rows t / 32 and t / 32 + 16 in registers; each pivot's row and column go through shared
// memory (fcol, frow), two barriers per pivot, so the pivot chain is a barrier, a division and
// one FMA per step rather than a warp's serial sweep over the block.
constexpr int kGjThreads = 512;
__device__ __forceinline__ void gj_cta_invert(double* D, double* fcol, double* frow, double thr) {
    static_assert(kGjThreads == 16 * kGjBlock, "two entries of the 32 x 32 block per thread");
    const int t = threadIdx.x, j = t & 31, i0 = t >> 5, i1 = i0 + 16;
    double a0 = D[i0 * kGjDS + j], a1 = D[i1 * kGjDS + j];
    for (int k = 0; k < kGjBlock; k++) {
        if (j == k) {
            fcol[i0] = a0;
            fcol[i1] = a1;
        }
        if (i0 == k) frow[j] = a0;
        if (i1 == k) frow[j] = a1;
        __syncthreads();
        const double p = frow[k];
        if (!(p > thr)) {  // vanishing pivot: drop variable k (row k and column k)
            if (i0 == k || j == k) a0 = 0.0;
            if (i1 == k || j == k) a1 = 0.0;
        } else {
            const double dk = ((j == k) ? 1.0 : frow[j]) / p;  // the new pivot row
            a0 = (i0 == k) ? dk : ((j == k) ? 0.0 : a0) - fcol[i0] * dk;
            a1 = (i1 == k) ? dk : ((j == k) ? 0.0 : a1) - fcol[i1] * dk;
        }
        __syncthreads();
    }
    D[i0 * kGjDS + j] = a0;
    D[i1 * kGjDS + j] = a1;
    __syncthreads();
}

__global__ void __launch_bounds__(kGjThreads) k_gauss_jordan(int n, double* __restrict__ M) {
    extern __shared__ double S[];  // n * n, then Cb (n x 32), Rb (32 x n), D (32 x 33), f (32)
    __shared__ double gj_fcol[kGjBlock], gj_frow[kGjBlock];
    double* Cb = S + (size_t)n * n;
    double* Rb = Cb + (size_t)n * kGjBlock;
    double* D = Rb + (size_t)kGjBlock * n;
    __shared__ double dmax_s;
    const int t = threadIdx.x;
    for (int e = t; e < n * n; e += kGjThreads) S[e] = M[e];
    __syncthreads();
    if (t == 0) {
        double m = 0;
        for (int i = 0; i < n; i++) m = fmax(m, fabs(S[i * n + i]));
        dmax_s = m;
    }
    __syncthreads();
    const double thr = 1e-12 * dmax_s;
    for (int i = t; i < n; i += kGjThreads) S[i * n + i] *= (1.0 + 1e-8);
    __syncthreads();
    constexpr int DS = kGjDS;
    for (int b0 = 0; b0 < n; b0 += kGjBlock) {
        const int m = min(kGjBlock, n - b0);
        for (int e = t; e < kGjBlock * kGjBlock; e += kGjThreads) {
            const int r = e / kGjBlock, c = e % kGjBlock;
            D[r * DS + c] = (r < m && c < m) ? S[(b0 + r) * n + b0 + c] : (r == c ? 1.0 : 0.0);
        }
        for (int e = t; e < n * m; e += kGjThreads) Cb[(e / m) * kGjBlock + e % m] = S[(e / m) * n + b0 + e % m];
        __syncthreads();
        gj_cta_invert(D, gj_fcol, gj_frow, thr);
        // Rb = D^-1 S_bo (columns outside the block)
        for (int e = t; e < m * n; e += kGjThreads) {
            const int ii = e / n, jc = e % n;
            if (jc >= b0 && jc < b0 + m) continue;
            double acc = 0;
            for (int kk = 0; kk < m; kk++) acc += D[ii * DS + kk] * S[(b0 + kk) * n + jc];
            Rb[ii * n + jc] = acc;
        }
        __syncthreads();
        for (int e = t; e < n * n; e += kGjThreads) {
            const int i = e / n, jc = e % n;
            const bool ib = i >= b0 && i < b0 + m, jb = jc >= b0 && jc < b0 + m;
            double v;
            if (ib) {
                v = jb ? D[(i - b0) * DS + (jc - b0)] : Rb[(i - b0) * n + jc];
            } else if (jb) {
                double acc = 0;
                for (int kk = 0; kk < m; kk++) acc += Cb[i * kGjBlock + kk] * D[kk * DS + (jc - b0)];
                v = -acc;
            } else {
                double acc = 0;
                for (int kk = 0; kk < m; kk++) acc += Cb[i * kGjBlock + kk] * Rb[kk * n + jc];
                v = S[e] - acc;
            }
            S[e] = v;
        }
        __syncthreads();
    }
    for (int e = t; e < n * n; e += kGjThreads) M[e] = S[e];
}

__global__ void k_ra_fill(int nc, const int32_t* __restrict__ mptr, const int32_t* __restrict__ midx, const int32_t* __restrict__ rp,
                          const int32_t* __restrict__ ci, const double* __restrict__ v, const double* __restrict__ diag,
                          const int32_t* __restrict__ ra_ptr, int32_t* __restrict__ ra_col, double* __restrict__ ra_val) {
    for (int J = blockIdx.x * blockDim.x + threadIdx.x; J < nc; J += gridDim.x * blockDim.x) {
        int e = ra_ptr[J];
        for (int m = mptr[J]; m < mptr[J + 1]; m++) {
            const int I = midx[m];
            ra_col[e] = I;
            ra_val[e] = diag[I];
            e++;
            for (int k = rp[I]; k < rp[I + 1]; k++) {
                ra_col[e] = ci[k];
                ra_val[e] = v[k];
                e++;
            }
        }
    }
}

// Fused restriction rows of level l >= 1 into level l + 1 (clustered kernel): row J holds
// the members of aggregate J (column m < n: r_l[m], weight 1), then for each member I its
// diagonal and couplings (column n + c: z_l[c], weight -a), the rows of P^T A_l, so
// r_{l+1} = P^T (r_l - A_l z_l) is one gathered dot product.  rr_ptr = mptr + ra_ptr, both
// prefix sums (ra_ptr: the P^T A_l row lengths).
__global__ void k_rr_fill(int nc, int n, const int32_t* __restrict__ mptr, const int32_t* __restrict__ midx,
                          const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                          const double* __restrict__ diag, const int32_t* __restrict__ ra_ptr, int32_t* __restrict__ rr_ptr,
                          int32_t* __restrict__ rr_col, double* __restrict__ rr_val) {
    for (int J = blockIdx.x * blockDim.x + threadIdx.x; J < nc; J += gridDim.x * blockDim.x) {
        int e = mptr[J] + ra_ptr[J];
        rr_ptr[J] = e;
        if (J == nc - 1) rr_ptr[nc] = mptr[nc] + ra_ptr[nc];
        for (int m = mptr[J]; m < mptr[J + 1]; m++, e++) {
            rr_col[e] = midx[m];
            rr_val[e] = 1.0;
        }
        for (int m = mptr[J]; m < mptr[J + 1]; m++) {
            const int I = midx[m];
            rr_col[e] = n + I;
            rr_val[e] = -diag[I];
            e++;
            for (int k = rp[I]; k < rp[I + 1]; k++, e++) {
                rr_col[e] = n + ci[k];
                rr_val[e] = -v[k];
            }
        }
    }
}

// Fused prolongation-smoother rows of level l (1 <= l < coarsest): row I holds its diagonal
// and off-diagonal couplings twice, on z_l (column c < n) and on the coarse correction
// (column n + aggregate of c), so w = r_l - A_l (z_l + P zc) is one gathered dot product.
__global__ void k_pq_fill(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                          const double* __restrict__ diag, const int32_t* __restrict__ agg, int32_t* __restrict__ pq_ptr,
                          int32_t* __restrict__ pq_col, double* __restrict__ pq_val) {
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < n; I += gridDim.x * blockDim.x) {
        int e = 2 * (rp[I] + I);
        pq_ptr[I] = e;
        if (I == n - 1) pq_ptr[n] = 2 * (rp[n] + n);
        pq_col[e] = I;
        pq_val[e] = diag[I];
        pq_col[e + 1] = n + agg[I];
        pq_val[e + 1] = diag[I];
        e += 2;
        for (int k = rp[I]; k < rp[I + 1]; k++, e += 2) {
            const int c = ci[k];
            pq_col[e] = c;
            pq_val[e] = v[k];
            pq_col[e + 1] = n + agg[c];
            pq_val[e + 1] = v[k];
        }
    }
}

// ---------------------------------------------------------------------------
// Solve kernel

constexpr int kGroup = 8;  // lanes cooperating on one coarse row

struct MgArgs {
    int n;
    const int32_t* rp;
    const int32_t* ci;
    const double* val;
    const double* b;
    double* x;
    const double* x0;  // when set, the solve starts from x0 (batched solves); else r = b - A x is given
    double *r, *z0, *z, *w, *p, *q;
    const double* tinv;
    const int32_t *row_off, *row_base, *row_m;
    const int32_t* cta_row;
    int levels;            // number of levels including level 0
    const MgLevel* lv;     // device descriptors
    const double* cinv;    // dense inverse of the coarsest level, or nullptr
    double omega0;
    double* partA;
    double* partB;
    double* stats;
    unsigned long long* bar;  // monotonic arrival counter (zeroed before the launch)
    long long spin_limit;     // polls of a barrier wait before it gives up
    int* err;
    double tol;
    long long max_iter;
    int max_restarts;
    int cap_b;  // stop at |r| <= tol min(|r0|, |b|) (batched solves); else |r| <= tol |r0| (Direct_Electrifying.cpp:1571, 1619)
};

// Grid barrier on a monotonic counter: one release-reduction per CTA (no return
// value to wait for; the release orders the CTA's writes, which __syncthreads
// gathered under thread 0, before the arrival), then an acquire spin until all
// CTAs of this round arrived.  Bounded: after `limit` polls the CTA records
// DEV_TIMEOUT and returns false.
__device__ __forceinline__ bool mg_sync(unsigned long long* bar, unsigned long long& target, int* err, int* s_ok, long long limit) {
    __syncthreads();
    if (threadIdx.x == 0) {
        target += gridDim.x;
        asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(bar) : "memory");
        long long spins = 0;
        int ok = 1;
        while (true) {
            unsigned long long v;
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(bar) : "memory");
            if (v >= target) break;
            if (++spins > limit || ((spins & 1023) == 0 && *((volatile int*)err) != 0)) {
                atomicCAS(err, 0, (int)DEV_TIMEOUT);
                ok = 0;
                break;
            }
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// Dense inverse of a coarsest level too large for one CTA: blocked Gauss-Jordan (32 pivots
// per block, the drop rule and regularisation of k_gauss_jordan) over the whole grid, one
// cooperative launch with one grid barrier per block.  CTA c keeps the column strip
// [c0, c1) of the matrix in shared memory.  Block step b: every CTA reads the block's column
// panel S[:, b] (global, double-buffered; the strips holding the panel's columns wrote it at
// the end of step b - 1), inverts the diagonal block D = S_bb (one warp), and updates its own
// columns j: outside the block R_j = D^-1 S_bj, S_ij -= S_ib R_j (rows outside), S_bj = R_j;
// inside it S_ij = -S_ib (D^-1)_j (rows outside), S_bj = (D^-1)_j.  The products sum over the
// block's pivots in order, as k_gauss_jordan's do.
constexpr int kGjgThreads = 512;
static_assert(kGjgThreads == kGjThreads, "gj_cta_invert runs on the whole CTA");
constexpr int kMgDenseGridMax = 1280;  // largest dense coarsest (the grid Gauss-Jordan's strip budget)
constexpr int kGjgMaxStrip = 10;       // columns per CTA strip (the launch uses at least n / 10 CTAs)
static_assert(kMgDenseGridMax <= 3 * kGjgThreads, "the grid Gauss-Jordan updates three rows per thread");

template <int W>
__global__ void __launch_bounds__(kGjgThreads) k_gauss_jordan_grid(int n, double* __restrict__ M, double* __restrict__ panel,
                                                                   unsigned long long* bar, unsigned long long* dmax_bits, int* err,
                                                                   long long limit) {
    extern __shared__ double gsm[];
    __shared__ double Dm[kGjBlock * kGjDS];
    __shared__ double R[kGjBlock * W];  // the block rows' new values on the strip (rows past the block: 0)
    __shared__ double gj_fcol[kGjBlock], gj_frow[kGjBlock];
    __shared__ int s_ok;
    const int G = gridDim.x, t = threadIdx.x;
    const int c0 = (int)((long long)n * blockIdx.x / G), c1 = (int)((long long)n * (blockIdx.x + 1) / G), w = c1 - c0;
    double* S = gsm;  // the strip, column-major: S[jj * n + i] = M[i][c0 + jj]
    unsigned long long target = 0;
    // the strip, its regularised diagonal, and the largest diagonal (the drop threshold)
    for (int e = t; e < n * w; e += kGjgThreads) {
        const int i = e / w, jj = e % w;
        double v = M[(size_t)i * n + c0 + jj];
        if (i == c0 + jj) v *= (1.0 + 1e-8);
        S[(size_t)jj * n + i] = v;
    }
    if (t == 0) {
        double m = 0;
        for (int jj = 0; jj < w; jj++) m = fmax(m, fabs(M[(size_t)(c0 + jj) * n + c0 + jj]));
        atomicMax(dmax_bits, (unsigned long long)__double_as_longlong(m));  // non-negative: the bits order as the values
    }
    __syncthreads();
    // panel of block 0 (columns 0 .. 31, column-major; columns past n are zero) from the strips holding them
    for (int e = t; e < n * w; e += kGjgThreads) {
        const int jj = e / n, i = e % n, j = c0 + jj;
        if (j < kGjBlock) panel[(size_t)j * n + i] = S[e];
    }
    if (blockIdx.x == 0)
        for (int e = n * n < kGjBlock * n ? n * n + t : kGjBlock * n; e < kGjBlock * n; e += kGjgThreads) panel[e] = 0.0;
    if (!mg_sync(bar, target, err, &s_ok, limit)) return;
    const double thr = 1e-12 * __longlong_as_double((long long)__ldcg(dmax_bits));
    const int nblk = (n + kGjBlock - 1) / kGjBlock;
    for (int bk = 0; bk < nblk; bk++) {
        const int b0 = bk * kGjBlock, m = min(kGjBlock, n - b0);
        const double* P = panel + (size_t)(bk & 1) * n * kGjBlock;  // P[kk * n + i] = S[i][b0 + kk] (0 for kk >= m)
        double* Pn = panel + (size_t)((bk + 1) & 1) * n * kGjBlock;
        for (int e = t; e < kGjBlock * kGjBlock; e += kGjgThreads) {
            const int c = e / kGjBlock, r = e % kGjBlock;
            Dm[r * kGjDS + c] = (r < m && c < m) ? __ldcg(&P[(size_t)c * n + b0 + r]) : (r == c ? 1.0 : 0.0);
        }
        __syncthreads();
        gj_cta_invert(Dm, gj_fcol, gj_frow, thr);
        // X = the block rows' new values on the strip: D^-1 S_b,j outside the block, (D^-1)_j inside
        for (int e = t; e < kGjBlock * W; e += kGjgThreads) {
            const int ii = e / W, jj = e % W, j = c0 + jj;
            double v = 0;
            if (ii < m && jj < w) {
                if (j >= b0 && j < b0 + m) {
                    v = Dm[ii * kGjDS + (j - b0)];
                } else {
                    for (int kk = 0; kk < m; kk++) v += Dm[ii * kGjDS + kk] * S[(size_t)jj * n + b0 + kk];
                }
            }
            R[e] = v;
        }
        __syncthreads();
        // rows: three per thread (t, t + 512, t + 1024); S_ij <- (j in the block ? 0 : S_ij) - sum_k S_ik X_kj,
        // the sums over the block's pivots in order; the block's own rows take X
        constexpr int RPT = 3;
        int ri[RPT];
        bool live[RPT], upd[RPT];
#pragma unroll
        for (int q = 0; q < RPT; q++) {
            ri[q] = t + q * kGjgThreads;
            live[q] = ri[q] < n;
            upd[q] = live[q] && !(ri[q] >= b0 && ri[q] < b0 + m);
        }
        double acc[RPT][W];
#pragma unroll
        for (int q = 0; q < RPT; q++)
#pragma unroll
            for (int jj = 0; jj < W; jj++) acc[q][jj] = 0.0;
#pragma unroll
        for (int kc = 0; kc < kGjBlock; kc += 4) {
            double ph[RPT][4];
#pragma unroll
            for (int q = 0; q < RPT; q++)
#pragma unroll
                for (int u = 0; u < 4; u++) ph[q][u] = upd[q] ? __ldcg(&P[(size_t)(kc + u) * n + ri[q]]) : 0.0;
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int jj = 0; jj < W; jj++) {
                    const double x = R[(kc + u) * W + jj];
#pragma unroll
                    for (int q = 0; q < RPT; q++) acc[q][jj] += ph[q][u] * x;
                }
        }
#pragma unroll
        for (int q = 0; q < RPT; q++) {
            if (!live[q]) continue;
            const int i = ri[q];
#pragma unroll
            for (int jj = 0; jj < W; jj++) {
                if (jj >= w) continue;
                const int j = c0 + jj;
                double v;
                if (!upd[q]) {
                    v = R[(i - b0) * W + jj];
                } else {
                    const double old = (j >= b0 && j < b0 + m) ? 0.0 : S[(size_t)jj * n + i];
                    v = old - acc[q][jj];
                }
                S[(size_t)jj * n + i] = v;
            }
        }
        __syncthreads();
        // the next block's panel (columns past n zero) from the strips that hold its columns
        if (bk + 1 < nblk) {
            const int nb0 = b0 + kGjBlock, nm = min(kGjBlock, n - nb0);
            for (int e = t; e < n * w; e += kGjgThreads) {
                const int jj = e / n, i = e % n, j = c0 + jj;
                if (j >= nb0 && j < nb0 + nm) Pn[(size_t)(j - nb0) * n + i] = S[e];
            }
            if (blockIdx.x == 0)
                for (int e = nm * n + t; e < kGjBlock * n; e += kGjgThreads) Pn[e] = 0.0;
        }
        if (!mg_sync(bar, target, err, &s_ok, limit)) return;
    }
    for (int e = t; e < n * w; e += kGjgThreads) {
        const int i = e / w, jj = e % w;
        M[(size_t)i * n + c0 + jj] = S[(size_t)jj * n + i];
    }
}

// Cluster variant: the hardware cluster barrier (release/acquire at cluster
// scope orders the global-memory writes of all CTAs of the cluster).
template <bool CL>
__device__ __forceinline__ bool sync_all(unsigned long long* bar, unsigned long long& target, int* err, int* s_ok, long long limit) {
    if constexpr (CL) {
        asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
        asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
        return true;
    } else {
        return mg_sync(bar, target, err, s_ok, limit);
    }
}

__device__ __forceinline__ void mg_reduce1(double a, double* sm, double& ra) {
    a = warp_sum(a);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = a;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        double x = lane < nw ? sm[lane] : 0.0;
        x = warp_sum(x);
        if (lane == 0) sm[64] = x;
    }
    __syncthreads();
    ra = sm[64];
    __syncthreads();
}

__device__ __forceinline__ double mg_sum_partials(const double* part, int nb, double* sm) {
    if (threadIdx.x < 32) {
        double a = 0;
        for (int i = threadIdx.x; i < nb; i += 32) a += __ldcg(&part[i]);
        a = warp_sum(a);
        if (threadIdx.x == 0) sm[66] = a;
    }
    __syncthreads();
    const double s = sm[66];
    __syncthreads();
    return s;
}

__device__ __forceinline__ double group_sum(double v, unsigned mask) {
    for (int o = kGroup / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, kGroup);
    return v;
}

// Gathered dot products of the solve phases.  The entries of a chunk (U per
// thread) have their column indices and values loaded first and their vector
// entries second, so a chunk costs two dependent L2 round trips instead of two
// per entry; the sum still runs in entry order.  Vectors other CTAs write are
// read with __ldcg (L2).
template <int U>
__device__ __forceinline__ double gather_dot(const int32_t* __restrict__ ci, const double* __restrict__ v, const double* x, int b, int e,
                                             int first = 0, int step = 1) {
    double s = 0;
    for (int k0 = b + first; k0 < e; k0 += U * step) {
        int c[U];
        double w[U], xv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = k0 + u * step;
            c[u] = k < e ? ci[k] : 0;
            w[u] = k < e ? v[k] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) xv[u] = (k0 + u * step < e) ? __ldcg(&x[c[u]]) : 0.0;
#pragma unroll
        for (int u = 0; u < U; u++) s += w[u] * xv[u];
    }
    return s;
}

// sum_k v[k] (x[ci[k]] + y[cg[k]])
template <int U>
__device__ __forceinline__ double gather_dot2(const int32_t* __restrict__ ci, const int32_t* __restrict__ cg, const double* __restrict__ v,
                                              const double* x, const double* y, int b, int e, int first = 0, int step = 1) {
    double s = 0;
    for (int k0 = b + first; k0 < e; k0 += U * step) {
        int c[U], g[U];
        double w[U], xv[U], yv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = k0 + u * step;
            c[u] = k < e ? ci[k] : 0;
            g[u] = k < e ? cg[k] : 0;
            w[u] = k < e ? v[k] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool ok = k0 + u * step < e;
            xv[u] = ok ? __ldcg(&x[c[u]]) : 0.0;
            yv[u] = ok ? __ldcg(&y[g[u]]) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) s += w[u] * (xv[u] + yv[u]);
    }
    return s;
}

// sum_m x[idx[m]]
template <int U>
__device__ __forceinline__ double gather_sum(const int32_t* __restrict__ idx, const double* x, int b, int e, int first, int step) {
    double s = 0;
    for (int k0 = b + first; k0 < e; k0 += U * step) {
        int c[U];
        double xv[U];
#pragma unroll
        for (int u = 0; u < U; u++) c[u] = (k0 + u * step < e) ? idx[k0 + u * step] : 0;
#pragma unroll
        for (int u = 0; u < U; u++) xv[u] = (k0 + u * step < e) ? __ldcg(&x[c[u]]) : 0.0;
#pragma unroll
        for (int u = 0; u < U; u++) s += xv[u];
    }
    return s;
}

__device__ __forceinline__ double block_apply(const MgArgs& a, const double* __restrict__ v, int i) {
    const int off = a.row_off[i], base = a.row_base[i], m = a.row_m[i];
    double s = 0;
    for (int j = 0; j < m; j++) s += a.tinv[off + j] * v[base + j];
    return s;
}

// One MG-PCG solve by `nctas` CTAs (this is CTA `cta` of them).
template <bool CL>
__device__ void mg_pcg_body(const MgArgs& a, int cta, int nctas) {
    __shared__ double sm[72];
    __shared__ MgLevel lv[kMgMaxLevels];
    __shared__ double rc[kMgDenseMax];
    __shared__ int s_ok;
    if (threadIdx.x < a.levels) lv[threadIdx.x] = a.lv[threadIdx.x];
    __syncthreads();
    const int C = a.levels - 1;
    const int nb = nctas;
    const int gt = cta * blockDim.x + threadIdx.x, gs = nctas * blockDim.x;
    const int grp = gt / kGroup, glane = gt % kGroup, ngrp = gs / kGroup;
    const unsigned gmask = ((1u << kGroup) - 1) << ((threadIdx.x & 31) & ~(kGroup - 1));
    const int r_lo = a.cta_row[cta], r_hi = a.cta_row[cta + 1];
    if (a.x0) {  // start from x0: x = x0, r = b - A x0 (own rows; x0 is read-only, no barrier needed)
        for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
            double s = 0;
            for (int kk = a.rp[i]; kk < a.rp[i + 1]; kk++) s += a.val[kk] * a.x0[a.ci[kk]];
            a.x[i] = a.x0[i];
            a.r[i] = a.b[i] - s;
        }
    }
    unsigned long long target = 0;
    double R0 = 0, rr = 0, rz = 0, beta = 0, bnorm = 0;
    if (a.cap_b) {  // |b| (partB is next written after the first barrier of the loop)
        double bb_l = 0;
        for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) bb_l += a.b[i] * a.b[i];
        double s0;
        mg_reduce1(bb_l, sm, s0);
        if (threadIdx.x == 0) a.partB[cta] = s0;
        if (!sync_all<CL>(a.bar, target, a.err, &s_ok, a.spin_limit)) return;
        bnorm = sqrt(mg_sum_partials(a.partB, nb, sm));
    }
    long long k = 0;
    int restarts = 0;
    bool fresh = true;      // p = z, q = A z on the next direction update
    bool recursive = false; // r is the recursively updated residual (not b - A x)
    while (true) {
        // ---- pre-smoother z0 = w M0^-1 r on own rows; r.r ----
        __syncthreads();
        double rr_l = 0;
        for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
            a.z0[i] = a.omega0 * block_apply(a, a.r, i);
            const double ri = a.r[i];
            rr_l += ri * ri;
        }
        double s0;
        mg_reduce1(rr_l, sm, s0);
        if (threadIdx.x == 0) a.partA[cta] = s0;
        if (!sync_all<CL>(a.bar, target, a.err, &s_ok, a.spin_limit)) return;
        rr = mg_sum_partials(a.partA, nb, sm);
        if (k == 0 && !recursive && restarts == 0) R0 = a.tol * (a.cap_b ? fmin(sqrt(rr), bnorm) : sqrt(rr));
        if (k > 0 && sqrt(rr) <= R0) {
            if (!recursive || restarts >= a.max_restarts) break;
            // the recursive residual met the test: replace it by the FP64 true residual
            for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
                a.r[i] = a.b[i] - gather_dot<4>(a.ci, a.val, a.x, a.rp[i], a.rp[i + 1]);
            }
            restarts++;
            recursive = false;
            fresh = true;
            continue;
        }
        if (k >= a.max_iter) break;
        // ---- restriction 0 -> 1 inside the CTA (its blocks are its own rows) ----
        {
            const MgLevel& F = lv[0];
            const MgLevel& G = lv[1];
            for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
                a.w[i] = a.r[i] - gather_dot<4>(a.ci, a.val, a.z0, a.rp[i], a.rp[i + 1]);
            }
            __syncthreads();
            const bool smooth = (C > 1) || a.cinv == nullptr;
            if (r_hi > r_lo) {
                const int b0 = F.agg[r_lo], b1 = F.agg[r_hi - 1];
                for (int J = b0 + threadIdx.x; J <= b1; J += blockDim.x) {
                    double s = 0;
                    for (int m = F.mptr[J]; m < F.mptr[J + 1]; m++) s += a.w[F.midx[m]];
                    G.r[J] = s;
                    if (smooth) G.z[J] = G.l1inv[J] * s;
                }
            }
            if (!sync_all<CL>(a.bar, target, a.err, &s_ok, a.spin_limit)) return;
        }
        // ---- restrictions l -> l+1 (l >= 1): r_{l+1} = P^T r_l - (P^T A_l) z_l ----
        for (int l = 1; l < C; l++) {
            const MgLevel& F = lv[l];
            const MgLevel& G = lv[l + 1];
            const bool smooth = (l + 1 < C) || a.cinv == nullptr;
            for (int J = grp; J < G.n; J += ngrp) {
                double s = gather_sum<2>(F.midx, F.r, F.mptr[J], F.mptr[J + 1], glane, kGroup) -
                           gather_dot<4>(F.ra_col, F.ra_val, F.z, F.ra_ptr[J], F.ra_ptr[J + 1], glane, kGroup);
                s = group_sum(s, gmask);
                if (glane == 0) {
                    G.r[J] = s;
                    if (smooth) G.z[J] = G.l1inv[J] * s;
                }
            }
            if (!sync_all<CL>(a.bar, target, a.err, &s_ok, a.spin_limit)) return;
        }
        // ---- coarsest: dense inverse, one warp per row ----
        if (a.cinv) {
            const MgLevel& Cl = lv[C];
            const int nC = Cl.n;
            const int wpb = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
            if (cta * wpb < nC) {
                for (int j = threadIdx.x; j < nC; j += blockDim.x) rc[j] = __ldcg(&Cl.r[j]);
                __syncthreads();
                for (int i = cta * wpb + warp; i < nC; i += nctas * wpb) {
                    const double* row = a.cinv + (size_t)i * nC;
                    double s = 0;
                    for (int j = lane; j < nC; j += 32) s += row[j] * rc[j];
                    s = warp_sum(s);
                    if (lane == 0) Cl.zf[i] = s;
                }
            }
            if (!sync_all<CL>(a.bar, target, a.err, &s_ok, a.spin_limit)) return;
        }
        // ---- prolongation + l1-Jacobi post-smoother, levels C-1 .. 1 ----
        for (int l = C - 1; l >= 1; l--) {
            const MgLevel& F = lv[l];
            const double* zc = lv[l + 1].zf;
            for (int I = grp; I < F.n; I += ngrp) {
                double w = -gather_dot2<4>(F.ci, F.cagg, F.val, F.z, zc, F.rp[I], F.rp[I + 1], glane, kGroup);
                w = group_sum(w, gmask);
                if (glane == 0) {
                    const double zp = __ldcg(&F.z[I]) + __ldcg(&zc[F.agg[I]]);
                    w += __ldcg(&F.r[I]) - F.diag[I] * zp;
                    F.zf[I] = zp + F.l1inv[I] * w;
                }
            }
            if (!sync_all<CL>(a.bar, target, a.err, &s_ok, a.spin_limit)) return;
        }
        // ---- level-0 post-smoother: z = z0 + P z1, z += w M0^-1 (r - A z); r.z ----
        {
            const double* zc = lv[1].zf;
            const int32_t* agg = lv[0].agg;
            const int32_t* cagg = lv[0].cagg;
            for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
                a.w[i] = a.r[i] - gather_dot2<4>(a.ci, cagg, a.val, a.z0, zc, a.rp[i], a.rp[i + 1]);
                a.z[i] = a.z0[i] + __ldcg(&zc[agg[i]]);
            }
            __syncthreads();
            double rz_l = 0;
            for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
                const double zi = a.z[i] + a.omega0 * block_apply(a, a.w, i);
                a.z[i] = zi;
                rz_l += a.r[i] * zi;
            }
            mg_reduce1(rz_l, sm, s0);
            if (threadIdx.x == 0) a.partB[cta] = s0;
            if (!sync_all<CL>(a.bar, target, a.err, &s_ok, a.spin_limit)) return;
            const double rz_new = mg_sum_partials(a.partB, nb, sm);
            beta = fresh ? 0.0 : rz_new / rz;
            rz = rz_new;
        }
        // ---- q = A z + beta q, p = z + beta p; p.q ----
        double pq_l = 0;
        for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
            const double w = gather_dot<4>(a.ci, a.val, a.z, a.rp[i], a.rp[i + 1]);
            const double zi = a.z[i];
            const double qi = fresh ? w : w + beta * a.q[i];
            const double pi = fresh ? zi : zi + beta * a.p[i];
            a.q[i] = qi;
            a.p[i] = pi;
            pq_l += pi * qi;
        }
        mg_reduce1(pq_l, sm, s0);
        if (threadIdx.x == 0) a.partA[nb + cta] = s0;
        if (!sync_all<CL>(a.bar, target, a.err, &s_ok, a.spin_limit)) return;
        const double pq = mg_sum_partials(a.partA + nb, nb, sm);
        fresh = false;
        k++;
        // ---- x += alpha p, r -= alpha q ----
        const double alpha = rz / pq;
        for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
            a.x[i] += alpha * a.p[i];
            a.r[i] -= alpha * a.q[i];
        }
        recursive = true;
    }
    if (cta == 0 && threadIdx.x == 0) {
        a.stats[0] = (double)k;
        a.stats[1] = rr;
        a.stats[2] = R0;
        a.stats[3] = (double)restarts;
    }
}

template <bool CL>
__global__ void __launch_bounds__(CL ? kMgClusterThreads : kMgThreads) k_mg_pcg(MgArgs a) {
    mg_pcg_body<CL>(a, blockIdx.x, gridDim.x);
}

// Batched solves: every 16-CTA cluster takes the next system of the queue and
// runs the MG-PCG on it; `slots` passes the index from cluster rank 0 to the others.
__global__ void __launch_bounds__(kMgClusterThreads) k_mg_batch(const MgArgs* __restrict__ all, int count, int* queue, int* slots) {
    const int cl = blockIdx.x / kMgClusterCtas, rank = blockIdx.x % kMgClusterCtas;
    while (true) {
        if (rank == 0 && threadIdx.x == 0) slots[cl] = atomicAdd(queue, 1);
        asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
        asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
        const int s = __ldcg(&slots[cl]);
        asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
        asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
        if (s >= count) return;
        const MgArgs a = all[s];
        mg_pcg_body<true>(a, rank, kMgClusterCtas);
    }
}

// ---------------------------------------------------------------------------
// Shared-memory-resident clustered grid kernel for systems above one cluster's size.
//
// The grid is K clusters of kSmCtas CTAs, one CTA per SM (cooperative launch).  Every
// operator of the V-cycle is static during the solve, so each CTA copies once, at launch,
// the rows it owns into shared memory: its level-0 rows (CSR, column aggregates, chain-block
// inverses, aggregate ranges) with the CG vectors of those rows, and its share of the fused
// restriction / prolongation rows of every coarse level.  A phase then costs one round trip
// for the vector entries other CTAs wrote, plus its barrier, instead of three to six
// dependent L2 round trips for indices, weights and vectors.  Levels lc .. coarsest (at most
// kSmRows rows at lc) are solved by every cluster on its own copy of their vectors between
// hardware cluster barriers (~0.3 us) instead of grid barriers (~1.1 us plus skew).  A row
// set that does not fit the shared-memory budget is read from global memory instead.
constexpr int kSmCtas = 8;          // CTAs per cluster (portable size)
constexpr int kSmThreads = 512;
constexpr int kSmRows = 1000;       // largest level the clusters solve alone
constexpr int kSmMaxClusters = 18;  // 144 CTAs
constexpr int kSmBytes = 200 * 1024;

struct MgSmLevel {
    int n;
    const int32_t* rr_ptr;  // fused restriction rows into level l + 1 (1 <= l < coarsest)
    const int32_t* rr_col;
    const double* rr_val;
    const int32_t* pq_ptr;  // fused prolongation-smoother rows of level l (1 <= l < coarsest)
    const int32_t* pq_col;
    const double* pq_val;
    const int32_t* agg;
    const double* l1inv;
    double* r;
    double* z;
    double* zf;
    int priv;      // bit 0: r and z per cluster (stride n), bit 1: zf per cluster
    int rr_lanes;  // lanes per restriction row into l + 1 / per prolongation row of l (powers of two)
    int pq_lanes;
};

struct MgSmArgs {
    int lc;                  // first level the clusters solve alone (>= 1)
    const MgSmLevel* lv;     // levels 0 .. coarsest
    int* cl_fail;            // per cluster: a grid-barrier wait of one of its CTAs gave up
    const int32_t* mptr0;    // level-0 aggregates (the chain blocks): first row of each, then n
    int smem_bytes;          // dynamic shared memory of the launch
    int grid_coarse;         // dense coarsest solved by all CTAs between grid barriers (lc = coarsest, no clusters)
};

// Rows [lo, hi) of one fused operator.  ptr[i - lo] - sub and ptr[i - lo + 1] - sub bound the
// entries of row i in col / val; agg and l1inv are indexed by i - lo.  Staged copies have
// sub = 0; a set read from global memory points into the global arrays with sub = ptr[lo].
struct SmRows {
    int lo, hi, sub;
    const int32_t* ptr;
    const int32_t* col;
    const double* val;
    const int32_t* agg;
    const double* l1inv;
};

// The CTA's level-0 rows [lo, hi): CSR (entries ent_sub-based), column aggregates, chain-block
// inverse rows (tinv, row offsets tofs-based, block bases lo-based), aggregates alo .. ahi with
// their row ranges (lo-based), and the CG vectors of its rows (lo-based).
struct SmL0 {
    int lo, hi, alo, ahi;
    int rp_sub, roff_sub, rbase_sub, mptr_sub;
    const int32_t *rp, *ci, *cagg, *roff, *rbase, *rm, *agg, *mptr;
    const double *val, *tinv, *b;
    double *r, *x, *p, *q, *z, *z0, *w;
};

struct SmPlan {
    SmL0 l0;
    SmRows R[kMgMaxLevels];  // restriction rows into level l + 1 (index l)
    SmRows Q[kMgMaxLevels];  // prolongation rows of level l
    int clo, chi;            // coarsest rows of this CTA (dense inverse rows)
    const double* cinv;      // its rows, (i - clo) * nC based
    unsigned int used;
};

struct SmStage {  // one copy from global into shared memory
    void* dst;
    const void* src;
    int count, elem, rebase;  // elem 4: int32 (minus rebase), 8: double
};

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Grid barrier (bounded).  A CTA whose wait gave up marks its cluster and carries on through
// the iteration with the same control flow (its data are then stale, the device status says
// why); sm_cluster_ok, once per iteration before the first data-dependent branch, lets every
// CTA of a marked cluster leave together, so no cluster barrier ever waits on a CTA that has
// returned and no CTA branches on partial sums another CTA of its cluster read differently.
__device__ __forceinline__ void sm_sync(const MgArgs& a, int* cl_fail, unsigned long long& target, int cid, int* s_ok) {
    if (!mg_sync(a.bar, target, a.err, s_ok, a.spin_limit) && threadIdx.x == 0) atomicExch(&cl_fail[cid], 1);
}

__device__ __forceinline__ bool sm_cluster_ok(const int* cl_fail, int cid) {
    cluster_sync_all();
    return __ldcg(&cl_fail[cid]) == 0;
}

// sum_k val[k] v(col[k]) with v(c) = v0[c] for c < n, else v1[c - n]; chunks of U entries
// per lane (indices and weights first, vector entries second).
template <int U>
__device__ __forceinline__ double fused_dot(const int32_t* col, const double* val, int b, int e, int first, int step, int n,
                                            const double* v0, const double* v1) {
    double s = 0;
    for (int k0 = b + first; k0 < e; k0 += U * step) {
        int c[U];
        double w[U], xv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = k0 + u * step;
            c[u] = k < e ? col[k] : 0;
            w[u] = k < e ? val[k] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) xv[u] = (k0 + u * step < e) ? (c[u] < n ? __ldcg(&v0[c[u]]) : __ldcg(&v1[c[u] - n])) : 0.0;
#pragma unroll
        for (int u = 0; u < U; u++) s += w[u] * xv[u];
    }
    return s;
}

// Level-0 row gather: sum_q val[q] v(ci[q]) over entries [b, e), v(c) = vs[c - lo] for the
// CTA's own rows [lo, hi) (shared memory), else the global vector vg; with zc, each entry also
// adds zc[cagg[q]].  Chunks of U entries: indices and weights first, vector entries second.
template <int U>
__device__ __forceinline__ double own_dot(const int32_t* ci, const double* val, const int32_t* cagg, int b, int e, int lo, int hi,
                                          const double* vs, const double* vg, const double* zc) {
    double s = 0;
    for (int q0 = b; q0 < e; q0 += U) {
        int c[U], g[U];
        double w[U], x[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int q = q0 + u;
            c[u] = q < e ? ci[q] : lo;
            w[u] = q < e ? val[q] : 0.0;
            g[u] = (zc && q < e) ? cagg[q] : 0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            x[u] = (c[u] >= lo && c[u] < hi) ? vs[c[u] - lo] : __ldcg(&vg[c[u]]);
            if (zc) x[u] += __ldcg(&zc[g[u]]);
        }
#pragma unroll
        for (int u = 0; u < U; u++) s += w[u] * x[u];
    }
    return s;
}

// Sum of the nb per-CTA partials: one load per thread, then the CTA reduction.
__device__ __forceinline__ double sm_sum_partials(const double* part, int nb, double* sm) {
    double v = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) v += __ldcg(&part[i]);
    double r;
    mg_reduce1(v, sm, r);
    return r;
}

__device__ __forceinline__ double lanes_sum(double v, int lanes) {
    const unsigned mask = lanes >= 32 ? 0xffffffffu : (((1u << lanes) - 1) << ((threadIdx.x & 31) & ~(lanes - 1)));
    for (int o = lanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, lanes);
    return v;
}

// r_{l+1} = P^T (r_l - A_l z_l) and its l1-Jacobi smoothing on the rows of R.
__device__ __forceinline__ void sm_restrict(const SmRows& R, int lanes, int nF, const double* rF, const double* zF, double* rG, double* zG,
                                            bool smooth) {
    const int grp = threadIdx.x / lanes, gl = threadIdx.x % lanes, ngrp = blockDim.x / lanes;
    for (int J = R.lo + grp; J < R.hi; J += ngrp) {
        const int j = J - R.lo;
        double v = fused_dot<4>(R.col, R.val, R.ptr[j] - R.sub, R.ptr[j + 1] - R.sub, gl, lanes, nF, rF, zF);
        v = lanes_sum(v, lanes);
        if (gl == 0) {
            rG[J] = v;
            if (smooth) zG[J] = R.l1inv[j] * v;
        }
    }
}

// zp = z_l + P zc, zf_l = zp + D^-1 (r_l - A_l zp) on the rows of Q.
__device__ __forceinline__ void sm_prolong(const SmRows& Q, int lanes, int nF, const double* rF, const double* zF, const double* zc, double* zf) {
    const int grp = threadIdx.x / lanes, gl = threadIdx.x % lanes, ngrp = blockDim.x / lanes;
    for (int I = Q.lo + grp; I < Q.hi; I += ngrp) {
        const int i = I - Q.lo;
        double zp = 0, rI = 0;
        if (gl == 0) {
            zp = __ldcg(&zF[I]) + __ldcg(&zc[Q.agg[i]]);
            rI = __ldcg(&rF[I]);
        }
        double v = fused_dot<4>(Q.col, Q.val, Q.ptr[i] - Q.sub, Q.ptr[i + 1] - Q.sub, gl, lanes, nF, zF, zc);
        v = lanes_sum(v, lanes);
        if (gl == 0) zf[I] = zp + Q.l1inv[i] * (rI - v);
    }
}

// Thread 0: place rows [lo, hi) of (ptr, col, val) plus optional per-row agg / l1inv into the
// shared budget, or point at global memory; records the copies in st[] (returns their count).
__device__ int sm_place_rows(SmRows& R, int lo, int hi, const int32_t* ptr, const int32_t* col, const double* val, const int32_t* agg,
                             const double* l1inv, unsigned char* base, unsigned int cap, unsigned int& used, SmStage* st, int ns, int max_st) {
    R.lo = lo;
    R.hi = hi;
    R.agg = agg ? agg + lo : nullptr;
    R.l1inv = l1inv ? l1inv + lo : nullptr;
    if (hi <= lo || !ptr) {
        R.ptr = ptr ? ptr + lo : nullptr;
        R.col = col;
        R.val = val;
        R.sub = 0;
        return ns;
    }
    const int e0 = ptr[lo], e1 = ptr[hi], E = e1 - e0, nr = hi - lo;
    auto al = [](unsigned int u) { return (u + 15u) & ~15u; };
    unsigned int u = al(used);
    const unsigned int o_ptr = u;
    u = al(u + 4u * (nr + 1));
    const unsigned int o_col = u;
    u = al(u + 4u * E);
    const unsigned int o_val = u;
    u = al(u + 8u * E);
    const unsigned int o_agg = u;
    if (agg) u = al(u + 4u * nr);
    const unsigned int o_l1 = u;
    if (l1inv) u = al(u + 8u * nr);
    if (u > cap || ns + 5 > max_st) {  // read from global memory
        R.ptr = ptr + lo;
        R.col = col + e0;
        R.val = val + e0;
        R.sub = e0;
        return ns;
    }
    used = u;
    R.ptr = reinterpret_cast<const int32_t*>(base + o_ptr);
    R.col = reinterpret_cast<const int32_t*>(base + o_col);
    R.val = reinterpret_cast<const double*>(base + o_val);
    R.sub = 0;
    st[ns++] = SmStage{base + o_ptr, ptr + lo, nr + 1, 4, e0};
    st[ns++] = SmStage{base + o_col, col + e0, E, 4, 0};
    st[ns++] = SmStage{base + o_val, val + e0, E, 8, 0};
    if (agg) {
        R.agg = reinterpret_cast<const int32_t*>(base + o_agg);
        st[ns++] = SmStage{base + o_agg, agg + lo, nr, 4, 0};
    }
    if (l1inv) {
        R.l1inv = reinterpret_cast<const double*>(base + o_l1);
        st[ns++] = SmStage{base + o_l1, l1inv + lo, nr, 8, 0};
    }
    return ns;
}

constexpr int kSmMaxStages = 160;

__global__ void __launch_bounds__(kSmThreads) k_mg_pcg_sm(MgArgs a, MgSmArgs sa) {
    extern __shared__ __align__(16) unsigned char sm_dyn[];
    __shared__ double sm[72];
    __shared__ MgSmLevel lv[kMgMaxLevels];
    __shared__ SmPlan P;
    __shared__ SmStage st[kSmMaxStages];
    __shared__ int n_st;
    __shared__ int s_ok;
    __shared__ double rc[kMgDenseGridMax];
    const int cta = blockIdx.x, nb = gridDim.x;
    const int cid = cta / kSmCtas, crank = cta % kSmCtas;
    const int C = a.levels - 1, Lc = sa.lc;
    if (threadIdx.x < a.levels) {
        MgSmLevel L = sa.lv[threadIdx.x];
        if (L.priv & 1) {
            L.r += (size_t)cid * L.n;
            L.z += (size_t)cid * L.n;
        }
        if (L.priv & 2) L.zf += (size_t)cid * L.n;
        lv[threadIdx.x] = L;
    }
    __syncthreads();
    // ---- placement (thread 0), then the copies (all threads) ----
    if (threadIdx.x == 0) {
        const unsigned int cap = (unsigned int)sa.smem_bytes;
        unsigned int used = 0;
        int ns = 0;
        auto al = [](unsigned int u) { return (u + 15u) & ~15u; };
        auto take = [&](unsigned int bytes) -> unsigned char* {
            const unsigned int u = al(used);
            if (u + bytes > cap) return nullptr;
            used = u + bytes;
            return sm_dyn + u;
        };
        SmL0& L = P.l0;
        const MgLevel& G0 = a.lv[0];
        L.lo = a.cta_row[cta];
        L.hi = a.cta_row[cta + 1];
        const int nr = L.hi - L.lo;
        // vectors of the own rows (x, r from global; the others are written before read)
        double* vec = nr > 0 ? reinterpret_cast<double*>(take(8u * 7 * nr)) : nullptr;
        if (vec) {
            L.r = vec; L.x = vec + nr; L.p = vec + 2 * nr; L.q = vec + 3 * nr; L.z = vec + 4 * nr; L.z0 = vec + 5 * nr; L.w = vec + 6 * nr;
            st[ns++] = SmStage{L.r, a.r + L.lo, nr, 8, 0};
            st[ns++] = SmStage{L.x, a.x + L.lo, nr, 8, 0};
        } else {
            L.r = a.r + L.lo; L.x = a.x + L.lo; L.p = a.p + L.lo; L.q = a.q + L.lo; L.z = a.z + L.lo; L.z0 = a.z0 + L.lo; L.w = a.w + L.lo;
        }
        L.b = a.b + L.lo;
        // CSR rows with their column aggregates
        const int e0 = nr > 0 ? a.rp[L.lo] : 0, E = nr > 0 ? a.rp[L.hi] - e0 : 0;
        unsigned char* m_rp = nr > 0 ? take(4u * (nr + 1)) : nullptr;
        unsigned char* m_ci = m_rp ? take(4u * E) : nullptr;
        unsigned char* m_cg = m_ci ? take(4u * E) : nullptr;
        unsigned char* m_v = m_cg ? take(8u * E) : nullptr;
        if (m_v) {
            L.rp = reinterpret_cast<const int32_t*>(m_rp); L.rp_sub = 0;
            L.ci = reinterpret_cast<const int32_t*>(m_ci);
            L.cagg = reinterpret_cast<const int32_t*>(m_cg);
            L.val = reinterpret_cast<const double*>(m_v);
            st[ns++] = SmStage{m_rp, a.rp + L.lo, nr + 1, 4, e0};
            st[ns++] = SmStage{m_ci, a.ci + e0, E, 4, 0};
            st[ns++] = SmStage{m_cg, G0.cagg + e0, E, 4, 0};
            st[ns++] = SmStage{m_v, a.val + e0, E, 8, 0};
        } else {
            L.rp = a.rp + L.lo; L.rp_sub = e0;
            L.ci = a.ci + e0; L.cagg = G0.cagg + e0; L.val = a.val + e0;
        }
        // row -> aggregate, and the own aggregates' row ranges
        L.alo = nr > 0 ? G0.agg[L.lo] : 0;
        L.ahi = nr > 0 ? G0.agg[L.hi - 1] + 1 : 0;
        const int na = L.ahi - L.alo;
        unsigned char* m_ag = nr > 0 ? take(4u * nr) : nullptr;
        unsigned char* m_mp = m_ag ? take(4u * (na + 1)) : nullptr;
        if (m_mp) {
            L.agg = reinterpret_cast<const int32_t*>(m_ag);
            L.mptr = reinterpret_cast<const int32_t*>(m_mp); L.mptr_sub = 0;
            st[ns++] = SmStage{m_ag, G0.agg + L.lo, nr, 4, 0};
            st[ns++] = SmStage{m_mp, sa.mptr0 + L.alo, na + 1, 4, L.lo};
        } else {
            L.agg = G0.agg + L.lo;
            L.mptr = sa.mptr0 + L.alo; L.mptr_sub = L.lo;
        }
        // chain-block inverse rows (both smoother phases read them: before the coarse rows)
        const int t0 = nr > 0 ? a.row_off[L.lo] : 0;
        const int T = nr > 0 ? a.row_off[L.hi - 1] + a.row_m[L.hi - 1] - t0 : 0;
        unsigned char* m_meta = nr > 0 && ns + 4 <= kSmMaxStages ? take(12u * nr) : nullptr;
        unsigned char* m_t = m_meta ? take(8u * T) : nullptr;
        if (m_t) {
            L.roff = reinterpret_cast<const int32_t*>(m_meta); L.roff_sub = 0;
            L.rbase = L.roff + nr; L.rbase_sub = 0;
            L.rm = L.rbase + nr;
            L.tinv = reinterpret_cast<const double*>(m_t);
            st[ns++] = SmStage{m_meta, a.row_off + L.lo, nr, 4, t0};
            st[ns++] = SmStage{m_meta + 4u * nr, a.row_base + L.lo, nr, 4, L.lo};
            st[ns++] = SmStage{m_meta + 8u * nr, a.row_m + L.lo, nr, 4, 0};
            st[ns++] = SmStage{m_t, a.tinv + t0, T, 8, 0};
        } else {
            L.roff = a.row_off + L.lo; L.roff_sub = t0;
            L.rbase = a.row_base + L.lo; L.rbase_sub = L.lo;
            L.rm = a.row_m + L.lo;
            L.tinv = a.tinv + t0;
        }
        // coarse levels: grid rows below lc, cluster rows from lc on
        auto lanes_for = [](long long entries, int rows) {
            int ln = 2;
            while (ln < 32 && (long long)ln * 4 * rows < entries) ln <<= 1;  // about one chunk of 4 entries per lane
            return ln;
        };
        for (int l = 1; l < C; l++) {
            MgSmLevel& F = lv[l];
            const MgSmLevel& G = lv[l + 1];
            F.rr_lanes = lanes_for(F.rr_ptr[G.n], G.n);
            F.pq_lanes = lanes_for(F.pq_ptr[F.n], F.n);
            const bool sec_r = l >= Lc, sec_q = l >= Lc;
            const int n1 = G.n, n0 = F.n;
            const int rlo = sec_r ? (int)((long long)n1 * crank / kSmCtas) : (int)((long long)n1 * cta / nb);
            const int rhi = sec_r ? (int)((long long)n1 * (crank + 1) / kSmCtas) : (int)((long long)n1 * (cta + 1) / nb);
            ns = sm_place_rows(P.R[l], rlo, rhi, F.rr_ptr, F.rr_col, F.rr_val, nullptr, G.l1inv, sm_dyn, cap, used, st, ns, kSmMaxStages);
            const int qlo = sec_q ? (int)((long long)n0 * crank / kSmCtas) : (int)((long long)n0 * cta / nb);
            const int qhi = sec_q ? (int)((long long)n0 * (crank + 1) / kSmCtas) : (int)((long long)n0 * (cta + 1) / nb);
            ns = sm_place_rows(P.Q[l], qlo, qhi, F.pq_ptr, F.pq_col, F.pq_val, F.agg, F.l1inv, sm_dyn, cap, used, st, ns, kSmMaxStages);
        }
        const int nC = lv[C].n;
        P.clo = sa.grid_coarse ? (int)((long long)nC * cta / nb) : (int)((long long)nC * crank / kSmCtas);
        P.chi = sa.grid_coarse ? (int)((long long)nC * (cta + 1) / nb) : (int)((long long)nC * (crank + 1) / kSmCtas);
        P.cinv = nullptr;
        if (a.cinv) {
            const int cr = P.chi - P.clo;
            unsigned char* m_c = cr > 0 && ns < kSmMaxStages ? take(8u * cr * nC) : nullptr;
            if (m_c) {
                P.cinv = reinterpret_cast<const double*>(m_c);
                st[ns++] = SmStage{m_c, a.cinv + (size_t)P.clo * nC, cr * nC, 8, 0};
            } else {
                P.cinv = a.cinv + (size_t)P.clo * nC;
            }
        }
        P.used = used;
        n_st = ns;
    }
    __syncthreads();
    for (int q = 0; q < n_st; q++) {
        const SmStage S = st[q];
        if (S.elem == 8) {
            double* d = static_cast<double*>(S.dst);
            const double* g = static_cast<const double*>(S.src);
            for (int i = threadIdx.x; i < S.count; i += blockDim.x) d[i] = g[i];
        } else {
            int32_t* d = static_cast<int32_t*>(S.dst);
            const int32_t* g = static_cast<const int32_t*>(S.src);
            for (int i = threadIdx.x; i < S.count; i += blockDim.x) d[i] = g[i] - S.rebase;
        }
    }
    __syncthreads();
    const SmL0& L = P.l0;
    const int lo = L.lo, hi = L.hi;
    // chain-block inverse row of own row li applied to a vector of own rows
    auto block_row = [&](int li, const double* v) {
        const int off = L.roff[li] - L.roff_sub, base = L.rbase[li] - L.rbase_sub, m = L.rm[li];
        double s = 0;
        for (int j = 0; j < m; j++) s += L.tinv[off + j] * v[base + j];
        return s;
    };
    auto row_b = [&](int li) { return L.rp[li] - L.rp_sub; };
    unsigned long long target = 0;
    double R0 = 0, rr = 0, rz = 0, beta = 0;
    long long k = 0;
    int restarts = 0;
    bool fresh = true;
    bool recursive = false;
    double s0;
    while (true) {
        // ---- pre-smoother z0 = w M0^-1 r on own rows; r.r ----
        __syncthreads();
        double rr_l = 0;
        for (int li = threadIdx.x; li < hi - lo; li += blockDim.x) {
            const double z0 = a.omega0 * block_row(li, L.r);
            L.z0[li] = z0;
            a.z0[lo + li] = z0;
            const double ri = L.r[li];
            rr_l += ri * ri;
        }
        mg_reduce1(rr_l, sm, s0);
        if (threadIdx.x == 0) a.partA[cta] = s0;
        sm_sync(a, sa.cl_fail, target, cid, &s_ok);
        if (!sa.grid_coarse && !sm_cluster_ok(sa.cl_fail, cid)) break;
        rr = sm_sum_partials(a.partA, nb, sm);
        if (k == 0 && !recursive && restarts == 0) R0 = a.tol * sqrt(rr);
        if (k > 0 && sqrt(rr) <= R0) {
            if (!recursive || restarts >= a.max_restarts) break;
            // the recursive residual met the test: replace it by the FP64 true residual
            for (int li = threadIdx.x; li < hi - lo; li += blockDim.x)
                L.r[li] = L.b[li] - own_dot<4>(L.ci, L.val, nullptr, row_b(li), row_b(li + 1), lo, hi, L.x, a.x, nullptr);
            restarts++;
            recursive = false;
            fresh = true;
            continue;
        }
        if (k >= a.max_iter) break;
        // ---- w = r - A z0; level 0 -> 1 over the own aggregates (the chain blocks) ----
        {
            for (int li = threadIdx.x; li < hi - lo; li += blockDim.x)
                L.w[li] = L.r[li] - own_dot<4>(L.ci, L.val, nullptr, row_b(li), row_b(li + 1), lo, hi, L.z0, a.z0, nullptr);
            __syncthreads();
            const MgSmLevel& G = lv[1];
            const bool smooth = (C > 1) || a.cinv == nullptr;
            for (int J = L.alo + threadIdx.x; J < L.ahi; J += blockDim.x) {
                const int j = J - L.alo;
                const int m0 = L.mptr[j] - L.mptr_sub, m1 = L.mptr[j + 1] - L.mptr_sub;
                double v = 0;
                for (int m = m0; m < m1; m++) v += L.w[m];
                G.r[J] = v;
                if (smooth) G.z[J] = G.l1inv[J] * v;
            }
            sm_sync(a, sa.cl_fail, target, cid, &s_ok);
        }
        // ---- restrictions l -> l + 1 grid-wide (1 <= l < lc) ----
        for (int l = 1; l < Lc; l++) {
            sm_restrict(P.R[l], lv[l].rr_lanes, lv[l].n, lv[l].r, lv[l].z, lv[l + 1].r, lv[l + 1].z, (l + 1 < C) || a.cinv == nullptr);
            sm_sync(a, sa.cl_fail, target, cid, &s_ok);
        }
        // ---- levels lc .. coarsest: every cluster on its own copy ----
        for (int l = Lc; l < C; l++) {
            sm_restrict(P.R[l], lv[l].rr_lanes, lv[l].n, lv[l].r, lv[l].z, lv[l + 1].r, lv[l + 1].z, (l + 1 < C) || a.cinv == nullptr);
            cluster_sync_all();
        }
        {
            const MgSmLevel& Cl = lv[C];
            const int nC = Cl.n;
            const int wpb = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
            if (a.cinv) {  // dense inverse of the coarsest level (r_C staged once), one warp per row
                for (int j = threadIdx.x; j < nC; j += blockDim.x) rc[j] = __ldcg(&Cl.r[j]);
                __syncthreads();
                for (int i = P.clo + warp; i < P.chi; i += wpb) {
                    const double* row = P.cinv + (size_t)(i - P.clo) * nC;
                    double v = 0;
                    for (int j = lane; j < nC; j += 32) v += row[j] * rc[j];
                    v = warp_sum(v);
                    if (lane == 0) Cl.zf[i] = v;
                }
            } else {  // l1-Jacobi only: the correction is the smoothed z
                for (int i = P.clo + threadIdx.x; i < P.chi; i += blockDim.x) Cl.zf[i] = __ldcg(&Cl.z[i]);
            }
            if (sa.grid_coarse)
                sm_sync(a, sa.cl_fail, target, cid, &s_ok);
            else
                cluster_sync_all();
        }
        for (int l = C - 1; l >= Lc; l--) {
            sm_prolong(P.Q[l], lv[l].pq_lanes, lv[l].n, lv[l].r, lv[l].z, lv[l + 1].zf, lv[l].zf);
            cluster_sync_all();
        }
        // ---- prolongations lc - 1 .. 1 grid-wide ----
        for (int l = Lc - 1; l >= 1; l--) {
            sm_prolong(P.Q[l], lv[l].pq_lanes, lv[l].n, lv[l].r, lv[l].z, lv[l + 1].zf, lv[l].zf);
            sm_sync(a, sa.cl_fail, target, cid, &s_ok);
        }
        // ---- level-0 post-smoother: z = z0 + P z1, z += w M0^-1 (r - A z); r.z ----
        {
            const double* zc = lv[1].zf;
            for (int li = threadIdx.x; li < hi - lo; li += blockDim.x) {
                const double zci = __ldcg(&zc[L.agg[li]]);
                L.w[li] = L.r[li] - own_dot<4>(L.ci, L.val, L.cagg, row_b(li), row_b(li + 1), lo, hi, L.z0, a.z0, zc);
                L.z[li] = L.z0[li] + zci;
            }
            __syncthreads();
            double rz_l = 0;
            for (int li = threadIdx.x; li < hi - lo; li += blockDim.x) {
                const double zi = L.z[li] + a.omega0 * block_row(li, L.w);
                L.z[li] = zi;
                a.z[lo + li] = zi;
                rz_l += L.r[li] * zi;
            }
            mg_reduce1(rz_l, sm, s0);
            if (threadIdx.x == 0) a.partB[cta] = s0;
            sm_sync(a, sa.cl_fail, target, cid, &s_ok);
            const double rz_new = sm_sum_partials(a.partB, nb, sm);
            beta = fresh ? 0.0 : rz_new / rz;
            rz = rz_new;
        }
        // ---- q = A z + beta q, p = z + beta p; p.q ----
        double pq_l = 0;
        for (int li = threadIdx.x; li < hi - lo; li += blockDim.x) {
            const double w = own_dot<4>(L.ci, L.val, nullptr, row_b(li), row_b(li + 1), lo, hi, L.z, a.z, nullptr);
            const double zi = L.z[li];
            const double qi = fresh ? w : w + beta * L.q[li];
            const double pi = fresh ? zi : zi + beta * L.p[li];
            L.q[li] = qi;
            L.p[li] = pi;
            pq_l += pi * qi;
        }
        mg_reduce1(pq_l, sm, s0);
        if (threadIdx.x == 0) a.partA[nb + cta] = s0;
        sm_sync(a, sa.cl_fail, target, cid, &s_ok);
        const double pq = sm_sum_partials(a.partA + nb, nb, sm);
        fresh = false;
        k++;
        // ---- x += alpha p, r -= alpha q (x also to global: other CTAs read it for a true residual) ----
        const double alpha = rz / pq;
        for (int li = threadIdx.x; li < hi - lo; li += blockDim.x) {
            const double xi = L.x[li] + alpha * L.p[li];
            L.x[li] = xi;
            a.x[lo + li] = xi;
            L.r[li] -= alpha * L.q[li];
        }
        recursive = true;
    }
    if (cta == 0 && threadIdx.x == 0) {
        a.stats[0] = (double)k;
        a.stats[1] = rr;
        a.stats[2] = R0;
        a.stats[3] = (double)restarts;
    }
}

// Exclusive scan of n ints in one CTA (the setup's arrays are short enough):
// each thread scans a contiguous chunk; out may alias in; *total gets the sum.
__global__ void __launch_bounds__(1024) k_scan_single(const int32_t* in, int32_t* out, int n, int32_t* total) {
    __shared__ int32_t part[1024];
    const int t = threadIdx.x, T = blockDim.x;
    const int ch = (n + T - 1) / T;
    const int lo = min(n, t * ch), hi = min(n, lo + ch);
    int32_t s = 0;
    for (int i = lo; i < hi; i++) s += in[i];
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < T; o <<= 1) {  // Hillis-Steele inclusive scan of the chunk sums
        const int32_t v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int32_t run = part[t] - s;
    for (int i = lo; i < hi; i++) {
        const int32_t v = in[i];
        out[i] = run;
        run += v;
    }
    if (t == T - 1 && total) *total = part[T - 1];
}

void scan_small(const int32_t* in, int32_t* out, int n, int32_t* total, MgWork& g, cudaStream_t s, int64_t& launches) {
    if (n <= (1 << 20)) {
        k_scan_single<<<1, 1024, 0, s>>>(in, out, n, total);
        launches++;
    } else {
        exclusive_scan_i32(in, out, n, total, g.scan_tmp, s, launches);
    }
}

// Members of level-0 aggregates (chain blocks: consecutive rows).
__global__ void k_members_contig(int n, int nc, const int32_t* __restrict__ agg, int32_t* __restrict__ mptr, int32_t* __restrict__ midx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i == 0 || agg[i] != agg[i - 1]) mptr[agg[i]] = i;
        midx[i] = i;
        if (i == n - 1) mptr[nc] = n;
    }
}

__global__ void k_member_count(int n, const int32_t* __restrict__ agg, int32_t* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) atomicAdd(&cnt[agg[i]], 1);
}

__global__ void k_member_place(int n, const int32_t* __restrict__ agg, const int32_t* __restrict__ mptr, int32_t* __restrict__ cursor,
                               int32_t* __restrict__ midx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int J = agg[i];
        midx[mptr[J] + atomicAdd(&cursor[J], 1)] = i;
    }
}

// Members of every aggregate in ascending row order (insertion sort; aggregates are small).
__global__ void k_member_sort(int nc, const int32_t* __restrict__ mptr, int32_t* __restrict__ midx) {
    for (int J = blockIdx.x * blockDim.x + threadIdx.x; J < nc; J += gridDim.x * blockDim.x) {
        const int b = mptr[J], e = mptr[J + 1];
        for (int i = b + 1; i < e; i++) {
            const int v = midx[i];
            int j = i - 1;
            while (j >= b && midx[j] > v) {
                midx[j + 1] = midx[j];
                j--;
            }
            midx[j + 1] = v;
        }
    }
}

// Per aggregate: couplings gathered from its members' rows (seg_len) and the
// length of its restriction row P^T A_l (members' rows with their diagonals).
__global__ void k_agg_lengths(int nc, const int32_t* __restrict__ mptr, const int32_t* __restrict__ midx, const int32_t* __restrict__ rp,
                              int32_t* __restrict__ seg_len, int32_t* __restrict__ ra_len) {
    for (int J = blockIdx.x * blockDim.x + threadIdx.x; J < nc; J += gridDim.x * blockDim.x) {
        int s = 0;
        for (int m = mptr[J]; m < mptr[J + 1]; m++) {
            const int I = midx[m];
            s += rp[I + 1] - rp[I];
        }
        seg_len[J] = s;
        if (ra_len) ra_len[J] = s + (mptr[J + 1] - mptr[J]);
    }
}

// Coarse row J: the cross-aggregate couplings of its members (in member then entry
// order), gathered as keys (coarse column, gather position) with their values, are sorted
// (keys are unique, so the order equals a stable sort by column) and summed per column in
// gather order (deterministic); the row's diagonal comes from the summed row sums (no
// cancellation of the large intra-aggregate entries), and its l1-Jacobi weight from
// |d| + sum |a|.  `reduce_row` does the summing and writes the compacted row at seg_off[J].
__device__ __forceinline__ void reduce_row(int J, int cnt, double rs, const uint64_t* key, const double* val, uint64_t* __restrict__ okey,
                                           double* __restrict__ oval, int32_t* __restrict__ ulen, double* __restrict__ rs_c,
                                           double* __restrict__ diag, double* __restrict__ l1inv) {
    int u = 0;
    double off = 0, offabs = 0;
    for (int i = 0; i < cnt;) {  // sum runs of equal columns, in gather order
        const uint32_t c = (uint32_t)(key[i] >> 32);
        double acc = 0;
        while (i < cnt && (uint32_t)(key[i] >> 32) == c) acc += val[i++];
        okey[u] = c;
        oval[u] = acc;
        u++;
        off += acc;
        offabs += fabs(acc);
    }
    ulen[J] = u;
    const double d = rs - off;
    rs_c[J] = rs;
    diag[J] = d;
    const double l1 = fabs(d) + offabs;
    l1inv[J] = l1 > 0 ? 1.0 / l1 : 0.0;
}

// One warp per coarse row: the lanes gather a member row's couplings 32 at a time (ballot
// ranks keep the gather order), a bitonic sort orders them in shared memory, lane 0 sums the
// runs.  Rows with more than kCrCap couplings are listed for k_coarse_rows_long.
constexpr int kCrWarps = 4;
constexpr int kCrCap = 512;  // power of two
__global__ void __launch_bounds__(kCrWarps * 32) k_coarse_rows(int nc, const int32_t* __restrict__ mptr, const int32_t* __restrict__ midx,
                                                               const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                               const double* __restrict__ v, const int32_t* __restrict__ agg,
                                                               const double* __restrict__ rs_f, const int32_t* __restrict__ seg_off,
                                                               uint64_t* __restrict__ skey, double* __restrict__ sval, int32_t* __restrict__ ulen,
                                                               double* __restrict__ rs_c, double* __restrict__ diag, double* __restrict__ l1inv,
                                                               int32_t* __restrict__ long_rows, int32_t* __restrict__ n_long) {
    __shared__ uint64_t sk[kCrWarps][kCrCap];
    __shared__ double sv[kCrWarps][kCrCap];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint64_t* K = sk[warp];
    double* V = sv[warp];
    for (int J = blockIdx.x * kCrWarps + warp; J < nc; J += gridDim.x * kCrWarps) {
        int cnt = 0;
        double rs = 0;
        for (int m = mptr[J]; m < mptr[J + 1]; m++) {
            const int I = midx[m];
            if (lane == 0) rs += rs_f[I];
            const int b = rp[I], e = rp[I + 1];
            for (int k0 = b; k0 < e; k0 += 32) {
                const int k = k0 + lane;
                int c = -1;
                double x = 0;
                if (k < e) {
                    c = agg[ci[k]];
                    x = v[k];
                }
                const bool keep = k < e && c != J;
                const unsigned bal = __ballot_sync(0xffffffffu, keep);
                const int pos = cnt + __popc(bal & ((1u << lane) - 1));
                if (keep && pos < kCrCap) {
                    K[pos] = ((uint64_t)(uint32_t)c << 32) | (uint32_t)pos;
                    V[pos] = x;
                }
                cnt += __popc(bal);
            }
        }
        if (cnt > kCrCap) {
            if (lane == 0) long_rows[atomicAdd(n_long, 1)] = J;
            __syncwarp();
            continue;
        }
        int P = 1;
        while (P < cnt) P <<= 1;
        for (int i = cnt + lane; i < P; i += 32) K[i] = ~0ull;
        __syncwarp();
        for (int size = 2; size <= P; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int i = lane; i < P; i += 32) {
                    const int j = i ^ stride;
                    if (j > i) {
                        const bool up = (i & size) == 0;
                        const uint64_t ki = K[i], kj = K[j];
                        if ((ki > kj) == up) {
                            K[i] = kj;
                            K[j] = ki;
                            const double t = V[i];
                            V[i] = V[j];
                            V[j] = t;
                        }
                    }
                }
                __syncwarp();
            }
        if (lane == 0) {
            const int o = seg_off[J];
            reduce_row(J, cnt, rs, K, V, skey + o, sval + o, ulen, rs_c, diag, l1inv);
        }
        __syncwarp();
    }
}

// The rows k_coarse_rows listed as too long for shared memory: one thread each, gathered and
// Shell-sorted in the global scratch at seg_off[J].
__global__ void k_coarse_rows_long(const int32_t* __restrict__ long_rows, const int32_t* __restrict__ n_long, const int32_t* __restrict__ mptr,
                                   const int32_t* __restrict__ midx, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                   const double* __restrict__ v, const int32_t* __restrict__ agg, const double* __restrict__ rs_f,
                                   const int32_t* __restrict__ seg_off, uint64_t* __restrict__ skey, double* __restrict__ sval,
                                   int32_t* __restrict__ ulen, double* __restrict__ rs_c, double* __restrict__ diag, double* __restrict__ l1inv) {
    const int nl = *n_long;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nl; t += gridDim.x * blockDim.x) {
        const int J = long_rows[t];
        const int o = seg_off[J];
        int cnt = 0;
        double rs = 0;
        for (int m = mptr[J]; m < mptr[J + 1]; m++) {
            const int I = midx[m];
            rs += rs_f[I];
            for (int k = rp[I]; k < rp[I + 1]; k++) {
                const int c = agg[ci[k]];
                if (c == J) continue;
                skey[o + cnt] = ((uint64_t)(uint32_t)c << 32) | (uint32_t)cnt;
                sval[o + cnt] = v[k];
                cnt++;
            }
        }
        int gap = 1;
        while (gap * 9 / 4 + 1 < cnt) gap = gap * 9 / 4 + 1;
        for (;; gap = max(1, (gap - 1) * 4 / 9)) {  // ..., 2, 1: the last pass is insertion sort
            for (int i = gap; i < cnt; i++) {
                const uint64_t key = skey[o + i];
                const double x = sval[o + i];
                int j = i;
                while (j >= gap && skey[o + j - gap] > key) {
                    skey[o + j] = skey[o + j - gap];
                    sval[o + j] = sval[o + j - gap];
                    j -= gap;
                }
                skey[o + j] = key;
                sval[o + j] = x;
            }
            if (gap == 1) break;
        }
        reduce_row(J, cnt, rs, skey + o, sval + o, skey + o, sval + o, ulen, rs_c, diag, l1inv);
    }
}

__global__ void k_coarse_copy(int nc, const int32_t* __restrict__ seg_off, const int32_t* __restrict__ ulen, const int32_t* __restrict__ rp_c,
                              const uint64_t* __restrict__ scol, const double* __restrict__ sval, int32_t* __restrict__ ci_c,
                              double* __restrict__ v_c) {
    for (int J = blockIdx.x * blockDim.x + threadIdx.x; J < nc; J += gridDim.x * blockDim.x) {
        const int o = seg_off[J], d = rp_c[J];
        for (int i = 0; i < ulen[J]; i++) {
            ci_c[d + i] = (int32_t)scol[o + i];
            v_c[d + i] = sval[o + i];
        }
    }
}

__global__ void k_cagg_rows(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const int32_t* __restrict__ agg,
                            int32_t* __restrict__ cagg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; k++) cagg[k] = agg[ci[k]];
}

// ---------------------------------------------------------------------------
// Smoothed level-1 prolongator (hierarchies of the clustered kernel).
//
// Why: with piecewise-constant aggregates below the chain level the V-cycle is weak on
// the chain graph, whose junction conductances span five orders of magnitude.  Smoothing
// the first pairwise prolongator once, Q = (I - w D^-1 A_1) P with D the l1-Jacobi
// diagonal and w = 4/3, takes a real-resistor pass of the 25k-CNT network from ~90 to
// ~35 PCG iterations and its unit pass from 54 to 39.  Then A_2 = Q^T A_1 Q, the
// restriction rows are Q^T on r_1 and -Q^T A_1 on z_1, and the prolongation-smoother rows
// are A_1 on z_1 and A_1 (Q + w P) on zc, so that the solve kernel's unchanged
//   zf = z + zc[agg] + D^-1 (r - A_1 z - A_1 (Q + w P) zc)
// equals z + Q zc + D^-1 (r - A_1 (z + Q zc)), since Q zc = zc[agg] - w D^-1 T zc with
// T = A_1 P.  Every product is a row gather: output row J sums w * (row s of B) over its
// sources (s, w); the terms are sorted by column (keys (column, gather position) are
// unique) and summed in gather order, so no result depends on thread timing.
constexpr double kSaOmega = 4.0 / 3.0;
constexpr int kGrWarps = 4;
constexpr int kGrCap = 512;  // power of two

struct RowSrc {  // sources of output row J: (J, 1) when ptr is null, else (J, diag[J]) (with diag) and row J of the CSR
    const int32_t* ptr;
    const int32_t* idx;
    const double* val;
    const double* diag;
};
struct RowMat {  // row s of B: (s, diag[s]) (with diag), then its CSR entries; val2 / diag2: a second value set
    const int32_t* ptr;
    const int32_t* col;
    const double* val;
    const double* diag;
    const double* val2;
    const double* diag2;
    const int32_t* cmap;  // column map (null: identity)
};
struct GatherOut {
    const int32_t* seg;                 // per output row: offset of its segment (candidate terms)
    uint64_t* gkey;                     // long rows: gathered terms (segment layout)
    double* gv;
    double* gv2;
    uint64_t* okey;                     // summed runs (segment layout)
    double* ov;
    double* ov2;
    int32_t* ulen;                      // runs per row
    int32_t* longr;                     // rows with more than kGrCap terms
    int32_t* nlong;
    int skip_diag;                      // drop column J of row J
    const double* rsv;                  // with rs_out: row sum of row J = sum_t w_t rsv[s_t]
    double* rs_out;
    double* diag_out;
    double* l1_out;
};

__device__ __forceinline__ int src_count(const RowSrc& S, int J) { return S.ptr ? (S.ptr[J + 1] - S.ptr[J]) + (S.diag ? 1 : 0) : 1; }

__device__ __forceinline__ void src_get(const RowSrc& S, int J, int t, int& s, double& w) {
    if (!S.ptr) {
        s = J;
        w = 1.0;
        return;
    }
    if (S.diag) {
        if (t == 0) {
            s = J;
            w = S.diag[J];
            return;
        }
        t--;
    }
    const int k = S.ptr[J] + t;
    s = S.idx[k];
    w = S.val[k];
}

__device__ __forceinline__ int mat_len(const RowMat& B, int s) { return (B.ptr[s + 1] - B.ptr[s]) + (B.diag ? 1 : 0); }

__device__ __forceinline__ void mat_get(const RowMat& B, int s, int t, int& c, double& v, double& v2) {
    if (B.diag && t == 0) {
        c = s;
        v = B.diag[s];
        v2 = B.diag2 ? B.diag2[s] : 0.0;
    } else {
        const int k = B.ptr[s] + t - (B.diag ? 1 : 0);
        c = B.col[k];
        v = B.val[k];
        v2 = B.val2 ? B.val2[k] : 0.0;
    }
    if (B.cmap) c = B.cmap[c];
}

__global__ void k_gather_len(int nrows, RowSrc S, RowMat B, int32_t* __restrict__ seg) {
    for (int J = blockIdx.x * blockDim.x + threadIdx.x; J < nrows; J += gridDim.x * blockDim.x) {
        int c = 0;
        const int ns = src_count(S, J);
        for (int t = 0; t < ns; t++) {
            int s;
            double w;
            src_get(S, J, t, s, w);
            c += mat_len(B, s);
        }
        seg[J] = c;
        if (J == 0) seg[nrows] = 0;
    }
}

// Sorted keys of one row (gather positions in their low half) summed into runs of equal
// columns in gather order; with rs_out, the row's diagonal from its row sum (skip_diag rows)
// and its l1-Jacobi weight, as reduce_row does.
__device__ __forceinline__ void gather_reduce(int J, int cnt, const uint64_t* key, const double* val, const double* val2, double rs,
                                              const GatherOut& O, int o) {
    int u = 0;
    double off = 0, offabs = 0;
    for (int i = 0; i < cnt;) {
        const uint32_t c = (uint32_t)(key[i] >> 32);
        double acc = 0, acc2 = 0;
        while (i < cnt && (uint32_t)(key[i] >> 32) == c) {
            const uint32_t p = (uint32_t)key[i];
            acc += val[p];
            if (val2) acc2 += val2[p];
            i++;
        }
        O.okey[o + u] = c;
        O.ov[o + u] = acc;
        if (val2) O.ov2[o + u] = acc2;
        u++;
        off += acc;
        offabs += fabs(acc);
    }
    O.ulen[J] = u;
    if (O.rs_out) {
        const double d = rs - off;
        O.rs_out[J] = rs;
        O.diag_out[J] = d;
        const double l1 = fabs(d) + offabs;
        O.l1_out[J] = l1 > 0 ? 1.0 / l1 : 0.0;
    }
}

// One warp per output row: ballot-ranked gather into shared memory, bitonic sort of the
// keys, lane 0 sums the runs.  Rows with more than kGrCap terms go to k_gather_rows_long.
__global__ void __launch_bounds__(kGrWarps * 32) k_gather_rows(int nrows, RowSrc S, RowMat B, GatherOut O) {
    extern __shared__ __align__(16) unsigned char gr_sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool two = B.val2 != nullptr;
    uint64_t* K = reinterpret_cast<uint64_t*>(gr_sm) + warp * kGrCap;
    double* V = reinterpret_cast<double*>(gr_sm) + (kGrWarps + warp) * kGrCap;
    double* V2 = two ? reinterpret_cast<double*>(gr_sm) + (2 * kGrWarps + warp) * kGrCap : nullptr;
    for (int J = blockIdx.x * kGrWarps + warp; J < nrows; J += gridDim.x * kGrWarps) {
        int cnt = 0;
        double rs = 0;
        const int ns = src_count(S, J);
        for (int t = 0; t < ns; t++) {
            int s;
            double w;
            src_get(S, J, t, s, w);
            if (O.rsv && lane == 0) rs += w * O.rsv[s];
            const int L = mat_len(B, s);
            for (int k0 = 0; k0 < L; k0 += 32) {
                const int k = k0 + lane;
                int c = 0;
                double x = 0, x2 = 0;
                bool keep = false;
                if (k < L) {
                    mat_get(B, s, k, c, x, x2);
                    keep = !(O.skip_diag && c == J);
                }
                const unsigned bal = __ballot_sync(0xffffffffu, keep);
                const int pos = cnt + __popc(bal & ((1u << lane) - 1u));
                if (keep && pos < kGrCap) {
                    K[pos] = ((uint64_t)(uint32_t)c << 32) | (uint32_t)pos;
                    V[pos] = w * x;
                    if (two) V2[pos] = w * x2;
                }
                cnt += __popc(bal);
            }
        }
        if (cnt > kGrCap) {
            if (lane == 0) O.longr[atomicAdd(O.nlong, 1)] = J;
            __syncwarp();
            continue;
        }
        int P = 1;
        while (P < cnt) P <<= 1;
        for (int i = cnt + lane; i < P; i += 32) K[i] = ~0ull;
        __syncwarp();
        for (int size = 2; size <= P; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int i = lane; i < P; i += 32) {
                    const int j = i ^ stride;
                    if (j > i) {
                        const bool up = (i & size) == 0;
                        const uint64_t ki = K[i], kj = K[j];
                        if ((ki > kj) == up) {
                            K[i] = kj;
                            K[j] = ki;
                        }
                    }
                }
                __syncwarp();
            }
        if (lane == 0) gather_reduce(J, cnt, K, V, V2, rs, O, O.seg[J]);
        __syncwarp();
    }
}

// The rows k_gather_rows listed as too long: one thread each, gathered and Shell-sorted in
// the global scratch at the row's segment (same keys, so the same sums as the warp path).
__global__ void k_gather_rows_long(RowSrc S, RowMat B, GatherOut O) {
    const int nl = *O.nlong;
    const bool two = B.val2 != nullptr;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nl; q += gridDim.x * blockDim.x) {
        const int J = O.longr[q];
        const int o = O.seg[J];
        uint64_t* K = O.gkey + o;
        double* V = O.gv + o;
        double* V2 = two ? O.gv2 + o : nullptr;
        int cnt = 0;
        double rs = 0;
        const int ns = src_count(S, J);
        for (int t = 0; t < ns; t++) {
            int s;
            double w;
            src_get(S, J, t, s, w);
            if (O.rsv) rs += w * O.rsv[s];
            const int L = mat_len(B, s);
            for (int k = 0; k < L; k++) {
                int c;
                double x, x2;
                mat_get(B, s, k, c, x, x2);
                if (O.skip_diag && c == J) continue;
                K[cnt] = ((uint64_t)(uint32_t)c << 32) | (uint32_t)cnt;
                V[cnt] = w * x;
                if (two) V2[cnt] = w * x2;
                cnt++;
            }
        }
        int gap = 1;
        while (gap * 9 / 4 + 1 < cnt) gap = gap * 9 / 4 + 1;
        for (;; gap = max(1, (gap - 1) * 4 / 9)) {  // ..., 2, 1: the last pass is insertion sort
            for (int i = gap; i < cnt; i++) {
                const uint64_t key = K[i];
                int j = i;
                while (j >= gap && K[j - gap] > key) {
                    K[j] = K[j - gap];
                    j -= gap;
                }
                K[j] = key;
            }
            if (gap == 1) break;
        }
        gather_reduce(J, cnt, K, V, V2, rs, O, o);
    }
}

__global__ void k_gather_copy(int nrows, const int32_t* __restrict__ seg, const int32_t* __restrict__ ulen, const int32_t* __restrict__ rp,
                              const uint64_t* __restrict__ okey, const double* __restrict__ ov, const double* __restrict__ ov2,
                              int32_t* __restrict__ col, double* __restrict__ val, double* __restrict__ val2) {
    for (int J = blockIdx.x * blockDim.x + threadIdx.x; J < nrows; J += gridDim.x * blockDim.x) {
        const int o = seg[J], d = rp[J];
        for (int i = 0; i < ulen[J]; i++) {
            col[d + i] = (int32_t)okey[o + i];
            val[d + i] = ov[o + i];
            if (val2) val2[d + i] = ov2[o + i];
        }
    }
}

// Q = P - w D^-1 T and Q + w P on T's pattern (T_i always holds column agg[i]).
__global__ void k_sa_q(int n, const int32_t* __restrict__ tp, const int32_t* __restrict__ tc, const double* __restrict__ tv,
                       const int32_t* __restrict__ agg, const double* __restrict__ l1inv, double* __restrict__ qv, double* __restrict__ qpv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int a = agg[i];
        const double m = l1inv[i];
        for (int k = tp[i]; k < tp[i + 1]; k++) {
            const double base = tc[k] == a ? 1.0 : 0.0;
            const double q = base - kSaOmega * m * tv[k];
            qv[k] = q;
            qpv[k] = q + kSaOmega * base;
        }
    }
}

// Transpose of a CSR with unique columns per row: count, place, then each column's rows in order.
__global__ void k_col_count(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col, int32_t* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; k++) atomicAdd(&cnt[col[k]], 1);
}

__global__ void k_col_place(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col, const double* __restrict__ val,
                            const int32_t* __restrict__ cptr, int32_t* __restrict__ cursor, int32_t* __restrict__ ridx, double* __restrict__ rval) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            const int c = col[k];
            const int p = cptr[c] + atomicAdd(&cursor[c], 1);
            ridx[p] = i;
            rval[p] = val[k];
        }
}

__global__ void k_seg_sort(int nc, const int32_t* __restrict__ ptr, int32_t* __restrict__ idx, double* __restrict__ val) {
    for (int J = blockIdx.x * blockDim.x + threadIdx.x; J < nc; J += gridDim.x * blockDim.x) {
        const int b = ptr[J], e = ptr[J + 1];
        for (int i = b + 1; i < e; i++) {
            const int x = idx[i];
            const double y = val[i];
            int j = i - 1;
            while (j >= b && idx[j] > x) {
                idx[j + 1] = idx[j];
                val[j + 1] = val[j];
                j--;
            }
            idx[j + 1] = x;
            val[j + 1] = y;
        }
    }
}

// v = A_1 Q 1 for the coarse row sums: Q 1 = 1 - w D^-1 rs, so v = rs - w A_1 (D^-1 rs); rs
// is nonzero only next to prescribed nodes, so the chain conductances never cancel here.
__global__ void k_sa_y(int n, const double* __restrict__ l1inv, const double* __restrict__ rs, double* __restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = l1inv[i] * rs[i];
}

__global__ void k_sa_v(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ val,
                       const double* __restrict__ diag, const double* __restrict__ rs, const double* __restrict__ y, double* __restrict__ v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = diag[i] * y[i];
        for (int k = rp[i]; k < rp[i + 1]; k++) s += val[k] * y[ci[k]];
        v[i] = rs[i] - kSaOmega * s;
    }
}

// Fused restriction rows of the smoothed level: row J = Q^T row J on r_1 (columns < n), then
// -(Q^T A_1) row J on z_1 (columns n + c).
__global__ void k_rr_fill_sa(int nc, int n, const int32_t* __restrict__ qtp, const int32_t* __restrict__ qti, const double* __restrict__ qtv,
                             const int32_t* __restrict__ ap, const int32_t* __restrict__ ac, const double* __restrict__ av,
                             int32_t* __restrict__ rr_ptr, int32_t* __restrict__ rr_col, double* __restrict__ rr_val) {
    for (int J = blockIdx.x * blockDim.x + threadIdx.x; J < nc; J += gridDim.x * blockDim.x) {
        int e = qtp[J] + ap[J];
        rr_ptr[J] = e;
        if (J == nc - 1) rr_ptr[nc] = qtp[nc] + ap[nc];
        for (int k = qtp[J]; k < qtp[J + 1]; k++, e++) {
            rr_col[e] = qti[k];
            rr_val[e] = qtv[k];
        }
        for (int k = ap[J]; k < ap[J + 1]; k++, e++) {
            rr_col[e] = n + ac[k];
            rr_val[e] = -av[k];
        }
    }
}

// Fused prolongation-smoother rows of the smoothed level: row I = A_1 row I with its diagonal
// on z_1, then A_1 (Q + w P) row I on zc (columns n + J).
__global__ void k_pq_fill_sa(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                             const double* __restrict__ diag, const int32_t* __restrict__ wp, const int32_t* __restrict__ wc,
                             const double* __restrict__ wv, int32_t* __restrict__ pq_ptr, int32_t* __restrict__ pq_col,
                             double* __restrict__ pq_val) {
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < n; I += gridDim.x * blockDim.x) {
        int e = rp[I] + I + wp[I];
        pq_ptr[I] = e;
        if (I == n - 1) pq_ptr[n] = rp[n] + n + wp[n];
        pq_col[e] = I;
        pq_val[e] = diag[I];
        e++;
        for (int k = rp[I]; k < rp[I + 1]; k++, e++) {
            pq_col[e] = ci[k];
            pq_val[e] = v[k];
        }
        for (int k = wp[I]; k < wp[I + 1]; k++, e++) {
            pq_col[e] = n + wc[k];
            pq_val[e] = wv[k];
        }
    }
}

// One row-gather product: the compacted CSR (optr, ocol, oval[, oval2]) of nrows rows, its
// arrays sized by the candidate-term count (one host read), which is returned (>= entries).
long long gather_product(MgWork& g, int nrows, const RowSrc& S, const RowMat& B, bool skip_diag, const double* rsv, double* rs_out,
                         double* diag_out, double* l1_out, DBuf<int32_t>& optr, DBuf<int32_t>& ocol, DBuf<double>& oval,
                         DBuf<double>* oval2, cudaStream_t s, int64_t& launches) {
    MgWork::Smoothed& w = g.sa;
    w.seg.ensure(nrows + 1);
    k_gather_len<<<grid_for(nrows), 256, 0, s>>>(nrows, S, B, w.seg.get());
    launches++;
    scan_small(w.seg.get(), w.seg.get(), nrows + 1, g.total.get(), g, s, launches);
    int cand = 0;
    CICY_CUDA(cudaMemcpyAsync(&cand, g.total.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    const size_t cap = (size_t)std::max(cand, 1);
    const bool two = B.val2 != nullptr;
    w.gkey.ensure(cap);
    w.gv.ensure(cap);
    w.okey.ensure(cap);
    w.ov.ensure(cap);
    if (two) {
        w.gv2.ensure(cap);
        w.ov2.ensure(cap);
    }
    w.ulen.ensure(nrows + 1);
    w.longr.ensure(nrows + 1);
    CICY_CUDA(cudaMemsetAsync(g.total.get() + 1, 0, sizeof(int32_t), s));
    CICY_CUDA(cudaMemsetAsync(w.ulen.get() + nrows, 0, sizeof(int32_t), s));
    const GatherOut O{w.seg.get(),  w.gkey.get(), w.gv.get(),  two ? w.gv2.get() : nullptr, w.okey.get(), w.ov.get(),
                      two ? w.ov2.get() : nullptr, w.ulen.get(), w.longr.get(), g.total.get() + 1, skip_diag ? 1 : 0,
                      rsv, rs_out, diag_out, l1_out};
    const int smem = (int)(sizeof(double) * kGrWarps * kGrCap * (two ? 3 : 2));
    static bool attr = false;
    if (!attr) {
        CICY_CUDA(cudaFuncSetAttribute(k_gather_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(double) * kGrWarps * kGrCap * 3)));
        attr = true;
    }
    k_gather_rows<<<grid_for((long long)nrows * 32, kGrWarps * 32), kGrWarps * 32, smem, s>>>(nrows, S, B, O);
    k_gather_rows_long<<<grid_for(nrows, 128), 128, 0, s>>>(S, B, O);
    optr.ensure(nrows + 1);
    scan_small(w.ulen.get(), optr.get(), nrows + 1, nullptr, g, s, launches);
    ocol.ensure(cap);
    oval.ensure(cap);
    if (two) oval2->ensure(cap);
    k_gather_copy<<<grid_for(nrows), 256, 0, s>>>(nrows, w.seg.get(), w.ulen.get(), optr.get(), w.okey.get(), w.ov.get(),
                                                  two ? w.ov2.get() : nullptr, ocol.get(), oval.get(), two ? oval2->get() : nullptr);
    launches += 3;
    CICY_LAUNCH_CHECK();
    return cand;
}

// Level 2 from level 1 through the smoothed prolongator (nc pairwise aggregates in
// g.L[1].agg), with level 1's fused restriction and prolongation-smoother rows.
void coarsen_smoothed(MgWork& g, int nc, cudaStream_t s, int64_t& launches) {
    MgWork::Lvl& F = g.L[1];
    MgWork::Lvl& G = g.L[2];
    MgWork::Smoothed& w = g.sa;
    const int n = F.n;
    const RowSrc one{nullptr, nullptr, nullptr, nullptr};
    const RowSrc a1_src{F.rp_ptr, F.ci_ptr, F.val_ptr, F.diag.get()};
    const RowMat a1{F.rp_ptr, F.ci_ptr, F.val_ptr, F.diag.get(), nullptr, nullptr, nullptr};
    const RowMat a1_agg{F.rp_ptr, F.ci_ptr, F.val_ptr, F.diag.get(), nullptr, nullptr, F.agg.get()};
    // T = A_1 P, then Q and Q + w P on its pattern
    const long long nt = gather_product(g, n, one, a1_agg, false, nullptr, nullptr, nullptr, nullptr, w.tp, w.tc, w.tv, nullptr, s, launches);
    w.qv.ensure(nt);
    w.qpv.ensure(nt);
    k_sa_q<<<grid_for(n), 256, 0, s>>>(n, w.tp.get(), w.tc.get(), w.tv.get(), F.agg.get(), F.l1inv.get(), w.qv.get(), w.qpv.get());
    // Q^T: each aggregate's rows in ascending order
    w.qtp.ensure(nc + 1);
    w.qti.ensure(nt);
    w.qtv.ensure(nt);
    g.flag.ensure(nc + 1);
    CICY_CUDA(cudaMemsetAsync(g.flag.get(), 0, sizeof(int32_t) * (nc + 1), s));
    k_col_count<<<grid_for(n), 256, 0, s>>>(n, w.tp.get(), w.tc.get(), g.flag.get());
    scan_small(g.flag.get(), w.qtp.get(), nc + 1, nullptr, g, s, launches);
    CICY_CUDA(cudaMemsetAsync(g.flag.get(), 0, sizeof(int32_t) * (nc + 1), s));
    k_col_place<<<grid_for(n), 256, 0, s>>>(n, w.tp.get(), w.tc.get(), w.qv.get(), w.qtp.get(), g.flag.get(), w.qti.get(), w.qtv.get());
    k_seg_sort<<<grid_for(nc), 256, 0, s>>>(nc, w.qtp.get(), w.qti.get(), w.qtv.get());
    launches += 4;
    const RowSrc qt_src{w.qtp.get(), w.qti.get(), w.qtv.get(), nullptr};
    // W = A_1 Q and A_1 (Q + w P)
    const RowMat q{w.tp.get(), w.tc.get(), w.qv.get(), nullptr, w.qpv.get(), nullptr, nullptr};
    const long long nw = gather_product(g, n, a1_src, q, false, nullptr, nullptr, nullptr, nullptr, w.wp, w.wc, w.wv, &w.wpv, s, launches);
    // Q^T A_1 (the restriction rows' part on z_1)
    const long long na = gather_product(g, nc, qt_src, a1, false, nullptr, nullptr, nullptr, nullptr, w.ap, w.ac, w.av, nullptr, s, launches);
    // A_2 = Q^T W off the diagonal; its diagonal from the row sums Q^T A_1 Q 1
    w.y.ensure(n);
    w.v.ensure(n);
    k_sa_y<<<grid_for(n), 256, 0, s>>>(n, F.l1inv.get(), F.rs.get(), w.y.get());
    k_sa_v<<<grid_for(n), 256, 0, s>>>(n, F.rp_ptr, F.ci_ptr, F.val_ptr, F.diag.get(), F.rs.get(), w.y.get(), w.v.get());
    launches += 2;
    G.n = nc;
    G.rs.ensure(nc);
    G.diag.ensure(nc);
    G.l1inv.ensure(nc);
    const RowMat wm{w.wp.get(), w.wc.get(), w.wv.get(), nullptr, nullptr, nullptr, nullptr};
    const long long n2 = gather_product(g, nc, qt_src, wm, true, w.v.get(), G.rs.get(), G.diag.get(), G.l1inv.get(), G.rp, G.ci, G.val,
                                        nullptr, s, launches);
    G.nnz = (int)std::max<long long>(n2, 1);
    G.rp_ptr = G.rp.get();
    G.ci_ptr = G.ci.get();
    G.val_ptr = G.val.get();
    // level 1's fused rows
    F.rr_ptr.ensure(nc + 1);
    F.rr_col.ensure(std::max<long long>(nt + na, 1));
    F.rr_val.ensure(std::max<long long>(nt + na, 1));
    k_rr_fill_sa<<<grid_for(nc), 256, 0, s>>>(nc, n, w.qtp.get(), w.qti.get(), w.qtv.get(), w.ap.get(), w.ac.get(), w.av.get(), F.rr_ptr.get(),
                                               F.rr_col.get(), F.rr_val.get());
    F.pq_ptr.ensure(n + 1);
    F.pq_col.ensure(std::max<long long>((long long)F.nnz + n + nw, 1));
    F.pq_val.ensure(std::max<long long>((long long)F.nnz + n + nw, 1));
    k_pq_fill_sa<<<grid_for(n), 256, 0, s>>>(n, F.rp_ptr, F.ci_ptr, F.val_ptr, F.diag.get(), w.wp.get(), w.wc.get(), w.wpv.get(),
                                              F.pq_ptr.get(), F.pq_col.get(), F.pq_val.get());
    launches += 2;
    CICY_LAUNCH_CHECK();
}

// Galerkin coarse level l+1 from level l and its aggregates (g.L[l].agg, nc of
// them), plus level l's member lists, restriction rows (l >= 1) and column
// aggregates.  No host synchronisation: buffers are sized by the fine level's
// non-zeros, an upper bound of the coarse level's.
void coarsen(MgWork& g, int l, int nc, cudaStream_t s, int64_t& launches) {
    if ((int)g.L.size() < l + 2) g.L.resize(l + 2);
    if (g.fused && g.smooth && l == 1) {
        coarsen_smoothed(g, nc, s, launches);
        return;
    }
    MgWork::Lvl& F = g.L[l];
    MgWork::Lvl& G = g.L[l + 1];
    const int nf = F.n, nnz = F.nnz;
    F.mptr.ensure(nc + 1);
    F.midx.ensure(std::max(nf, 1));
    if (l == 0) {
        k_members_contig<<<grid_for(nf), 256, 0, s>>>(nf, nc, F.agg.get(), F.mptr.get(), F.midx.get());
        launches++;
    } else {
        g.flag.ensure(nc + 1);
        CICY_CUDA(cudaMemsetAsync(g.flag.get(), 0, sizeof(int32_t) * (nc + 1), s));
        k_member_count<<<grid_for(nf), 256, 0, s>>>(nf, F.agg.get(), g.flag.get());
        scan_small(g.flag.get(), F.mptr.get(), nc + 1, nullptr, g, s, launches);
        CICY_CUDA(cudaMemsetAsync(g.flag.get(), 0, sizeof(int32_t) * (nc + 1), s));
        k_member_place<<<grid_for(nf), 256, 0, s>>>(nf, F.agg.get(), F.mptr.get(), g.flag.get(), F.midx.get());
        k_member_sort<<<grid_for(nc), 256, 0, s>>>(nc, F.mptr.get(), F.midx.get());
        launches += 3;
    }
    // lengths and offsets
    g.pos.ensure(nc + 1);
    g.head.ensure(nc + 1);
    g.uidx.ensure(nc + 1);
    if (l >= 1) F.ra_ptr.ensure(nc + 1);
    k_agg_lengths<<<grid_for(nc), 256, 0, s>>>(nc, F.mptr.get(), F.midx.get(), F.rp_ptr, g.pos.get(), l >= 1 ? F.ra_ptr.get() : nullptr);
    launches++;
    scan_small(g.pos.get(), g.pos.get(), nc + 1, nullptr, g, s, launches);  // seg_off
    // coarse rows
    g.keys.ensure(std::max(nnz, 1));
    g.sval.ensure(std::max(nnz, 1));
    G.n = nc;
    G.nnz = nnz;  // capacity bound
    G.rp.ensure(nc + 1);
    G.ci.ensure(std::max(nnz, 1));
    G.val.ensure(std::max(nnz, 1));
    G.rs.ensure(nc);
    G.diag.ensure(nc);
    G.l1inv.ensure(nc);
    g.long_rows.ensure(nc + 1);
    CICY_CUDA(cudaMemsetAsync(g.total.get() + 1, 0, sizeof(int32_t), s));
    k_coarse_rows<<<grid_for((long long)nc * 32, kCrWarps * 32), kCrWarps * 32, 0, s>>>(
        nc, F.mptr.get(), F.midx.get(), F.rp_ptr, F.ci_ptr, F.val_ptr, F.agg.get(), F.rs.get(), g.pos.get(), g.keys.get(), g.sval.get(),
        g.head.get(), G.rs.get(), G.diag.get(), G.l1inv.get(), g.long_rows.get(), g.total.get() + 1);
    k_coarse_rows_long<<<grid_for(nc, 128), 128, 0, s>>>(g.long_rows.get(), g.total.get() + 1, F.mptr.get(), F.midx.get(), F.rp_ptr,
                                                       F.ci_ptr, F.val_ptr, F.agg.get(), F.rs.get(), g.pos.get(), g.keys.get(),
                                                       g.sval.get(), g.head.get(), G.rs.get(), G.diag.get(), G.l1inv.get());
    launches++;
    scan_small(g.head.get(), G.rp.get(), nc + 1, nullptr, g, s, launches);
    k_coarse_copy<<<grid_for(nc), 256, 0, s>>>(nc, g.pos.get(), g.head.get(), G.rp.get(), g.keys.get(), g.sval.get(), G.ci.get(),
                                               G.val.get());
    launches += 2;
    G.rp_ptr = G.rp.get();
    G.ci_ptr = G.ci.get();
    G.val_ptr = G.val.get();
    // restriction rows of level l (l >= 1) and its column aggregates; the clustered kernel
    // (g.fused) reads the fused rows instead of P^T A_l and the coarse column aggregates
    if (l >= 1) {
        scan_small(F.ra_ptr.get(), F.ra_ptr.get(), nc + 1, nullptr, g, s, launches);
        if (!g.fused) {
            F.ra_col.ensure(std::max(nnz + nf, 1));
            F.ra_val.ensure(std::max(nnz + nf, 1));
            k_ra_fill<<<grid_for(nc), 256, 0, s>>>(nc, F.mptr.get(), F.midx.get(), F.rp_ptr, F.ci_ptr, F.val_ptr, F.diag.get(),
                                                    F.ra_ptr.get(), F.ra_col.get(), F.ra_val.get());
            launches++;
        }
    }
    if (!g.fused || l == 0) {
        F.cagg.ensure(std::max(nnz, 1));
        k_cagg_rows<<<grid_for(nf), 256, 0, s>>>(nf, F.rp_ptr, F.ci_ptr, F.agg.get(), F.cagg.get());
        launches++;
    }
    if (g.fused && l >= 1) {
        F.rr_ptr.ensure(nc + 1);
        F.rr_col.ensure(std::max(nnz + 2 * nf, 1));
        F.rr_val.ensure(std::max(nnz + 2 * nf, 1));
        k_rr_fill<<<grid_for(nc), 256, 0, s>>>(nc, nf, F.mptr.get(), F.midx.get(), F.rp_ptr, F.ci_ptr, F.val_ptr, F.diag.get(), F.ra_ptr.get(),
                                                F.rr_ptr.get(), F.rr_col.get(), F.rr_val.get());
        F.pq_ptr.ensure(nf + 1);
        F.pq_col.ensure(std::max(2 * (nnz + nf), 1));
        F.pq_val.ensure(std::max(2 * (nnz + nf), 1));
        k_pq_fill<<<grid_for(nf), 256, 0, s>>>(nf, F.rp_ptr, F.ci_ptr, F.val_ptr, F.diag.get(), F.agg.get(), F.pq_ptr.get(),
                                                F.pq_col.get(), F.pq_val.get());
        launches += 2;
    }
    CICY_LAUNCH_CHECK();
}

// Pairwise aggregates of level l; returns their number.
int pairwise(MgWork& g, int l, cudaStream_t s, int64_t& launches) {
    MgWork::Lvl& F = g.L[l];
    const int n = F.n;
    g.mate.ensure(n + 1);
    g.best.ensure(n + 1);
    g.rep.ensure(n + 1);
    g.flag.ensure(n + 1);
    g.pos.ensure(n + 1);
    k_fill_neg<<<grid_for(n), 256, 0, s>>>(n, g.mate.get());
    launches++;
    for (int round = 0; round < 3; round++) {
        k_strongest<<<grid_for(n), 256, 0, s>>>(n, 1, F.rp_ptr, F.ci_ptr, F.val_ptr, g.mate.get(), g.best.get());
        k_handshake<<<grid_for(n), 256, 0, s>>>(n, g.best.get(), g.mate.get());
        launches += 2;
    }
    k_pair_rep<<<grid_for(n), 256, 0, s>>>(n, g.mate.get(), g.rep.get());
    k_strongest<<<grid_for(n), 256, 0, s>>>(n, 0, F.rp_ptr, F.ci_ptr, F.val_ptr, g.mate.get(), g.best.get());
    k_join<<<grid_for(n), 256, 0, s>>>(n, g.mate.get(), g.best.get(), g.rep.get());
    k_is_rep<<<grid_for(n), 256, 0, s>>>(n, g.rep.get(), g.flag.get());
    launches += 4;
    scan_small(g.flag.get(), g.pos.get(), n, g.total.get(), g, s, launches);
    F.agg.ensure(n + 1);
    k_agg_ids<<<grid_for(n), 256, 0, s>>>(n, g.rep.get(), g.pos.get(), F.agg.get());
    launches++;
    int nc = 0;
    CICY_CUDA(cudaMemcpyAsync(&nc, g.total.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    CICY_LAUNCH_CHECK();
    return nc;
}

}  // namespace

// ---------------------------------------------------------------------------
void build_mg_hierarchy(SolverWork& w, const SolverSystem& sys, cudaStream_t s, int64_t& launches, bool fused, bool smooth, int* status) {
    MgWork& g = w.mg;
    const int n = sys.n;
    g.fused = fused;
    g.smooth = smooth;
    TraceSeq tr(s);
    g.total.ensure(2);
    if (g.L.empty()) g.L.resize(1);
    MgWork::Lvl& L0 = g.L[0];
    L0.n = n;
    L0.nnz = sys.nnz;
    L0.rp_ptr = sys.rp;
    L0.ci_ptr = sys.ci;
    L0.val_ptr = sys.val;
    L0.agg.ensure(n + 1);
    L0.rs.ensure(n + 1);
    k_block_of_row<<<grid_for(n), 256, 0, s>>>(n, w.is_start.get(), w.start_scan.get(), L0.agg.get());
    k_rowsum0<<<grid_for(n), 256, 0, s>>>(n, sys.rp, sys.ci, sys.val, L0.rs.get());
    launches += 2;
    int nc = w.n_blocks;
    int C = 0;
    // the clustered kernel solves a dense coarsest of up to kMgDenseGridMax rows on all CTAs
    int dense_cap = kMgDenseMax;
    if (fused) {
        int dev = 0, sms = 0;
        CICY_CUDA(cudaGetDevice(&dev));
        CICY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        dense_cap = std::max(kMgDenseMax, std::min(kMgDenseGridMax, sms * kGjgMaxStrip));
    }
    for (int l = 0;; l++) {
        coarsen(g, l, nc, s, launches);
        tr.mark("mg.coarsen");
        C = l + 1;
        if (g.L[C].n <= dense_cap || C + 1 >= kMgMaxLevels) break;
        const int nc2 = pairwise(g, C, s, launches);
        tr.mark("mg.pairwise");
        if (nc2 > 0.9 * g.L[C].n) break;
        nc = nc2;
    }
    g.dense = false;
    MgWork::Lvl& Lc = g.L[C];
    if (Lc.n <= kMgDenseMax) {
        g.cinv.ensure((size_t)Lc.n * Lc.n);
        CICY_CUDA(cudaMemsetAsync(g.cinv.get(), 0, sizeof(double) * Lc.n * Lc.n, s));
        k_dense_coarse<<<grid_for(Lc.n, 128), 128, 0, s>>>(Lc.n, Lc.rp.get(), Lc.ci.get(), Lc.val.get(), Lc.diag.get(), g.cinv.get());
        const size_t smem = sizeof(double) * ((size_t)Lc.n * Lc.n + 2 * (size_t)Lc.n * kGjBlock + kGjBlock * (kGjBlock + 1) + kGjBlock);
        if (smem > 48 * 1024)
            CICY_CUDA(cudaFuncSetAttribute(k_gauss_jordan, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_gauss_jordan<<<1, kGjThreads, smem, s>>>(Lc.n, g.cinv.get());
        launches += 2;
        g.dense = true;
    } else if (Lc.n <= dense_cap) {
        // larger dense coarsest: the grid Gauss-Jordan (one cooperative launch, column strips)
        int nC = Lc.n, dev = 0, sms = 0;
        CICY_CUDA(cudaGetDevice(&dev));
        CICY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        g.cinv.ensure((size_t)nC * nC);
        g.gj_panel.ensure((size_t)2 * nC * kGjBlock);
        g.gj_sync.ensure(2);
        g.gj_err.ensure(1);
        CICY_CUDA(cudaMemsetAsync(g.gj_sync.get(), 0, sizeof(unsigned long long) * 2, s));
        int* err = status;
        if (!err) {
            CICY_CUDA(cudaMemsetAsync(g.gj_err.get(), 0, sizeof(int32_t), s));
            err = g.gj_err.get();
        }
        CICY_CUDA(cudaMemsetAsync(g.cinv.get(), 0, sizeof(double) * nC * nC, s));
        k_dense_coarse<<<grid_for(nC, 128), 128, 0, s>>>(nC, Lc.rp.get(), Lc.ci.get(), Lc.val.get(), Lc.diag.get(), g.cinv.get());
        const int G = std::max(1, std::min(sms, nC));
        const int wmax = (nC + G - 1) / G;
        if (wmax > kGjgMaxStrip) throw Fail{CICY_E_INTERNAL, "multigrid: dense coarsest too large for this GPU"};
        const size_t smem = sizeof(double) * (size_t)nC * wmax;
        void (*kern)(int, double*, double*, unsigned long long*, unsigned long long*, int*, long long) = nullptr;
        switch (wmax) {
            case 1: kern = k_gauss_jordan_grid<1>; break;
            case 2: kern = k_gauss_jordan_grid<2>; break;
            case 3: kern = k_gauss_jordan_grid<3>; break;
            case 4: kern = k_gauss_jordan_grid<4>; break;
            case 5: kern = k_gauss_jordan_grid<5>; break;
            case 6: kern = k_gauss_jordan_grid<6>; break;
            case 7: kern = k_gauss_jordan_grid<7>; break;
            case 8: kern = k_gauss_jordan_grid<8>; break;
            case 9: kern = k_gauss_jordan_grid<9>; break;
            default: kern = k_gauss_jordan_grid<10>; break;
        }
        CICY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        double* M = g.cinv.get();
        double* panel = g.gj_panel.get();
        unsigned long long* bar = g.gj_sync.get();
        unsigned long long* dmax = g.gj_sync.get() + 1;
        long long limit = w.spin_limit;
        void* args[] = {&nC, &M, &panel, &bar, &dmax, &err, &limit};
        CICY_CUDA(cudaLaunchCooperativeKernel((void*)kern, dim3(G), dim3(kGjgThreads), args, smem, s));
        launches += 2;
        g.dense = true;
    }
    tr.mark("mg.coarsest");
    tr.mark("mg.restriction_rows");
    // work vectors and device descriptors
    g.host_lv.assign(C + 1, MgLevel{});
    for (int l = 0; l <= C; l++) {
        MgWork::Lvl& L = g.L[l];
        MgLevel& d = g.host_lv[l];
        d.n = L.n;
        d.rp = L.rp_ptr;
        d.ci = L.ci_ptr;
        d.val = L.val_ptr;
        d.agg = (l < C) ? L.agg.get() : nullptr;
        d.mptr = (l < C) ? L.mptr.get() : nullptr;
        d.midx = (l < C) ? L.midx.get() : nullptr;
        d.cagg = (l < C) ? L.cagg.get() : nullptr;
        d.ra_ptr = (l >= 1 && l < C) ? L.ra_ptr.get() : nullptr;
        d.ra_col = (l >= 1 && l < C) ? L.ra_col.get() : nullptr;
        d.ra_val = (l >= 1 && l < C) ? L.ra_val.get() : nullptr;
        if (l >= 1) {
            L.r.ensure(L.n + 1);
            L.z.ensure(L.n + 1);
            d.diag = L.diag.get();
            d.l1inv = L.l1inv.get();
            d.r = L.r.get();
            d.z = L.z.get();
            if (l == C && !g.dense) {
                d.zf = L.z.get();
            } else {
                L.zf.ensure(L.n + 1);
                d.zf = L.zf.get();
            }
        }
    }
    g.dev_lv.ensure(C + 1);
    CICY_CUDA(cudaMemcpyAsync(g.dev_lv.get(), g.host_lv.data(), sizeof(MgLevel) * (C + 1), cudaMemcpyHostToDevice, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    g.levels = C + 1;
    CICY_LAUNCH_CHECK();
}

bool mg_fused_path(int n, bool allow_cluster) { return !(allow_cluster && n <= kMgClusterMaxRows); }

void pcg_solve_mg(SolverWork& w, const SolverSystem& sys, double tol, long long max_iter, bool allow_cluster, int num_sms, int* status,
                  cudaStream_t s, int64_t& launches, PcgStats& st) {
    const int n = sys.n;
    st = PcgStats{};
    if (n <= 0) return;
    MgWork& g = w.mg;
    w.r.ensure(n); w.z.ensure(n); w.p.ensure(n); w.q.ensure(n);
    g.z0.ensure(n);
    g.wtmp.ensure(n);
    k_residual<<<grid_for(n), 256, 0, s>>>(n, sys.rp, sys.ci, sys.val, sys.x, sys.b, w.r.get());
    launches++;
    // one 16-CTA cluster with hardware barriers when it can be launched, else the
    // grid-wide cooperative launch
    static int cl_state = 0;  // 0 unknown, 1 ok, -1 unsupported
    if (cl_state == 0) {
        cl_state = cudaFuncSetAttribute(k_mg_pcg<true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess ? 1 : -1;
        cudaGetLastError();
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    bool cluster = false;
    if (allow_cluster && !g.fused && cl_state > 0 && n <= kMgClusterMaxRows) {
        cfg.gridDim = dim3(kMgClusterCtas);
        cfg.blockDim = dim3(kMgClusterThreads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kMgClusterCtas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        cluster = cudaOccupancyMaxActiveClusters(&nclusters, (void*)k_mg_pcg<true>, &cfg) == cudaSuccess && nclusters >= 1;
        cudaGetLastError();
    }
    // above one cluster's size: the shared-memory-resident clustered grid kernel (one CTA per
    // SM, levels from lc on solved per cluster) when the fused rows exist and K clusters of
    // kSmCtas can be co-resident
    bool sec = false;
    const bool gridc = g.fused && g.dense;  // dense coarsest solved by all CTAs (no cluster levels)
    int K = 0, nbg = 0;
    cudaLaunchConfig_t scfg = {};
    cudaLaunchAttribute sattr[2];
    if (!cluster && g.fused && g.levels >= 2) {
        static int sm_state = 0;  // 0 unknown, 1 ok, -1 unsupported
        if (sm_state == 0) {
            sm_state = cudaFuncSetAttribute(k_mg_pcg_sm, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmBytes) == cudaSuccess ? 1 : -1;
            cudaGetLastError();
        }
        if (sm_state > 0 && gridc) {
            // dense coarsest on all CTAs: no clusters, one CTA per SM
            int occ = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mg_pcg_sm, kSmThreads, kSmBytes) == cudaSuccess && occ >= 1) {
                nbg = std::max(1, std::min({num_sms * occ, num_sms, ceil_div(n, 128)}));
                scfg.gridDim = dim3(nbg);
                scfg.blockDim = dim3(kSmThreads);
                scfg.dynamicSmemBytes = kSmBytes;
                scfg.stream = s;
                sattr[0].id = cudaLaunchAttributeCooperative;
                sattr[0].val.cooperative = 1;
                scfg.attrs = sattr;
                scfg.numAttrs = 1;
                sec = true;
            }
            cudaGetLastError();
        } else if (sm_state > 0) {
            K = std::max(1, std::min({ceil_div(n, kSmCtas * kSmThreads), kSmMaxClusters, num_sms / kSmCtas}));
            scfg.gridDim = dim3(K * kSmCtas);
            scfg.blockDim = dim3(kSmThreads);
            scfg.dynamicSmemBytes = kSmBytes;
            scfg.stream = s;
            sattr[0].id = cudaLaunchAttributeClusterDimension;
            sattr[0].val.clusterDim.x = kSmCtas;
            sattr[0].val.clusterDim.y = 1;
            sattr[0].val.clusterDim.z = 1;
            sattr[1].id = cudaLaunchAttributeCooperative;
            sattr[1].val.cooperative = 1;
            scfg.attrs = sattr;
            scfg.numAttrs = 2;
            int ncl = 0;
            if (cudaOccupancyMaxActiveClusters(&ncl, (void*)k_mg_pcg_sm, &scfg) == cudaSuccess && ncl >= 1) {
                K = std::min(K, ncl);
                scfg.gridDim = dim3(K * kSmCtas);
                sec = true;
            }
            cudaGetLastError();
        }
    }
    if (g.fused && !sec) throw Fail{CICY_E_INTERNAL, "multigrid: the clustered kernel cannot be launched for a hierarchy built for it"};
    int nb = kMgClusterCtas;
    if (sec) {
        nb = gridc ? nbg : K * kSmCtas;
    } else if (!cluster) {
        int occ = 0;
        CICY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mg_pcg<false>, kMgThreads, 0));
        const int cap = std::max(1, occ) * num_sms;
        nb = std::max(1, std::min({cap, num_sms, ceil_div(n, 2 * kMgThreads)}));
    }
    std::vector<MgSmLevel> hl;  // kept until the stream synchronisation below
    MgSmArgs sa{};
    if (sec) {
        // levels lc .. coarsest per cluster: r and z above lc, zf from lc on, K copies each
        const int C = g.levels - 1;
        int lc = C;
        for (int l = 1; l <= C && !gridc; l++)
            if (g.L[l].n <= kSmRows) {
                lc = l;
                break;
            }
        hl.assign(C + 1, MgSmLevel{});
        for (int l = 0; l <= C; l++) {
            MgWork::Lvl& L = g.L[l];
            MgSmLevel& d = hl[l];
            d.n = L.n;
            if (l == 0) continue;
            if (l < C) {
                d.rr_ptr = L.rr_ptr.get();
                d.rr_col = L.rr_col.get();
                d.rr_val = L.rr_val.get();
                d.pq_ptr = L.pq_ptr.get();
                d.pq_col = L.pq_col.get();
                d.pq_val = L.pq_val.get();
                d.agg = L.agg.get();
            }
            d.l1inv = L.l1inv.get();
            if (l > lc) {
                L.r_cl.ensure((size_t)K * L.n + 1);
                L.z_cl.ensure((size_t)K * L.n + 1);
                d.r = L.r_cl.get();
                d.z = L.z_cl.get();
                d.priv |= 1;
            } else {
                d.r = L.r.get();
                d.z = L.z.get();
            }
            if (l >= lc && !gridc) {
                L.zf_cl.ensure((size_t)K * L.n + 1);
                d.zf = L.zf_cl.get();
                d.priv |= 2;
            } else {
                d.zf = L.zf.get();
            }
        }
        g.sec_lv.ensure(sizeof(MgSmLevel) * (C + 1));
        CICY_CUDA(cudaMemcpyAsync(g.sec_lv.get(), hl.data(), sizeof(MgSmLevel) * (C + 1), cudaMemcpyHostToDevice, s));
        const int ncl = ceil_div(nb, kSmCtas);
        g.cl_fail.ensure(ncl);
        CICY_CUDA(cudaMemsetAsync(g.cl_fail.get(), 0, sizeof(int32_t) * ncl, s));
        sa.lc = lc;
        sa.grid_coarse = gridc ? 1 : 0;
        sa.lv = reinterpret_cast<const MgSmLevel*>(g.sec_lv.get());
        sa.cl_fail = g.cl_fail.get();
        sa.mptr0 = g.L[0].mptr.get();
        sa.smem_bytes = kSmBytes;
    }
    w.cta_row.ensure(nb + 1);
    launch_cta_rows(nb, n, w.is_start.get(), w.cta_row.get(), s);
    w.part.ensure(4 * nb + 8);
    g.bar.ensure(1);
    w.stats.ensure(4);
    CICY_CUDA(cudaMemsetAsync(g.bar.get(), 0, sizeof(unsigned long long), s));
    CICY_CUDA(cudaMemsetAsync(w.stats.get(), 0, sizeof(double) * 4, s));
    MgArgs a{};
    a.n = n;
    a.rp = sys.rp; a.ci = sys.ci; a.val = sys.val; a.b = sys.b; a.x = sys.x;
    a.r = w.r.get(); a.z0 = g.z0.get(); a.z = w.z.get(); a.w = g.wtmp.get(); a.p = w.p.get(); a.q = w.q.get();
    a.tinv = w.tinv.get(); a.row_off = w.row_off.get(); a.row_base = w.row_base.get(); a.row_m = w.row_m.get();
    a.cta_row = w.cta_row.get();
    a.levels = g.levels;
    a.lv = g.dev_lv.get();
    a.cinv = g.dense ? g.cinv.get() : nullptr;
    a.omega0 = kOmega0;
    a.partA = w.part.get();
    a.partB = w.part.get() + 2 * nb;
    a.stats = w.stats.get();
    a.bar = g.bar.get();
    a.spin_limit = w.spin_limit;
    a.err = status;
    a.tol = tol;
    a.max_iter = max_iter;
    a.max_restarts = kMgMaxRestarts;
    cudaEvent_t e0, e1;
    CICY_CUDA(cudaEventCreate(&e0));
    CICY_CUDA(cudaEventCreate(&e1));
    CICY_CUDA(cudaEventRecord(e0, s));
    if (cluster) {
        CICY_CUDA(cudaLaunchKernelEx(&cfg, k_mg_pcg<true>, a));
    } else if (sec) {
        CICY_CUDA(cudaLaunchKernelEx(&scfg, k_mg_pcg_sm, a, sa));
    } else {
        void* args[] = {&a};
        CICY_CUDA(cudaLaunchCooperativeKernel((void*)k_mg_pcg<false>, dim3(nb), dim3(kMgThreads), args, 0, s));
    }
    CICY_CUDA(cudaEventRecord(e1, s));
    launches++;
    double hs[4];
    CICY_CUDA(cudaMemcpyAsync(hs, w.stats.get(), sizeof(hs), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st.iterations = (long long)hs[0];
    st.restarts = (int)hs[3];
    st.seconds = ms * 1e-3;
    st.ctas = nb;
    st.levels = g.levels;
    st.cluster = cluster;
}

}  // namespace cicy

namespace cicy {

// ---------------------------------------------------------------------------
// Batched MG solves (used by batch.cu): per-system hierarchies built once, all
// systems solved by k_mg_batch, one 16-CTA cluster per system at a time.
namespace {
__global__ void k_diag_of(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                          double* __restrict__ d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double x = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++)
            if (ci[k] == i) x = v[k];
        d[i] = x;
    }
}
}  // namespace

struct MgBatch {
    std::vector<SolverWork*> works;
    std::vector<DBuf<double>*> diags;
    DBuf<MgArgs> args;
    DBuf<int> queue, slots;
    DBuf<double> stats;
    int count = 0, nclusters = 0;
    double tol = 0;
    ~MgBatch() {
        for (auto* w : works) delete w;
        for (auto* d : diags) {
            d->release();
            delete d;
        }
        args.release();
        queue.release();
        slots.release();
        stats.release();
    }
};

MgBatch* mg_batch_build(const std::vector<MgBatchInput>& in, double tol, long long iter_factor, cudaStream_t s, int64_t& launches) {
    static int cl_attr = 0;
    if (cl_attr == 0) {
        cl_attr = cudaFuncSetAttribute(k_mg_batch, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess ? 1 : -1;
        cudaGetLastError();
    }
    if (cl_attr < 0) throw Fail{CICY_E_DEVICE, "batched multigrid: 16-CTA clusters are not available"};
    MgBatch* B = new MgBatch;
    try {
        B->count = (int)in.size();
        B->tol = tol;
        B->stats.ensure(4 * in.size() + 4);
        std::vector<MgArgs> host(in.size());
        for (size_t k = 0; k < in.size(); k++) {
            const MgBatchInput& x = in[k];
            auto* w = new SolverWork;
            B->works.push_back(w);
            auto* d = new DBuf<double>;
            B->diags.push_back(d);
            d->ensure(x.n + 1);
            k_diag_of<<<grid_for(x.n), 256, 0, s>>>(x.n, x.rp, x.ci, x.val, d->get());
            launches++;
            SolverSystem ss;
            ss.n = x.n;
            ss.nnz = x.nnz;
            ss.rp = x.rp;
            ss.ci = x.ci;
            ss.val = x.val;
            ss.diag = d->get();
            ss.b = x.b;
            ss.x = x.x;
            build_block_preconditioner(*w, ss, x.nchains, x.cs, x.cl, nullptr, nullptr, false, s, launches);
            build_mg_hierarchy(*w, ss, s, launches);
            MgWork& g = w->mg;
            w->r.ensure(x.n); w->z.ensure(x.n); w->p.ensure(x.n); w->q.ensure(x.n);
            g.z0.ensure(x.n);
            g.wtmp.ensure(x.n);
            w->cta_row.ensure(kMgClusterCtas + 1);
            launch_cta_rows(kMgClusterCtas, x.n, w->is_start.get(), w->cta_row.get(), s);
            w->part.ensure(4 * kMgClusterCtas + 8);
            MgArgs a{};
            a.n = x.n;
            a.rp = x.rp; a.ci = x.ci; a.val = x.val; a.b = x.b; a.x = x.x; a.x0 = x.x0;
            a.r = w->r.get(); a.z0 = g.z0.get(); a.z = w->z.get(); a.w = g.wtmp.get(); a.p = w->p.get(); a.q = w->q.get();
            a.tinv = w->tinv.get(); a.row_off = w->row_off.get(); a.row_base = w->row_base.get(); a.row_m = w->row_m.get();
            a.cta_row = w->cta_row.get();
            a.levels = g.levels;
            a.lv = g.dev_lv.get();
            a.cinv = g.dense ? g.cinv.get() : nullptr;
            a.omega0 = kOmega0;
            a.partA = w->part.get();
            a.partB = w->part.get() + 2 * kMgClusterCtas;
            a.stats = B->stats.get() + 4 * k;
            a.bar = nullptr;
            a.spin_limit = kSpinLimit;
            a.err = nullptr;
            a.tol = tol;
            a.max_iter = iter_factor * (long long)x.n;
            a.max_restarts = kMgMaxRestarts;
            a.cap_b = 1;
            host[k] = a;
        }
        B->args.ensure(in.size());
        CICY_CUDA(cudaMemcpyAsync(B->args.get(), host.data(), sizeof(MgArgs) * in.size(), cudaMemcpyHostToDevice, s));
        B->queue.ensure(1);
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        cfg.gridDim = dim3(kMgClusterCtas);
        cfg.blockDim = dim3(kMgClusterThreads);
        cfg.stream = s;
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kMgClusterCtas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        CICY_CUDA(cudaOccupancyMaxActiveClusters(&nclusters, (void*)k_mg_batch, &cfg));
        if (nclusters < 1) throw Fail{CICY_E_DEVICE, "batched multigrid: no 16-CTA cluster fits"};
        B->nclusters = std::min(nclusters, B->count);
        B->slots.ensure(B->nclusters + 1);
        CICY_CUDA(cudaStreamSynchronize(s));
        CICY_LAUNCH_CHECK();
    } catch (...) {
        delete B;
        throw;
    }
    return B;
}

void mg_batch_enqueue(MgBatch* B, cudaStream_t s) {
    CICY_CUDA(cudaMemsetAsync(B->queue.get(), 0, sizeof(int), s));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(kMgClusterCtas * B->nclusters);
    cfg.blockDim = dim3(kMgClusterThreads);
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kMgClusterCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CICY_CUDA(cudaLaunchKernelEx(&cfg, k_mg_batch, (const MgArgs*)B->args.get(), B->count, B->queue.get(), B->slots.get()));
}

void mg_batch_stats(MgBatch* B, std::vector<double>& stats, cudaStream_t s) {
    stats.resize(4 * (size_t)B->count);
    CICY_CUDA(cudaMemcpyAsync(stats.data(), B->stats.get(), sizeof(double) * 4 * B->count, cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
}

int mg_batch_clusters(const MgBatch* B) { return B->nclusters; }

void mg_batch_free(MgBatch* B) { delete B; }

}  // namespace cicy
