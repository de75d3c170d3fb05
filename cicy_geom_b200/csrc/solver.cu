// Preconditioned conjugate gradient for the DEA systems (device).
//
// One persistent cooperative launch per solve.  Rows are partitioned over CTAs
// at CNT-chain boundaries, so the block preconditioner of a row only reads rows
// of its own CTA (a __syncthreads() suffices between r and z); the grid-wide
// barriers per iteration are two: after the residual/preconditioner phase
// (partials r.r, r.z) and after the search-direction phase (partial p.q):
//
//   B: x += a p ; r -= a q ; z = M^-1 r ; partials (r.r, r.z)       | grid barrier
//   A: w = A z ; q = w + b q ; p = z + b p ; partial (p.q)          | grid barrier
//
// which is the recurrence of Solve_DEA_equations_CG_SSS
// (Direct_Electrifying.cpp:1538-1659) with q = A p carried as A z + beta q.
// When the recursive residual meets |r| <= tol |r0|, the FP64 true residual
// b - A x replaces it (a restart) until the true residual meets the test too
// (at most kMaxRestarts times): iterative refinement in FP64.
//
// Preconditioners: Jacobi (upstream, Direct_Electrifying.cpp:1662-1676), and a
// block-Jacobi over CNT chains: the free nodes of one CNT are consecutive node
// ids (LM_matrix_for_cnts numbers them in element order) coupled only by the
// CNT's element resistors, so each chain's diagonal block is tridiagonal.  Chains
// are split into blocks of at most kBlockMax nodes whose inverses are formed
// explicitly at setup, so applying the preconditioner is a dense block mat-vec
// per row (no sequential sweep on the iteration's critical path).  The learned
// preconditioner is this block family with per-node and per-edge scalings.
//
// Mixed precision: q = A p is computed afresh each iteration (not carried as
// A z + beta q, whose FP32 rounding would accumulate) in FP32 difference form,
//   (A p)_i = rs_i p_i + sum_j g_ij (p_i - p_j)   (rs_i = row sum, g_ij = -a_ij),
// whose terms are edge currents (the differences are taken in FP64, then
// rounded), so the 1e4-1e10 spread between CNT and junction conductances does
// not cancel catastrophically as in an FP32 A p.  The new p of a neighbour row
// is rebuilt from z and the previous p (two p buffers), so this needs no extra
// grid barrier.  The preconditioner apply uses FP32 copies of the block
// inverses.  x, r, z, p, q, the dot products and the FP64 residual replacement
// (every time the recursive residual fell by inner_drop; search directions
// kept) stay FP64.
#include <algorithm>
#include <cmath>

#include "solver.cuh"

namespace cicy {

namespace {

constexpr int kCgThreads = 256;
constexpr int kMaxRestarts = 24;
constexpr int kMaxRestartsMixed = 400;

int grid_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)b;
}

// ---------------------------------------------------------------------------
// Preconditioner setup
__global__ void k_jacobi(int n, const double* __restrict__ diag, double* __restrict__ minv, float* __restrict__ minv32) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double m = 1 / diag[i];
        minv[i] = m;
        if (minv32) minv32[i] = (float)m;
    }
}

// Block starts: chain starts, and every kBlockMax-th node inside a chain.
__global__ void k_block_marks(int nchains, const int32_t* __restrict__ cstart, const int32_t* __restrict__ clen,
                              int32_t* __restrict__ is_start) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nchains; c += gridDim.x * blockDim.x)
        for (int k = 0; k < clen[c]; k += kBlockMax) is_start[cstart[c] + k] = 1;
}

__global__ void k_block_fill(int n, const int32_t* __restrict__ is_start, const int32_t* __restrict__ start_scan,
                             int32_t* __restrict__ blk_row) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (is_start[i]) blk_row[start_scan[i]] = i;
}

__global__ void k_block_sizes(int nb, int n, const int32_t* __restrict__ blk_row, int32_t* __restrict__ msq) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        int m = ((b + 1 < nb) ? blk_row[b + 1] : n) - blk_row[b];
        msq[b] = m * m;
    }
}

// Off-diagonal A[i][i+1] inside a block (0 if absent).
__device__ __forceinline__ double upper_entry(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                              const double* __restrict__ v, int i) {
    for (int k = rp[i]; k < rp[i + 1]; k++)
        if (ci[k] == i + 1) return v[k];
    return 0.0;
}

// Explicit inverse of one tridiagonal SPD block (LDL^T solves, one column at a time).
// Learned scalings: diagonal d'_k = c_k + s_k (d_k - c_k) with c_k the block coupling
// of row k; off-diagonal e'_k = t_k e_k.  s = t = 1 reproduces the exact block.
__global__ void k_block_inverse(int nb, int n, const int32_t* __restrict__ blk_row, const int32_t* __restrict__ blk_off,
                                const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                                const double* __restrict__ diag, const float* __restrict__ node_scale,
                                const float* __restrict__ edge_scale, double* __restrict__ tinv, float* __restrict__ tinv32,
                                int32_t* __restrict__ row_off, int32_t* __restrict__ row_base, int32_t* __restrict__ row_m) {
    double d[kBlockMax], e[kBlockMax], l[kBlockMax], piv[kBlockMax], y[kBlockMax];
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int r0 = blk_row[b];
        const int m = ((b + 1 < nb) ? blk_row[b + 1] : n) - r0;
        const int off = blk_off[b];
        for (int k = 0; k < m; k++) {
            d[k] = diag[r0 + k];
            e[k] = (k + 1 < m) ? upper_entry(rp, ci, v, r0 + k) : 0.0;
        }
        for (int k = 0; k < m; k++) {
            double coup = fabs(e[k]) + (k > 0 ? fabs(e[k - 1]) : 0.0);
            double s = node_scale ? (double)node_scale[r0 + k] : 1.0;
            d[k] = coup + s * (d[k] - coup);
        }
        if (edge_scale)
            for (int k = 0; k + 1 < m; k++) e[k] *= (double)edge_scale[r0 + k];
        // LDL^T of the tridiagonal block
        piv[0] = d[0];
        l[0] = 0;
        bool singular = !(piv[0] > 1e-13 * fabs(d[0]));
        for (int k = 1; k < m; k++) {
            l[k] = e[k - 1] / piv[k - 1];
            piv[k] = d[k] - l[k] * e[k - 1];
            singular |= !(piv[k] > 1e-13 * fabs(d[k]));
        }
        if (singular) {
            // A CNT with no coupling outside its own element chain (possible in a
            // single-direction pass: upstream drops junctions touching a prescribed
            // node) has a singular Laplacian block; use its diagonal instead.
            for (int k = 0; k < m; k++)
                for (int j = 0; j < m; j++) {
                    double t = (j == k) ? 1.0 / diag[r0 + k] : 0.0;
                    tinv[off + k * m + j] = t;
                    if (tinv32) tinv32[off + k * m + j] = (float)t;
                }
            for (int k = 0; k < m; k++) {
                row_off[r0 + k] = off + k * m;
                row_base[r0 + k] = r0;
                row_m[r0 + k] = m;
            }
            continue;
        }
        for (int j = 0; j < m; j++) {
            for (int k = 0; k < m; k++) y[k] = (k == j) ? 1.0 : 0.0;
            for (int k = 1; k < m; k++) y[k] -= l[k] * y[k - 1];
            y[m - 1] = y[m - 1] / piv[m - 1];
            for (int k = m - 2; k >= 0; k--) y[k] = y[k] / piv[k] - l[k + 1] * y[k + 1];
            for (int k = 0; k < m; k++) {
                tinv[off + k * m + j] = y[k];
                if (tinv32) tinv32[off + k * m + j] = (float)y[k];
            }
        }
        for (int k = 0; k < m; k++) {
            row_off[r0 + k] = off + k * m;
            row_base[r0 + k] = r0;
            row_m[r0 + k] = m;
        }
    }
}

// CTA row ranges that never split a block: CTA b starts at the first block start
// at or after b * n / nb.
__global__ void k_cta_rows(int nb_cta, int n, const int32_t* __restrict__ is_start, int32_t* __restrict__ cta_row) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= nb_cta; b += gridDim.x * blockDim.x) {
        if (b == nb_cta) { cta_row[b] = n; continue; }
        long long r = (long long)b * n / nb_cta;
        while (r < n && !is_start[r]) r++;
        cta_row[b] = (int)r;
    }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ void block_reduce2(double a, double b, double* sm, double& ra, double& rb) {
    a = warp_sum(a);
    b = warp_sum(b);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sm[w] = a; sm[32 + w] = b; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        double x = lane < nw ? sm[lane] : 0.0, y = lane < nw ? sm[32 + lane] : 0.0;
        x = warp_sum(x);
        y = warp_sum(y);
        if (lane == 0) { sm[64] = x; sm[65] = y; }
    }
    __syncthreads();
    ra = sm[64];
    rb = sm[65];
    __syncthreads();
}

__device__ __forceinline__ void sum_partials(const double* part, int stride, int nb, double* sm, double& s0, double& s1) {
    if (threadIdx.x < 32) {
        double a = 0, b = 0;
        for (int i = threadIdx.x; i < nb; i += 32) {
            a += __ldcg(&part[i * stride]);
            if (stride > 1) b += __ldcg(&part[i * stride + 1]);
        }
        a = warp_sum(a);
        b = warp_sum(b);
        if (threadIdx.x == 0) { sm[66] = a; sm[67] = b; }
    }
    __syncthreads();
    s0 = sm[66];
    s1 = sm[67];
    __syncthreads();
}

template <int PRE, bool MIXED>
struct Vec {
    using T = typename std::conditional<MIXED, float, double>::type;
};

template <int PRE, bool MIXED>
__device__ __forceinline__ double apply_precond(const PcgArgs& a, int i) {
    if (PRE == PRECOND_KIND_JACOBI) {
        if (MIXED) return (double)(a.minv32[i] * (float)a.r[i]);
        return a.minv[i] * a.r[i];
    } else {
        const int off = a.row_off[i], base = a.row_base[i], m = a.row_m[i];
        if (MIXED) {
            float s = 0;
            for (int j = 0; j < m; j++) s += a.tinv32[off + j] * (float)a.r[base + j];
            return (double)s;
        }
        double s = 0;
        for (int j = 0; j < m; j++) s += a.tinv[off + j] * a.r[base + j];
        return s;
    }
}

// z = M^-1 r on this CTA's rows, accumulating r.r and r.z.  The SPAI form needs
// y = T^-1 r of neighbouring rows in other CTAs: one extra grid barrier.
template <int PRE, bool MIXED>
__device__ __forceinline__ bool precond_all(const PcgArgs& a, int r_lo, int r_hi, double& rr_l, double& rz_l) {
    if constexpr (PRE == PRECOND_KIND_SPAI) {
        for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) a.y[i] = apply_precond<PRECOND_KIND_BLOCK, MIXED>(a, i);
        if (!grid_sync(a.bar, gridDim.x, a.err)) return false;
        for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
            if constexpr (MIXED) {
                float s = 0;
                for (int k = a.rp[i]; k < a.rp[i + 1]; k++) {
                    const float w = a.ew[k];
                    if (w != 0.0f) s += w * a.val32[k] * (float)__ldcg(&a.y[a.ci[k]]);
                }
                a.u[i] = (double)s;
            } else {
                double s = 0;
                for (int k = a.rp[i]; k < a.rp[i + 1]; k++) {
                    const float w = a.ew[k];
                    if (w != 0.0f) s += (double)w * (-a.val[k]) * __ldcg(&a.y[a.ci[k]]);
                }
                a.u[i] = s;
            }
        }
        __syncthreads();
        for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
            const int off = a.row_off[i], base = a.row_base[i], m = a.row_m[i];
            double s;
            if constexpr (MIXED) {
                float f = 0;
                for (int j = 0; j < m; j++) f += a.tinv32[off + j] * (float)a.u[base + j];
                s = a.y[i] + (double)f;
            } else {
                s = a.y[i];
                for (int j = 0; j < m; j++) s += a.tinv[off + j] * a.u[base + j];
            }
            a.z[i] = s;
            const double ri = a.r[i];
            rr_l += ri * ri;
            rz_l += ri * s;
        }
        return true;
    } else {
        for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
            const double zi = apply_precond<PRE, MIXED>(a, i);
            a.z[i] = zi;
            double ri = a.r[i];
            rr_l += ri * ri;
            rz_l += ri * zi;
        }
        return true;
    }
}

template <bool MIXED>
__device__ __forceinline__ double spmv_row_z(const PcgArgs& a, int i) {
    double s = 0;
    for (int k = a.rp[i]; k < a.rp[i + 1]; k++) s += a.val[k] * a.z[a.ci[k]];
    return s;
}

template <int PRE, bool MIXED>
__global__ void __launch_bounds__(kCgThreads) k_pcg(PcgArgs a) {
    __shared__ double sm[72];
    const int nb = gridDim.x;
    const int r_lo = a.cta_row[blockIdx.x], r_hi = a.cta_row[blockIdx.x + 1];
    // ---- start: r = b - A x0 given; z = M r; partials r.r, r.z
    double rr_l = 0, rz_l = 0;
    if (!precond_all<PRE, MIXED>(a, r_lo, r_hi, rr_l, rz_l)) return;
    double s0, s1;
    block_reduce2(rr_l, rz_l, sm, s0, s1);
    if (threadIdx.x == 0) { a.partA[2 * blockIdx.x] = s0; a.partA[2 * blockIdx.x + 1] = s1; }
    if (!grid_sync(a.bar, nb, a.err)) return;
    double rr, rz;
    sum_partials(a.partA, 2, nb, sm, rr, rz);
    const double R0 = a.tol * sqrt(rr);
    // mixed precision: the FP64 true residual replaces the recursive one each time
    // the latter has dropped by inner_drop (the search directions are kept)
    double anchor = sqrt(rr);
    double beta = 0.0, rr_new = rr, pq = 0, dummy;
    long long k = 0;
    int restarts = 0;
    bool fresh = true;  // first step or restart: p = z, q = A z (old p, q are not read)
    while (true) {
        // ---- A: FP64: w = A z, q = w + beta q, p = z + beta p, partial p.q
        //         mixed: p = z + beta p_old into the other p buffer, q = A p directly
        //         (FP32 difference form; p_j of other rows rebuilt from z_j and
        //         p_old_j), so FP32 rounding does not accumulate in q over iterations
        double* pcur = a.p;
        double pq_l = 0;
        if constexpr (MIXED) {
            const double* po = (k & 1) ? a.p2 : a.p;
            pcur = (k & 1) ? a.p : a.p2;
            const double bt = fresh ? 0.0 : beta;
            for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
                const double pi = fresh ? a.z[i] : a.z[i] + bt * po[i];
                float f = a.rs32[i] * (float)pi;
                for (int kk = a.rp[i]; kk < a.rp[i + 1]; kk++) {
                    const int j = a.ci[kk];
                    const double pj = fresh ? a.z[j] : a.z[j] + bt * po[j];
                    f += a.val32[kk] * (float)(pi - pj);
                }
                const double qi = (double)f;
                pcur[i] = pi;
                a.q[i] = qi;
                pq_l += pi * qi;
            }
        } else {
            for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
                const double w = spmv_row_z<false>(a, i);
                const double zi = a.z[i];
                const double qi = fresh ? w : w + beta * a.q[i];
                const double pi = fresh ? zi : zi + beta * a.p[i];
                a.q[i] = qi;
                a.p[i] = pi;
                pq_l += pi * qi;
            }
        }
        block_reduce2(pq_l, 0.0, sm, s0, s1);
        if (threadIdx.x == 0) a.partB[blockIdx.x] = s0;
        if (!grid_sync(a.bar, nb, a.err)) return;
        sum_partials(a.partB, 1, nb, sm, pq, dummy);
        fresh = false;
        k++;
        // ---- B: x += alpha p, r -= alpha q, z = M r, partials r.r, r.z
        // mixed: breakdown (p.Ap <= 0 from FP32 rounding) stops with x intact; FP64
        // keeps the upstream arithmetic (a zero initial residual gives 0/0 = NaN there)
        if (MIXED && (!(pq > 0) || !(rz > 0))) break;
        const double alpha = rz / pq;
        for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
            const double pi = pcur[i];
            const double qi = a.q[i];
            a.x[i] += alpha * pi;
            a.r[i] -= alpha * qi;
        }
        __syncthreads();  // the block preconditioner reads r of this CTA's other rows
        rr_l = 0;
        rz_l = 0;
        if (!precond_all<PRE, MIXED>(a, r_lo, r_hi, rr_l, rz_l)) return;
        block_reduce2(rr_l, rz_l, sm, s0, s1);
        if (threadIdx.x == 0) { a.partA[2 * blockIdx.x] = s0; a.partA[2 * blockIdx.x + 1] = s1; }
        if (!grid_sync(a.bar, nb, a.err)) return;
        double rz_new;
        sum_partials(a.partA, 2, nb, sm, rr_new, rz_new);
        const double rz_prev = rz;
        beta = rz_new / rz;
        rz = rz_new;
        if (sqrt(rr_new) <= R0 || (MIXED && sqrt(rr_new) <= a.inner_drop * anchor)) {
            if (restarts >= a.max_restarts) break;
            // ---- FP64 true residual r = b - A x (x is complete after the barrier above)
            rr_l = 0;
            for (int i = r_lo + threadIdx.x; i < r_hi; i += blockDim.x) {
                double s = 0;
                for (int kk = a.rp[i]; kk < a.rp[i + 1]; kk++) s += a.val[kk] * a.x[a.ci[kk]];
                double ri = a.b[i] - s;
                a.r[i] = ri;
            }
            __syncthreads();
            rz_l = 0;
            if (!precond_all<PRE, MIXED>(a, r_lo, r_hi, rr_l, rz_l)) return;
            block_reduce2(rr_l, rz_l, sm, s0, s1);
            if (threadIdx.x == 0) { a.partA[2 * blockIdx.x] = s0; a.partA[2 * blockIdx.x + 1] = s1; }
            if (!grid_sync(a.bar, nb, a.err)) return;
            sum_partials(a.partA, 2, nb, sm, rr_new, rz);
            restarts++;
            anchor = sqrt(rr_new);
            if (sqrt(rr_new) <= R0) break;
            if (MIXED) beta = rz / rz_prev;  // residual replacement: continue the directions
            else fresh = true;               // restart from the true residual
        }
        if (k >= a.max_iter) break;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.stats[0] = (double)k;
        a.stats[1] = rr_new;
        a.stats[2] = R0;
        a.stats[3] = (double)restarts;
    }
}

template <int PRE, bool MIXED>
void launch_pcg(PcgArgs& a, int nb, cudaStream_t s) {
    void* args[] = {&a};
    CICY_CUDA(cudaLaunchCooperativeKernel((void*)k_pcg<PRE, MIXED>, dim3(nb), dim3(kCgThreads), args, 0, s));
}

template <int PRE, bool MIXED>
int max_coop_blocks(int sms) {
    int occ = 0;
    CICY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pcg<PRE, MIXED>, kCgThreads, 0));
    return std::max(1, occ) * sms;
}

// FP32 conductances (g = -a off the diagonal, 0 on it) and FP32 row sums (FP64 sums).
__global__ void k_mixed_prep(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                             float* __restrict__ g, float* __restrict__ rs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            s += v[k];
            g[k] = ci[k] == i ? 0.0f : (float)(-v[k]);
        }
        rs[i] = (float)s;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
void build_block_preconditioner(SolverWork& w, const SolverSystem& sys, int nchains, const int32_t* chain_start,
                                const int32_t* chain_len, const float* node_scale, const float* edge_scale, bool mixed,
                                cudaStream_t s, int64_t& launches) {
    const int n = sys.n;
    w.total.ensure(2);
    w.is_start.ensure(n + 1);
    w.start_scan.ensure(n + 1);
    CICY_CUDA(cudaMemsetAsync(w.is_start.get(), 0, sizeof(int32_t) * (n + 1), s));
    k_block_marks<<<grid_for(nchains), 256, 0, s>>>(nchains, chain_start, chain_len, w.is_start.get());
    exclusive_scan_i32(w.is_start.get(), w.start_scan.get(), n, w.total.get(), w.scan_tmp, s, launches);
    int nblk = 0;
    CICY_CUDA(cudaMemcpyAsync(&nblk, w.total.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    w.blk_row.ensure(nblk + 1);
    w.blk_msq.ensure(nblk + 1);
    w.blk_off.ensure(nblk + 1);
    k_block_fill<<<grid_for(n), 256, 0, s>>>(n, w.is_start.get(), w.start_scan.get(), w.blk_row.get());
    k_block_sizes<<<grid_for(nblk), 256, 0, s>>>(nblk, n, w.blk_row.get(), w.blk_msq.get());
    exclusive_scan_i32(w.blk_msq.get(), w.blk_off.get(), nblk, w.total.get(), w.scan_tmp, s, launches);
    // the blocks' m^2 entries sum to at most kBlockMax per row: sized by that bound, no host read
    const size_t tot = (size_t)std::max(n, 1) * kBlockMax;
    w.tinv.ensure(tot);
    if (mixed) w.tinv32.ensure(tot);
    w.row_off.ensure(n + 1);
    w.row_base.ensure(n + 1);
    w.row_m.ensure(n + 1);
    k_block_inverse<<<grid_for(nblk, 128), 128, 0, s>>>(nblk, n, w.blk_row.get(), w.blk_off.get(), sys.rp, sys.ci, sys.val, sys.diag,
                                                       node_scale, edge_scale, w.tinv.get(), mixed ? w.tinv32.get() : nullptr,
                                                       w.row_off.get(), w.row_base.get(), w.row_m.get());
    launches += 4;
    CICY_LAUNCH_CHECK();
    w.n_blocks = nblk;
}

void pcg_solve(SolverWork& w, const SolverSystem& sys, int precond, bool mixed, double tol, long long max_iter, int num_sms,
               int* status, cudaStream_t s, int64_t& launches, PcgStats& st, const float* ew) {
    if (precond == PRECOND_KIND_SPAI && !ew) throw Fail{CICY_E_INTERNAL, "SPAI preconditioner: weights required"};
    const int n = sys.n;
    st = PcgStats{};
    if (n <= 0) return;
    // vectors
    w.r.ensure(n); w.z.ensure(n); w.p.ensure(n); w.q.ensure(n);
    if (mixed) {
        w.val32.ensure(std::max(sys.nnz, 1)); w.rs32.ensure(n); w.p2.ensure(n);
        k_mixed_prep<<<grid_for(n), 256, 0, s>>>(n, sys.rp, sys.ci, sys.val, w.val32.get(), w.rs32.get());
        launches++;
    }
    // r = b - A x0
    k_residual<<<grid_for(n), 256, 0, s>>>(n, sys.rp, sys.ci, sys.val, sys.x, sys.b, w.r.get());
    launches++;
    if (precond == PRECOND_KIND_JACOBI) {
        w.minv.ensure(n);
        if (mixed) w.minv32.ensure(n);
        k_jacobi<<<grid_for(n), 256, 0, s>>>(n, sys.diag, w.minv.get(), mixed ? w.minv32.get() : nullptr);
        launches++;
        w.is_start.ensure(n + 1);
        // any row may start a CTA range under Jacobi
        k_fill_ones<<<grid_for(n), 256, 0, s>>>(n, w.is_start.get());
        launches++;
    }
    // CTA row ranges
    int cap = 0;
    if (precond == PRECOND_KIND_JACOBI) cap = mixed ? max_coop_blocks<PRECOND_KIND_JACOBI, true>(num_sms) : max_coop_blocks<PRECOND_KIND_JACOBI, false>(num_sms);
    else if (precond == PRECOND_KIND_SPAI) cap = mixed ? max_coop_blocks<PRECOND_KIND_SPAI, true>(num_sms) : max_coop_blocks<PRECOND_KIND_SPAI, false>(num_sms);
    else cap = mixed ? max_coop_blocks<PRECOND_KIND_BLOCK, true>(num_sms) : max_coop_blocks<PRECOND_KIND_BLOCK, false>(num_sms);
    const int nb = std::max(1, std::min({cap, num_sms, ceil_div(n, kCgThreads)}));
    w.cta_row.ensure(nb + 1);
    k_cta_rows<<<1, 256, 0, s>>>(nb, n, w.is_start.get(), w.cta_row.get());
    w.part.ensure(4 * nb + 8);
    w.barrier.ensure(2);
    w.stats.ensure(4);
    CICY_CUDA(cudaMemsetAsync(w.barrier.get(), 0, sizeof(unsigned) * 2, s));
    CICY_CUDA(cudaMemsetAsync(w.stats.get(), 0, sizeof(double) * 4, s));
    launches++;
    PcgArgs a{};
    a.n = n;
    a.rp = sys.rp; a.ci = sys.ci; a.val = sys.val; a.val32 = mixed ? w.val32.get() : nullptr; a.rs32 = mixed ? w.rs32.get() : nullptr;
    a.b = sys.b; a.x = sys.x; a.r = w.r.get();
    a.z = w.z.get(); a.p = w.p.get(); a.q = w.q.get(); a.p2 = mixed ? w.p2.get() : nullptr;
    a.minv = w.minv.get(); a.minv32 = w.minv32.get();
    a.tinv = w.tinv.get(); a.tinv32 = w.tinv32.get();
    a.row_off = w.row_off.get(); a.row_base = w.row_base.get(); a.row_m = w.row_m.get();
    a.cta_row = w.cta_row.get();
    if (precond == PRECOND_KIND_SPAI) {
        w.y.ensure(n);
        w.u.ensure(n);
        a.y = w.y.get();
        a.u = w.u.get();
        a.ew = ew;
    }
    a.partA = w.part.get(); a.partB = w.part.get() + 2 * nb;
    a.stats = w.stats.get();
    a.bar = GridBarrier{w.barrier.get(), w.barrier.get() + 1, w.spin_limit};
    a.err = status;
    a.tol = tol;
    a.max_iter = max_iter;
    a.max_restarts = mixed ? kMaxRestartsMixed : kMaxRestarts;
    a.inner_drop = 1e-2;
    cudaEvent_t e0, e1;
    CICY_CUDA(cudaEventCreate(&e0));
    CICY_CUDA(cudaEventCreate(&e1));
    CICY_CUDA(cudaEventRecord(e0, s));
    if (precond == PRECOND_KIND_JACOBI) {
        if (mixed) launch_pcg<PRECOND_KIND_JACOBI, true>(a, nb, s); else launch_pcg<PRECOND_KIND_JACOBI, false>(a, nb, s);
    } else if (precond == PRECOND_KIND_SPAI) {
        if (mixed) launch_pcg<PRECOND_KIND_SPAI, true>(a, nb, s); else launch_pcg<PRECOND_KIND_SPAI, false>(a, nb, s);
    } else {
        if (mixed) launch_pcg<PRECOND_KIND_BLOCK, true>(a, nb, s); else launch_pcg<PRECOND_KIND_BLOCK, false>(a, nb, s);
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
}

__global__ void k_residual(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                           const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ r) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++) s += v[k] * x[ci[k]];
        r[i] = b[i] - s;
    }
}

__global__ void k_fill_ones(int n, int32_t* __restrict__ a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) a[i] = 1;
}

}  // namespace cicy

namespace cicy {

// Host wrappers shared with the cluster solver (solver_cluster.cu).
void launch_block_marks(int nchains, const int32_t* chain_start, const int32_t* chain_len, int32_t* is_start, cudaStream_t s) {
    if (nchains > 0) k_block_marks<<<grid_for(nchains), 256, 0, s>>>(nchains, chain_start, chain_len, is_start);
}

void launch_block_fill(int n, const int32_t* is_start, const int32_t* start_scan, int32_t* blk_row, cudaStream_t s) {
    k_block_fill<<<grid_for(n), 256, 0, s>>>(n, is_start, start_scan, blk_row);
}

void launch_cta_rows(int nb_cta, int n, const int32_t* is_start, int32_t* cta_row, cudaStream_t s) {
    k_cta_rows<<<1, 256, 0, s>>>(nb_cta, n, is_start, cta_row);
}

}  // namespace cicy

namespace cicy {

// Exported launchers of the FP64 Jacobi kernels for the allocation-free entry point (noalloc.cu).
void launch_jacobi_fp64(int n, const double* diag, double* minv, cudaStream_t s) {
    k_jacobi<<<grid_for(n), 256, 0, s>>>(n, diag, minv, nullptr);
}

int max_coop_blocks_jacobi_fp64(int num_sms) { return max_coop_blocks<PRECOND_KIND_JACOBI, false>(num_sms); }

void launch_pcg_jacobi_fp64(PcgArgs& a, int nb, cudaStream_t s) { launch_pcg<PRECOND_KIND_JACOBI, false>(a, nb, s); }

}  // namespace cicy
