// Batched Monte-Carlo solves: many independent DEA systems of uneven size.
//
// Method 0: one persistent kernel launch (captured in a CUDA graph and
// replayed).  Each CTA takes the next system from a largest-first queue (an
// atomic counter) and solves it alone with preconditioned CG; reductions are
// CTA-local (__syncthreads only), so an iteration costs a few hundred
// nanoseconds of synchronisation instead of the microseconds of a grid barrier.
// Preconditioners:
//   - Jacobi: z = r / diag (the upstream algorithm, Direct_Electrifying.cpp:1662-1676);
//   - chain: whole-chain block-Jacobi (each CNT's free nodes form one
//     tridiagonal block; LDL^T factored at the start of the system's solve by
//     one thread per chain, forward/backward sweeps per chain each iteration;
//     a singular block falls back to its diagonal);
//   - learned: T^-1 + T^-1 E_w T^-1 with T the chain blocks split every 32
//     nodes (the blocks the weights were trained on; the split is an LDL^T
//     multiplier of 0, so the same sweeps apply) and E_w the off-block
//     couplings scaled by the graph network's weights.
// Precision: FP64, or mixed: FP32 conductances in a difference-form SpMV,
//   q_i = rs_i p_i + sum_j g_ij (p_i - p_j)   (rs_i = row sum of A, g_ij = -a_ij),
// whose FP32 terms are edge currents (differences taken in FP64), so the
// 1e4-1e10 spread between CNT and junction conductances does not cancel
// catastrophically as in an FP32 A p; FP32 preconditioner factors; FP64 x, r,
// p, dots, and FP64 residual replacement each time |r| has fallen 100x.
// Stop when |r| <= tol min(|r0|, |b|): the test of Direct_Electrifying.cpp:1571,
// 1619 and the FP64-verified |b - A x| <= tol |b|, confirmed on the true residual.
//
// Method 2 solves the systems one after another with the per-network
// grid-wide persistent PCG; method 1 (multigrid, one cluster per system) lives
// in solver_mg.cu.  Per-system scratch lives in one device buffer with a fixed
// offset per system.  The autotuner times the candidate launch shapes
// (threads per CTA, CTAs per SM) on the batch itself and keeps the fastest.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <type_traits>
#include <vector>

#include "cicy_internal.h"
#include "csr_check.cuh"
#include "dev_common.cuh"
#include "solver.cuh"

namespace cicy {
namespace {

constexpr int kBatchRestarts = 24;       // FP64: true-residual restarts
constexpr int kBatchReplacements = 400;  // mixed: FP64 residual replacements
constexpr double kReplaceDrop = 1e-2;    // mixed: replace r once |r| fell by this factor since the last replacement
constexpr int kSpaiBlock = kBlockMax;    // block length of the learned preconditioner's T

struct BatchSys {
    int n, nnz, nchains;
    const int32_t* rp;
    const int32_t* ci;
    const double* val;
    const double* b;
    const double* x0;
    double* x;
    const int32_t* cs;
    const int32_t* cl;
    const float* ew;
    long long off;  // scratch offset (doubles)
};

// Scratch doubles of one system: r p q z y u (6n), factors (2n), FP32 g and row sums.
inline long long batch_scratch(long long n, long long nnz) {
    long long d = 8 * n + (nnz + n + 1) / 2 + 2;
    return (d + 1) & ~1LL;  // 16-byte aligned offsets
}

struct BatchArgs {
    const BatchSys* sys;
    const int* order;  // largest first
    int count;         // this launch takes order[first .. count)
    int first;
    int* queue;
    int* slots;        // cluster kernel: the system index of each cluster
    double* part;      // cluster kernel: partial sums, [cluster][bank][rank][2]
    double* scratch;
    double tol;
    long long iter_factor;
    long long* iterations;
    double* rel;
    int* flags;  // per system: 1 reached the tolerance, 2 hit the iteration cap
};

template <int T>
__device__ __forceinline__ double cta_sum(double v, double* sm) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = v;
    __syncthreads();
    if (w == 0) {
        double x = lane < T / 32 ? sm[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sm[32] = x;
    }
    __syncthreads();
    const double r = sm[32];
    __syncthreads();
    return r;
}

template <int T>
__device__ __forceinline__ void cta_sum2(double a, double b, double* sm, double& ra, double& rb) {
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sm[w] = a; sm[40 + w] = b; }
    __syncthreads();
    if (w == 0) {
        double x = lane < T / 32 ? sm[lane] : 0.0, y = lane < T / 32 ? sm[40 + lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            x += __shfl_xor_sync(0xffffffffu, x, o);
            y += __shfl_xor_sync(0xffffffffu, y, o);
        }
        if (lane == 0) { sm[32] = x; sm[33] = y; }
    }
    __syncthreads();
    ra = sm[32];
    rb = sm[33];
    __syncthreads();
}

__device__ __forceinline__ double upper(const BatchSys& S, int i) {
    for (int k = S.rp[i]; k < S.rp[i + 1]; k++)
        if (S.ci[k] == i + 1) return S.val[k];
    return 0.0;
}

__device__ __forceinline__ double diag_of(const BatchSys& S, int i) {
    for (int k = S.rp[i]; k < S.rp[i + 1]; k++)
        if (S.ci[k] == i) return S.val[k];
    return 0.0;
}

// LDL^T of every chain block (blocks of BLK nodes, BLK = 0: whole chains):
// lf[i] = l_i (multiplier, 0 at a block start), ip[i] = 1 / pivot_i; a singular
// block stores l = 0 and 1 / diag (its diagonal).
template <typename PT, int BLK>
__device__ void factor_chains(const BatchSys& S, PT* lf, PT* ip) {
    for (int c = threadIdx.x; c < S.nchains; c += blockDim.x) {
        const int s0 = S.cs[c], m = S.cl[c];
        const int bl = BLK > 0 ? BLK : m;
        for (int b0 = 0; b0 < m; b0 += bl) {
            const int bm = min(bl, m - b0);
            bool singular = false;
            double piv_prev = 0, e_prev = 0;
            for (int k = 0; k < bm; k++) {
                const int i = s0 + b0 + k;
                const double d = diag_of(S, i);
                double l = 0, piv = d;
                if (k > 0) {
                    l = e_prev / piv_prev;
                    piv = d - l * e_prev;
                }
                singular |= !(piv > 1e-13 * fabs(d));
                lf[i] = (PT)l;
                ip[i] = (PT)(1.0 / piv);
                piv_prev = piv;
                e_prev = (k + 1 < bm) ? upper(S, i) : 0.0;
            }
            if (singular)
                for (int k = 0; k < bm; k++) {
                    const int i = s0 + b0 + k;
                    lf[i] = (PT)0;
                    ip[i] = (PT)(1.0 / diag_of(S, i));
                }
        }
    }
}

// z = T^-1 r chain by chain: forward (y_k = r_k - l_k y_{k-1}), backward
// (z_k = y_k / p_k - l_{k+1} z_{k+1}); l = 0 at block starts ends a block.
template <typename PT>
__device__ void apply_chains(const BatchSys& S, const PT* lf, const PT* ip, const double* r, double* z) {
    for (int c = threadIdx.x; c < S.nchains; c += blockDim.x) {
        const int s0 = S.cs[c], m = S.cl[c];
        if (m <= 0) continue;
        PT y = (PT)r[s0];
        z[s0] = (double)y;
        for (int k = 1; k < m; k++) {
            y = (PT)r[s0 + k] - lf[s0 + k] * y;
            z[s0 + k] = (double)y;
        }
        PT zn = (PT)z[s0 + m - 1] * ip[s0 + m - 1];
        z[s0 + m - 1] = (double)zn;
        for (int k = m - 2; k >= 0; k--) {
            zn = (PT)z[s0 + k] * ip[s0 + k] - lf[s0 + k + 1] * zn;
            z[s0 + k] = (double)zn;
        }
    }
}

// FP64 residual r = b - A x, returns this thread's share of |r|^2.
template <int T>
__device__ __forceinline__ double true_residual(const BatchSys& S, double* r) {
    double tl = 0;
    for (int i = threadIdx.x; i < S.n; i += T) {
        double s = 0;
        for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) s += S.val[kk] * S.x[S.ci[kk]];
        const double ri = S.b[i] - s;
        r[i] = ri;
        tl += ri * ri;
    }
    return tl;
}

// PK: CICY_PRECOND_JACOBI (0), CICY_PRECOND_LEARNED (1), CICY_PRECOND_CHAIN (2).
template <int T, int PK, bool MX>
__global__ void __launch_bounds__(T) k_batch_pcg(BatchArgs a) {
    using PT = typename std::conditional<MX, float, double>::type;
    __shared__ double sm[80];
    __shared__ int s_q;
    while (true) {
        if (threadIdx.x == 0) s_q = a.first + atomicAdd(a.queue, 1);
        __syncthreads();
        const int q = s_q;
        __syncthreads();
        if (q >= a.count) return;
        const int id = a.order[q];
        const BatchSys S = a.sys[id];
        const int n = S.n;
        double* r = a.scratch + S.off;
        double* p = r + n;
        double* qv = p + n;
        double* z = qv + n;
        double* y = z + n;
        double* u = y + n;
        PT* lf = reinterpret_cast<PT*>(u + n);
        PT* ip = lf + n;
        float* g32 = reinterpret_cast<float*>(u + 3 * (long long)n);
        float* rs32 = g32 + S.nnz;
        // ---- setup: preconditioner factors, FP32 conductances and row sums
        if (PK == 0) {
            for (int i = threadIdx.x; i < n; i += T) ip[i] = (PT)(1.0 / diag_of(S, i));
        } else {
            factor_chains<PT, PK == 1 ? kSpaiBlock : 0>(S, lf, ip);
        }
        if (MX) {
            for (int i = threadIdx.x; i < n; i += T) {
                double rs = 0;
                for (int k = S.rp[i]; k < S.rp[i + 1]; k++) {
                    rs += S.val[k];
                    g32[k] = S.ci[k] == i ? 0.0f : (float)(-S.val[k]);
                }
                rs32[i] = (float)rs;
            }
        }
        // r = b - A x0, x = x0
        double rr_l = 0, bb_l = 0;
        for (int i = threadIdx.x; i < n; i += T) {
            double s = 0;
            for (int k = S.rp[i]; k < S.rp[i + 1]; k++) s += S.val[k] * S.x0[S.ci[k]];
            const double ri = S.b[i] - s;
            r[i] = ri;
            S.x[i] = S.x0[i];
            rr_l += ri * ri;
            bb_l += S.b[i] * S.b[i];
        }
        double rr, bb;
        cta_sum2<T>(rr_l, bb_l, sm, rr, bb);  // (its barriers also end the setup)
        const double R0 = a.tol * sqrt(fmin(rr, bb));  // |r| <= tol |r0| and |b - A x| <= tol |b|
        double anchor = sqrt(rr);
        const long long max_iter = a.iter_factor * (long long)n;
        long long k = 0;
        int restarts = 0, flag = 0;
        bool fresh = true;
        double rz = 0;
        while (true) {
            // ---- z = M^-1 r
            if (PK == 0) {
                for (int i = threadIdx.x; i < n; i += T) z[i] = (double)((PT)r[i] * ip[i]);
            } else if (PK == 2) {
                apply_chains<PT>(S, lf, ip, r, z);
            } else {
                apply_chains<PT>(S, lf, ip, r, y);
                __syncthreads();
                for (int i = threadIdx.x; i < n; i += T) {
                    if (MX) {
                        float s = 0;
                        for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) {
                            const float w = S.ew[kk];
                            if (w != 0.0f) s += w * g32[kk] * (float)y[S.ci[kk]];
                        }
                        u[i] = (double)s;
                    } else {
                        double s = 0;
                        for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) {
                            const float w = S.ew[kk];
                            if (w != 0.0f) s += (double)w * (-S.val[kk]) * y[S.ci[kk]];
                        }
                        u[i] = s;
                    }
                }
                __syncthreads();
                apply_chains<PT>(S, lf, ip, u, z);
                __syncthreads();
                for (int i = threadIdx.x; i < n; i += T) z[i] += y[i];
            }
            __syncthreads();
            double rz_l = 0;
            for (int i = threadIdx.x; i < n; i += T) rz_l += r[i] * z[i];
            const double rz_new = cta_sum<T>(rz_l, sm);
            const double beta = fresh ? 0.0 : rz_new / rz;
            rz = rz_new;
            for (int i = threadIdx.x; i < n; i += T) p[i] = z[i] + beta * (fresh ? 0.0 : p[i]);
            __syncthreads();
            // ---- q = A p
            double pq_l = 0;
            for (int i = threadIdx.x; i < n; i += T) {
                double s;
                if (MX) {
                    const double pi = p[i];
                    float f = rs32[i] * (float)pi;
                    for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) f += g32[kk] * (float)(pi - p[S.ci[kk]]);
                    s = (double)f;
                } else {
                    s = 0;
                    for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) s += S.val[kk] * p[S.ci[kk]];
                }
                qv[i] = s;
                pq_l += p[i] * s;
            }
            const double pq = cta_sum<T>(pq_l, sm);
            if (!(pq > 0) || !(rz > 0)) break;  // breakdown (p.Ap <= 0 from rounding): stop with x intact, flag 0
            fresh = false;
            k++;
            const double alpha = rz / pq;
            rr_l = 0;
            for (int i = threadIdx.x; i < n; i += T) {
                S.x[i] += alpha * p[i];
                const double ri = r[i] - alpha * qv[i];
                r[i] = ri;
                rr_l += ri * ri;
            }
            rr = cta_sum<T>(rr_l, sm);
            if (!(rr == rr)) break;
            const double rn = sqrt(rr);
            if (rn <= R0) {
                if (restarts >= (MX ? kBatchReplacements : kBatchRestarts)) break;
                rr = cta_sum<T>(true_residual<T>(S, r), sm);
                restarts++;
                if (sqrt(rr) <= R0) { flag = 1; break; }
                anchor = sqrt(rr);
                fresh = !MX;  // FP64: restart; mixed: residual replacement, directions kept
            } else if (MX && rn <= kReplaceDrop * anchor && restarts < kBatchReplacements) {
                rr = cta_sum<T>(true_residual<T>(S, r), sm);
                restarts++;
                anchor = sqrt(rr);
            }
            if (k >= max_iter) { flag = 2; break; }
        }
        // FP64 relative residual |b - A x| / |b|
        bb_l = 0;
        double tr_l = 0;
        for (int i = threadIdx.x; i < n; i += T) {
            double s = 0;
            for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) s += S.val[kk] * S.x[S.ci[kk]];
            const double ri = S.b[i] - s;
            tr_l += ri * ri;
            bb_l += S.b[i] * S.b[i];
        }
        double trr, bbb;
        cta_sum2<T>(tr_l, bb_l, sm, trr, bbb);
        if (threadIdx.x == 0) {
            a.iterations[id] = k;
            a.rel[id] = bbb > 0 ? sqrt(trr / bbb) : 0.0;
            a.flags[id] = flag;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// One 16-CTA cluster per system (large systems: one SM's L2 latency and
// bandwidth bound the one-CTA solve).  Each CTA owns the chains whose first row
// lies in its 1/16 of the rows, so the chain factors and sweeps stay CTA-local;
// SpMV and the learned coupling term read other CTAs' rows from global memory
// after a hardware cluster barrier (release/acquire).  Reductions: each CTA
// writes its partial to a bank of `part`, a cluster barrier, then every CTA sums
// the 16 partials in rank order (identical results, so every CTA takes the same
// branches).  One bank per reduction kind, so a bank is rewritten only after a
// later barrier.  Barriers per iteration: 3 (4 with the learned term).
constexpr int kClCtas = 16;
constexpr int kClThreads = 512;

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// First chain whose start row is >= row (chain starts ascend).
__device__ __forceinline__ int chain_at(const BatchSys& S, long long row) {
    int lo = 0, hi = S.nchains;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (S.cs[mid] < row) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Cluster-wide sum of (a, b): this CTA's partial into bank `bank`, barrier, sum of the 16.
__device__ __forceinline__ void cl_sum2(double a, double b, double* sm, double* part, int bank, int rank, double& ra, double& rb) {
    double pa, pb;
    cta_sum2<kClThreads>(a, b, sm, pa, pb);
    double* slot = part + (size_t)bank * kClCtas * 2;
    if (threadIdx.x == 0) {
        slot[2 * rank] = pa;
        slot[2 * rank + 1] = pb;
    }
    cluster_sync();
    ra = 0;
    rb = 0;
    for (int r = 0; r < kClCtas; r++) {
        ra += __ldcg(&slot[2 * r]);
        rb += __ldcg(&slot[2 * r + 1]);
    }
}

// z = T^-1 r over this CTA's chains (see apply_chains).
template <typename PT>
__device__ void apply_chains_range(const BatchSys& S, int c_lo, int c_hi, const PT* lf, const PT* ip, const double* r, double* z) {
    for (int c = c_lo + threadIdx.x; c < c_hi; c += blockDim.x) {
        const int s0 = S.cs[c], m = S.cl[c];
        PT y = (PT)r[s0];
        z[s0] = (double)y;
        for (int k = 1; k < m; k++) {
            y = (PT)r[s0 + k] - lf[s0 + k] * y;
            z[s0 + k] = (double)y;
        }
        PT zn = (PT)z[s0 + m - 1] * ip[s0 + m - 1];
        z[s0 + m - 1] = (double)zn;
        for (int k = m - 2; k >= 0; k--) {
            zn = (PT)z[s0 + k] * ip[s0 + k] - lf[s0 + k + 1] * zn;
            z[s0 + k] = (double)zn;
        }
    }
}

template <typename PT, int BLK>
__device__ void factor_chains_range(const BatchSys& S, int c_lo, int c_hi, PT* lf, PT* ip) {
    for (int c = c_lo + threadIdx.x; c < c_hi; c += blockDim.x) {
        const int s0 = S.cs[c], m = S.cl[c];
        const int bl = BLK > 0 ? BLK : m;
        for (int b0 = 0; b0 < m; b0 += bl) {
            const int bm = min(bl, m - b0);
            bool singular = false;
            double piv_prev = 0, e_prev = 0;
            for (int k = 0; k < bm; k++) {
                const int i = s0 + b0 + k;
                const double d = diag_of(S, i);
                double l = 0, piv = d;
                if (k > 0) {
                    l = e_prev / piv_prev;
                    piv = d - l * e_prev;
                }
                singular |= !(piv > 1e-13 * fabs(d));
                lf[i] = (PT)l;
                ip[i] = (PT)(1.0 / piv);
                piv_prev = piv;
                e_prev = (k + 1 < bm) ? upper(S, i) : 0.0;
            }
            if (singular)
                for (int k = 0; k < bm; k++) {
                    const int i = s0 + b0 + k;
                    lf[i] = (PT)0;
                    ip[i] = (PT)(1.0 / diag_of(S, i));
                }
        }
    }
}

template <int PK, bool MX>
__global__ void __launch_bounds__(kClThreads) k_batch_pcg_cl(BatchArgs a) {
    using PT = typename std::conditional<MX, float, double>::type;
    constexpr int T = kClThreads;
    __shared__ double sm[80];
    const int cl = blockIdx.x / kClCtas, rank = blockIdx.x % kClCtas;
    double* part = a.part + (size_t)cl * 5 * kClCtas * 2;
    while (true) {
        if (rank == 0 && threadIdx.x == 0) a.slots[cl] = a.first + atomicAdd(a.queue, 1);
        cluster_sync();
        const int q = __ldcg(&a.slots[cl]);
        cluster_sync();
        if (q >= a.count) return;
        const int id = a.order[q];
        const BatchSys S = a.sys[id];
        const int n = S.n;
        const int c_lo = chain_at(S, (long long)rank * n / kClCtas);
        const int c_hi = rank == kClCtas - 1 ? S.nchains : chain_at(S, (long long)(rank + 1) * n / kClCtas);
        const int r_lo = c_lo < S.nchains ? S.cs[c_lo] : n, r_hi = c_hi < S.nchains ? S.cs[c_hi] : n;
        double* r = a.scratch + S.off;
        double* p = r + n;
        double* qv = p + n;
        double* z = qv + n;
        double* y = z + n;
        double* u = y + n;
        PT* lf = reinterpret_cast<PT*>(u + n);
        PT* ip = lf + n;
        float* g32 = reinterpret_cast<float*>(u + 3 * (long long)n);
        float* rs32 = g32 + S.nnz;
        if (PK == 0) {
            for (int i = r_lo + threadIdx.x; i < r_hi; i += T) ip[i] = (PT)(1.0 / diag_of(S, i));
        } else {
            factor_chains_range<PT, PK == 1 ? kSpaiBlock : 0>(S, c_lo, c_hi, lf, ip);
        }
        if (MX) {
            for (int i = r_lo + threadIdx.x; i < r_hi; i += T) {
                double rs = 0;
                for (int k = S.rp[i]; k < S.rp[i + 1]; k++) {
                    rs += S.val[k];
                    g32[k] = S.ci[k] == i ? 0.0f : (float)(-S.val[k]);
                }
                rs32[i] = (float)rs;
            }
        }
        double rr_l = 0, bb_l = 0;
        for (int i = r_lo + threadIdx.x; i < r_hi; i += T) {
            double sacc = 0;
            for (int k = S.rp[i]; k < S.rp[i + 1]; k++) sacc += S.val[k] * S.x0[S.ci[k]];
            const double ri = S.b[i] - sacc;
            r[i] = ri;
            S.x[i] = S.x0[i];
            rr_l += ri * ri;
            bb_l += S.b[i] * S.b[i];
        }
        double rr, bb;
        cl_sum2(rr_l, bb_l, sm, part, 0, rank, rr, bb);
        const double R0 = a.tol * sqrt(fmin(rr, bb));
        double anchor = sqrt(rr);
        const long long max_iter = a.iter_factor * (long long)n;
        long long k = 0;
        int restarts = 0, flag = 0;
        bool fresh = true;
        double rz = 0, dummy;
        while (true) {
            // ---- z = M^-1 r (own rows)
            if (PK == 0) {
                for (int i = r_lo + threadIdx.x; i < r_hi; i += T) z[i] = (double)((PT)r[i] * ip[i]);
            } else if (PK == 2) {
                apply_chains_range<PT>(S, c_lo, c_hi, lf, ip, r, z);
            } else {
                apply_chains_range<PT>(S, c_lo, c_hi, lf, ip, r, y);
                cluster_sync();  // the coupling term reads y of other CTAs' rows
                for (int i = r_lo + threadIdx.x; i < r_hi; i += T) {
                    if (MX) {
                        float f = 0;
                        for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) {
                            const float w = S.ew[kk];
                            if (w != 0.0f) f += w * g32[kk] * (float)__ldcg(&y[S.ci[kk]]);
                        }
                        u[i] = (double)f;
                    } else {
                        double sacc = 0;
                        for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) {
                            const float w = S.ew[kk];
                            if (w != 0.0f) sacc += (double)w * (-S.val[kk]) * __ldcg(&y[S.ci[kk]]);
                        }
                        u[i] = sacc;
                    }
                }
                __syncthreads();
                apply_chains_range<PT>(S, c_lo, c_hi, lf, ip, u, z);
                __syncthreads();
                for (int i = r_lo + threadIdx.x; i < r_hi; i += T) z[i] += y[i];
            }
            __syncthreads();
            double rz_l = 0;
            for (int i = r_lo + threadIdx.x; i < r_hi; i += T) rz_l += r[i] * z[i];
            double rz_new;
            cl_sum2(rz_l, 0.0, sm, part, 1, rank, rz_new, dummy);
            const double beta = fresh ? 0.0 : rz_new / rz;
            rz = rz_new;
            for (int i = r_lo + threadIdx.x; i < r_hi; i += T) p[i] = z[i] + beta * (fresh ? 0.0 : p[i]);
            cluster_sync();  // q = A p reads p of other CTAs' rows
            // ---- q = A p (own rows)
            double pq_l = 0;
            for (int i = r_lo + threadIdx.x; i < r_hi; i += T) {
                double sq;
                if (MX) {
                    const double pi = p[i];
                    float f = rs32[i] * (float)pi;
                    for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) f += g32[kk] * (float)(pi - __ldcg(&p[S.ci[kk]]));
                    sq = (double)f;
                } else {
                    sq = 0;
                    for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) sq += S.val[kk] * __ldcg(&p[S.ci[kk]]);
                }
                qv[i] = sq;
                pq_l += p[i] * sq;
            }
            double pq;
            cl_sum2(pq_l, 0.0, sm, part, 2, rank, pq, dummy);
            if (!(pq > 0) || !(rz > 0)) break;  // breakdown: stop with x intact, flag 0
            fresh = false;
            k++;
            const double alpha = rz / pq;
            rr_l = 0;
            for (int i = r_lo + threadIdx.x; i < r_hi; i += T) {
                S.x[i] += alpha * p[i];
                const double ri = r[i] - alpha * qv[i];
                r[i] = ri;
                rr_l += ri * ri;
            }
            cl_sum2(rr_l, 0.0, sm, part, 3, rank, rr, dummy);  // (also makes x complete for a true residual)
            if (!(rr == rr)) break;
            const double rn = sqrt(rr);
            const bool conv = rn <= R0;
            const bool repl = !conv && MX && rn <= kReplaceDrop * anchor && restarts < kBatchReplacements;
            if (conv || repl) {
                if (conv && restarts >= (MX ? kBatchReplacements : kBatchRestarts)) break;
                double tl = 0;
                for (int i = r_lo + threadIdx.x; i < r_hi; i += T) {
                    double sacc = 0;
                    for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) sacc += S.val[kk] * __ldcg(&S.x[S.ci[kk]]);
                    const double ri = S.b[i] - sacc;
                    r[i] = ri;
                    tl += ri * ri;
                }
                cl_sum2(tl, 0.0, sm, part, 4, rank, rr, dummy);
                restarts++;
                if (conv && sqrt(rr) <= R0) { flag = 1; break; }
                anchor = sqrt(rr);
                if (conv) fresh = !MX;  // FP64: restart; mixed: residual replacement, directions kept
            }
            if (k >= max_iter) { flag = 2; break; }
        }
        // FP64 relative residual |b - A x| / |b| (x of all rows complete after a barrier)
        cluster_sync();
        bb_l = 0;
        double tr_l = 0;
        for (int i = r_lo + threadIdx.x; i < r_hi; i += T) {
            double sacc = 0;
            for (int kk = S.rp[i]; kk < S.rp[i + 1]; kk++) sacc += S.val[kk] * __ldcg(&S.x[S.ci[kk]]);
            const double ri = S.b[i] - sacc;
            tr_l += ri * ri;
            bb_l += S.b[i] * S.b[i];
        }
        double trr, bbb;
        cl_sum2(tr_l, bb_l, sm, part, 0, rank, trr, bbb);
        if (rank == 0 && threadIdx.x == 0) {
            a.iterations[id] = k;
            a.rel[id] = bbb > 0 ? sqrt(trr / bbb) : 0.0;
            a.flags[id] = flag;
        }
    }
}

// Structure check of every system (one CTA per system), before any solve reads it.
__global__ void __launch_bounds__(256) k_batch_check(const BatchSys* __restrict__ sys, int count, int* __restrict__ bad) {
    for (int id = blockIdx.x; id < count; id += gridDim.x) {
        const BatchSys S = sys[id];
        const int f = check_structure_part(threadIdx.x, blockDim.x, S.n, S.nnz, S.rp, S.ci, S.nchains, S.cs, S.cl);
        if (f) atomicOr(&bad[id], f);
    }
}

// FP64 |b - A x| / |b| of every system (one CTA per system).
__global__ void __launch_bounds__(256) k_batch_residual(const BatchSys* __restrict__ sys, int count, double* __restrict__ rel) {
    __shared__ double sm[80];
    for (int id = blockIdx.x; id < count; id += gridDim.x) {
        const BatchSys S = sys[id];
        double a = 0, b = 0;
        for (int i = threadIdx.x; i < S.n; i += 256) {
            double s = 0;
            for (int k = S.rp[i]; k < S.rp[i + 1]; k++) s += S.val[k] * S.x[S.ci[k]];
            const double ri = S.b[i] - s;
            a += ri * ri;
            b += S.b[i] * S.b[i];
        }
        double ta, tb;
        cta_sum2<256>(a, b, sm, ta, tb);
        if (threadIdx.x == 0) rel[id] = tb > 0 ? sqrt(ta / tb) : 0.0;
    }
}

template <int T>
void launch(const BatchArgs& a, int grid, int pk, bool mx, cudaStream_t s) {
    if (pk == 0) mx ? k_batch_pcg<T, 0, true><<<grid, T, 0, s>>>(a) : k_batch_pcg<T, 0, false><<<grid, T, 0, s>>>(a);
    else if (pk == 1) mx ? k_batch_pcg<T, 1, true><<<grid, T, 0, s>>>(a) : k_batch_pcg<T, 1, false><<<grid, T, 0, s>>>(a);
    else mx ? k_batch_pcg<T, 2, true><<<grid, T, 0, s>>>(a) : k_batch_pcg<T, 2, false><<<grid, T, 0, s>>>(a);
}

template <int PK, bool MX>
void* cl_kernel() {
    return (void*)k_batch_pcg_cl<PK, MX>;
}

void* cl_kernel_for(int pk, bool mx) {
    if (pk == 0) return mx ? cl_kernel<0, true>() : cl_kernel<0, false>();
    if (pk == 1) return mx ? cl_kernel<1, true>() : cl_kernel<1, false>();
    return mx ? cl_kernel<2, true>() : cl_kernel<2, false>();
}

// 16-CTA clusters are a non-portable size: opt every instantiation in once.
// Returns the number of clusters of one instantiation that fit at once (0: none).
int cl_setup(int sms) {
    static int clusters = -1;
    if (clusters >= 0) return clusters;
    clusters = 0;
    bool ok = true;
    for (int pk = 0; pk < 3; pk++)
        for (int mx = 0; mx < 2; mx++)
            ok &= cudaFuncSetAttribute(cl_kernel_for(pk, mx != 0), cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
    cudaGetLastError();
    if (!ok) return clusters;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(kClCtas);
    cfg.blockDim = dim3(kClThreads);
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int mn = 1 << 30;
    for (int pk = 0; pk < 3; pk++)
        for (int mx = 0; mx < 2; mx++) {
            int n = 0;
            if (cudaOccupancyMaxActiveClusters(&n, cl_kernel_for(pk, mx != 0), &cfg) != cudaSuccess) n = 0;
            mn = std::min(mn, n);
        }
    cudaGetLastError();
    clusters = std::max(0, std::min(mn, sms / kClCtas));
    return clusters;
}

void launch_cl(const BatchArgs& a, int nclusters, int pk, bool mx, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(kClCtas * nclusters);
    cfg.blockDim = dim3(kClThreads);
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    BatchArgs args = a;
    void* params[] = {&args};
    CICY_CUDA(cudaLaunchKernelExC(&cfg, cl_kernel_for(pk, mx), params));
}

__global__ void k_diag_extract(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                               double* __restrict__ d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double x = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++)
            if (ci[k] == i) x = v[k];
        d[i] = x;
    }
}

}  // namespace
}  // namespace cicy

// ---------------------------------------------------------------------------
struct cicy_batch {
    int device = 0;
    int count = 0;
    int precision = 0;
    int precond = CICY_PRECOND_CHAIN;  // methods 0 and 2
    double tol = 1e-8;
    long long iter_factor = 300;
    int threads = 512, ctas_per_sm = 2, sms = 148;
    int method = 0;  // 0: one CTA per system, 1: one 16-CTA cluster per system (multigrid), 2: one system at a time, grid-wide
    int split = 0;   // method 0: systems of at least this many rows run on 16-CTA clusters (0: none)
    int n_split = 0; // how many systems that is (the first ones of the largest-first order)
    int nclusters = 0;
    bool have_weights = false;
    cicy::MgBatch* mg = nullptr;
    int64_t launches = 0;
    std::vector<cicy_batch_system> inputs;
    cicy::DBuf<cicy::BatchSys> sys;
    cicy::DBuf<int> order, queue, flags, status, queue2, slots;
    cicy::DBuf<double> part;
    cicy::DBuf<double> scratch, rel, diag;
    cicy::DBuf<long long> iterations;
    std::vector<long long> diag_off, seq_iterations;
    cicy::SolverWork* sw = nullptr;  // method 2
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_threads = 0, graph_ctas = 0, graph_method = -1, graph_precond = -1, graph_precision = -1, graph_split = -1;
    cudaStream_t stream = nullptr, stream2 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    ~cicy_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
        if (stream2) cudaStreamDestroy(stream2);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (mg) cicy::mg_batch_free(mg);
        delete sw;
        sys.release(); order.release(); queue.release(); flags.release(); status.release(); scratch.release(); rel.release();
        diag.release(); iterations.release(); queue2.release(); slots.release(); part.release();
    }
};

namespace {

template <class F>
cicy_status batch_guard(int device, F&& f) {
    try {
        CICY_CUDA(cudaSetDevice(device));
        f();
        return CICY_OK;
    } catch (const cicy::Fail& e) {
        cicy::set_host_error(e.msg);
        return e.status;
    }
}

void enqueue(cicy_batch* B, cudaStream_t s) {
    if (B->method == 1) {
        cicy::mg_batch_enqueue(B->mg, s);
        cicy::k_batch_residual<<<std::min(B->count, B->sms * 4), 256, 0, s>>>(B->sys.get(), B->count, B->rel.get());
        CICY_LAUNCH_CHECK();
        return;
    }
    cicy::BatchArgs a{};
    a.sys = B->sys.get();
    a.order = B->order.get();
    a.count = B->count;
    a.first = 0;
    a.queue = B->queue.get();
    a.scratch = B->scratch.get();
    a.tol = B->tol;
    a.iter_factor = B->iter_factor;
    a.iterations = B->iterations.get();
    a.rel = B->rel.get();
    a.flags = B->flags.get();
    const bool mx = B->precision == CICY_PRECISION_MIXED;
    const int K = B->split > 0 ? B->n_split : 0;
    if (K > 0) {  // the largest systems on 16-CTA clusters, concurrently with the rest (fork/join)
        CICY_CUDA(cudaEventRecord(B->fork, s));
        CICY_CUDA(cudaStreamWaitEvent(B->stream2, B->fork, 0));
        cicy::BatchArgs c = a;
        c.first = 0;
        c.count = K;
        c.queue = B->queue2.get();
        c.slots = B->slots.get();
        c.part = B->part.get();
        CICY_CUDA(cudaMemsetAsync(B->queue2.get(), 0, sizeof(int), B->stream2));
        // with one-CTA solves running beside them, at most 8 clusters (neither kernel waits on the other:
        // a cluster not yet resident only starts later)
        const int ncl = std::min({B->nclusters, K, K < B->count ? 8 : B->nclusters});
        cicy::launch_cl(c, ncl, B->precond, mx, B->stream2);
        CICY_LAUNCH_CHECK();
        CICY_CUDA(cudaEventRecord(B->join, B->stream2));
    }
    if (K < B->count) {
        a.first = K;
        CICY_CUDA(cudaMemsetAsync(B->queue.get(), 0, sizeof(int), s));
        const int grid = std::max(1, std::min(B->count - K, B->sms * B->ctas_per_sm));
        switch (B->threads) {
            case 256: cicy::launch<256>(a, grid, B->precond, mx, s); break;
            case 512: cicy::launch<512>(a, grid, B->precond, mx, s); break;
            default: cicy::launch<1024>(a, grid, B->precond, mx, s); break;
        }
        CICY_LAUNCH_CHECK();
    }
    if (K > 0) CICY_CUDA(cudaStreamWaitEvent(s, B->join, 0));
}

// Method 2: every system through the per-network grid-wide persistent PCG, one
// after another; returns the sum of the solves' kernel times.
double solve_sequential(cicy_batch* B) {
    cudaStream_t s = B->stream;
    if (!B->sw) B->sw = new cicy::SolverWork;
    if (B->diag_off.empty()) {
        long long tot = 0;
        B->diag_off.resize(B->count);
        for (int i = 0; i < B->count; i++) {
            B->diag_off[i] = tot;
            tot += B->inputs[i].n;
        }
        B->diag.ensure((size_t)std::max(tot, 1LL));
        for (int i = 0; i < B->count; i++) {
            const cicy_batch_system& in = B->inputs[i];
            cicy::k_diag_extract<<<std::min((in.n + 255) / 256, B->sms * 8), 256, 0, s>>>(in.n, in.row_ptr, in.col_ind, in.values,
                                                                                     B->diag.get() + B->diag_off[i]);
            CICY_LAUNCH_CHECK();
        }
        B->status.ensure(1);
    }
    const bool mx = B->precision == CICY_PRECISION_MIXED;
    const int kind = B->precond == CICY_PRECOND_JACOBI ? cicy::PRECOND_KIND_JACOBI
                     : B->precond == CICY_PRECOND_LEARNED ? cicy::PRECOND_KIND_SPAI
                                                          : cicy::PRECOND_KIND_BLOCK;
    CICY_CUDA(cudaMemsetAsync(B->status.get(), 0, sizeof(int), s));
    B->seq_iterations.assign(B->count, 0);
    std::vector<int> fl(B->count, 0);
    double total = 0;
    for (int i = 0; i < B->count; i++) {
        const cicy_batch_system& in = B->inputs[i];
        cicy::SolverSystem ss;
        ss.n = in.n;
        ss.nnz = in.nnz;
        ss.rp = in.row_ptr;
        ss.ci = in.col_ind;
        ss.val = in.values;
        ss.diag = B->diag.get() + B->diag_off[i];
        ss.b = in.b;
        ss.x = in.x;
        CICY_CUDA(cudaMemcpyAsync(in.x, in.x0, sizeof(double) * in.n, cudaMemcpyDeviceToDevice, s));
        if (kind != cicy::PRECOND_KIND_JACOBI)
            cicy::build_block_preconditioner(*B->sw, ss, in.n_chains, in.chain_start, in.chain_len, nullptr, nullptr, mx, s, B->launches);
        cicy::PcgStats st;
        const long long max_iter = B->iter_factor * (long long)in.n;
        cicy::pcg_solve(*B->sw, ss, kind, mx, B->tol, max_iter, B->sms, B->status.get(), s, B->launches, st, in.edge_weights);
        total += st.seconds;
        B->seq_iterations[i] = st.iterations;
        fl[i] = st.iterations < max_iter ? 1 : 2;
    }
    int err = 0;
    CICY_CUDA(cudaMemcpyAsync(&err, B->status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaMemcpyAsync(B->flags.get(), fl.data(), sizeof(int) * B->count, cudaMemcpyHostToDevice, s));
    cicy::k_batch_residual<<<std::min(B->count, B->sms * 4), 256, 0, s>>>(B->sys.get(), B->count, B->rel.get());
    CICY_LAUNCH_CHECK();
    CICY_CUDA(cudaStreamSynchronize(s));
    if (err) throw cicy::Fail{CICY_E_TIMEOUT, "cicy_batch method 2: a grid barrier timed out"};
    return total;
}

// (Re)build the graph of one batch solve for the current launch shape.
void ensure_graph(cicy_batch* B) {
    if (B->exec && B->graph_threads == B->threads && B->graph_ctas == B->ctas_per_sm && B->graph_method == B->method &&
        B->graph_precond == B->precond && B->graph_precision == B->precision && B->graph_split == B->split)
        return;
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    B->exec = nullptr;
    B->graph = nullptr;
    CICY_CUDA(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
    try {
        enqueue(B, B->stream);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(B->stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    CICY_CUDA(cudaStreamEndCapture(B->stream, &B->graph));
    CICY_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
    B->graph_threads = B->threads;
    B->graph_ctas = B->ctas_per_sm;
    B->graph_method = B->method;
    B->graph_precond = B->precond;
    B->graph_precision = B->precision;
    B->graph_split = B->split;
}

double timed_solve(cicy_batch* B) {
    if (B->method == 2) return solve_sequential(B);
    ensure_graph(B);
    cudaEvent_t e0, e1;
    CICY_CUDA(cudaEventCreate(&e0));
    CICY_CUDA(cudaEventCreate(&e1));
    CICY_CUDA(cudaEventRecord(e0, B->stream));
    CICY_CUDA(cudaGraphLaunch(B->exec, B->stream));
    CICY_CUDA(cudaEventRecord(e1, B->stream));
    CICY_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms * 1e-3;
}

}  // namespace

extern "C" {

cicy_status cicy_batch_create(cicy_batch** out, int device, const cicy_batch_system* systems, int32_t count, double tol,
                              int32_t max_iter_factor, int32_t precision) {
    if (!out || !systems || count <= 0 || !(tol > 0) || max_iter_factor <= 0 || precision < 0 || precision > 1) {
        cicy::set_host_error("cicy_batch_create: invalid arguments");
        return CICY_E_INPUT;
    }
    *out = nullptr;
    bool weights = true;
    for (int i = 0; i < count; i++) {
        const cicy_batch_system& s = systems[i];
        if (s.n <= 0 || s.nnz <= 0 || !s.row_ptr || !s.col_ind || !s.values || !s.b || !s.x0 || !s.x || s.n_chains <= 0 ||
            !s.chain_start || !s.chain_len) {
            cicy::set_host_error("cicy_batch_create: system " + std::to_string(i) + " is incomplete");
            return CICY_E_INPUT;
        }
        weights &= s.edge_weights != nullptr;
    }
    cicy_batch* B = new cicy_batch;
    cicy_status st = batch_guard(device, [&] {
        B->device = device;
        B->count = count;
        B->inputs.assign(systems, systems + count);
        B->precision = precision;
        B->tol = tol;
        B->iter_factor = max_iter_factor;
        CICY_CUDA(cudaDeviceGetAttribute(&B->sms, cudaDevAttrMultiProcessorCount, device));
        CICY_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
        CICY_CUDA(cudaStreamCreateWithFlags(&B->stream2, cudaStreamNonBlocking));
        CICY_CUDA(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming));
        CICY_CUDA(cudaEventCreateWithFlags(&B->join, cudaEventDisableTiming));
        B->have_weights = weights;
        std::vector<cicy::BatchSys> h(count);
        long long off = 0;
        for (int i = 0; i < count; i++) {
            const cicy_batch_system& s = systems[i];
            h[i] = cicy::BatchSys{s.n, s.nnz, s.n_chains, s.row_ptr, s.col_ind, s.values, s.b, s.x0, s.x, s.chain_start, s.chain_len,
                                  s.edge_weights, off};
            off += cicy::batch_scratch(s.n, s.nnz);
        }
        std::vector<int> ord(count);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return systems[a].n > systems[b].n; });
        B->sys.ensure(count);
        B->order.ensure(count);
        B->queue.ensure(1);
        B->flags.ensure(count);
        B->rel.ensure(count);
        B->iterations.ensure(count);
        B->scratch.ensure((size_t)off + 2);
        CICY_CUDA(cudaMemcpyAsync(B->sys.get(), h.data(), sizeof(cicy::BatchSys) * count, cudaMemcpyHostToDevice, B->stream));
        CICY_CUDA(cudaMemcpyAsync(B->order.get(), ord.data(), sizeof(int) * count, cudaMemcpyHostToDevice, B->stream));
        // the solves trust the CSR and the chain partition: check them once here
        CICY_CUDA(cudaMemsetAsync(B->flags.get(), 0, sizeof(int) * count, B->stream));
        cicy::k_batch_check<<<std::min(count, B->sms * 4), 256, 0, B->stream>>>(B->sys.get(), count, B->flags.get());
        CICY_LAUNCH_CHECK();
        std::vector<int> bad(count);
        CICY_CUDA(cudaMemcpyAsync(bad.data(), B->flags.get(), sizeof(int) * count, cudaMemcpyDeviceToHost, B->stream));
        CICY_CUDA(cudaStreamSynchronize(B->stream));
        for (int i = 0; i < count; i++)
            if (bad[i])
                throw cicy::Fail{CICY_E_INPUT, "cicy_batch_create: system " + std::to_string(i) + ": " + cicy::structure_error(bad[i])};
        CICY_CUDA(cudaStreamSynchronize(B->stream));
    });
    if (st != CICY_OK) {
        delete B;
        return st;
    }
    *out = B;
    return CICY_OK;
}

cicy_status cicy_batch_destroy(cicy_batch* b) {
    if (b) {
        cudaSetDevice(b->device);
        delete b;
    }
    return CICY_OK;
}

cicy_status cicy_batch_set_shape(cicy_batch* b, int32_t threads, int32_t ctas_per_sm) {
    if (!b || (threads != 256 && threads != 512 && threads != 1024) || ctas_per_sm < 1 || ctas_per_sm > 8 ||
        threads * ctas_per_sm > 2048) {
        cicy::set_host_error("cicy_batch_set_shape: threads must be 256, 512 or 1024 and threads x CTAs per SM at most 2048");
        return CICY_E_INPUT;
    }
    b->threads = threads;
    b->ctas_per_sm = ctas_per_sm;
    return CICY_OK;
}

cicy_status cicy_batch_set_solver(cicy_batch* b, int32_t preconditioner, int32_t precision) {
    if (!b || (preconditioner != CICY_PRECOND_JACOBI && preconditioner != CICY_PRECOND_LEARNED && preconditioner != CICY_PRECOND_CHAIN) ||
        (precision != CICY_PRECISION_FP64 && precision != CICY_PRECISION_MIXED)) {
        cicy::set_host_error("cicy_batch_set_solver: preconditioner Jacobi, learned or chain; precision FP64 or mixed");
        return CICY_E_INPUT;
    }
    if (preconditioner == CICY_PRECOND_LEARNED && !b->have_weights) {
        cicy::set_host_error("cicy_batch_set_solver: the learned preconditioner needs edge_weights in every system");
        return CICY_E_INPUT;
    }
    b->precond = preconditioner;
    b->precision = precision;
    return CICY_OK;
}

namespace {
void apply_split(cicy_batch* b, int rows) {
    b->split = rows;
    b->n_split = 0;
    if (rows <= 0) return;
    for (const auto& in : b->inputs) b->n_split += in.n >= rows ? 1 : 0;
    if (b->n_split == 0) return;
    b->nclusters = cicy::cl_setup(b->sms);
    if (b->nclusters < 1) throw cicy::Fail{CICY_E_DEVICE, "cicy_batch_set_split: 16-CTA clusters are not available"};
    b->queue2.ensure(1);
    b->slots.ensure(b->nclusters);
    b->part.ensure((size_t)b->nclusters * 5 * cicy::kClCtas * 2);
}
}  // namespace

cicy_status cicy_batch_set_split(cicy_batch* b, int32_t rows) {
    if (!b || rows < 0) {
        cicy::set_host_error("cicy_batch_set_split: rows >= 0");
        return CICY_E_INPUT;
    }
    return batch_guard(b->device, [&] { apply_split(b, rows); });
}

cicy_status cicy_batch_enable_multigrid(cicy_batch* b, double* setup_seconds) {
    if (!b) return CICY_E_INPUT;
    return batch_guard(b->device, [&] {
        if (b->mg) return;
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<cicy::MgBatchInput> in(b->count);
        for (int i = 0; i < b->count; i++) {
            const cicy_batch_system& s = b->inputs[i];
            in[i] = cicy::MgBatchInput{s.n, s.nnz, s.n_chains, s.row_ptr, s.col_ind, s.values, s.b, s.x0, s.x, s.chain_start, s.chain_len};
        }
        b->mg = cicy::mg_batch_build(in, b->tol, b->iter_factor, b->stream, b->launches);
        if (setup_seconds) *setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    });
}

cicy_status cicy_batch_set_method(cicy_batch* b, int32_t method) {
    if (!b || method < 0 || method > 2 || (method == 1 && !b->mg)) {
        cicy::set_host_error("cicy_batch_set_method: 0 (one CTA per system), 1 (multigrid, after cicy_batch_enable_multigrid) or 2 "
                             "(one system at a time, grid-wide)");
        return CICY_E_INPUT;
    }
    b->method = method;
    return CICY_OK;
}

cicy_status cicy_batch_autotune(cicy_batch* b, int32_t* method, int32_t* threads, int32_t* ctas_per_sm, int32_t* split_rows,
                                double* seconds) {
    if (!b) return CICY_E_INPUT;
    return batch_guard(b->device, [&] {
        static const int cand[][3] = {{0, 256, 4}, {0, 256, 8}, {0, 512, 2}, {0, 512, 4}, {0, 1024, 1}, {0, 1024, 2}, {1, 1024, 1}};
        double best = 1e300;
        int bm = b->method, bt = b->threads, bc = b->ctas_per_sm;
        apply_split(b, 0);  // launch shapes first, every system on one CTA
        for (const auto& c : cand) {
            if (c[0] == 1 && !b->mg) continue;
            b->method = c[0];
            b->threads = c[1];
            b->ctas_per_sm = c[2];
            const double t0 = timed_solve(b);  // warm (also builds the graph)
            if (t0 > 1.5 * best) continue;      // clearly slower: not timed again
            const double t = std::min(t0, timed_solve(b));
            if (t < best) {
                best = t;
                bm = c[0];
                bt = c[1];
                bc = c[2];
            }
        }
        b->method = bm;
        b->threads = bt;
        b->ctas_per_sm = bc;
        // method 0: the largest systems on 16-CTA clusters, at a few size thresholds
        int bs = 0;
        if (bm == 0 && cicy::cl_setup(b->sms) > 0) {
            for (int rows : {131072, 32768, 8192}) {
                apply_split(b, rows);
                if (b->n_split == 0) continue;
                const double t0 = timed_solve(b);
                if (t0 > 1.5 * best) continue;
                const double t = std::min(t0, timed_solve(b));
                if (t < best) {
                    best = t;
                    bs = rows;
                }
            }
        }
        apply_split(b, bs);
        if (split_rows) *split_rows = b->method == 0 ? b->split : 0;
        if (method) *method = bm;
        if (threads) *threads = bt;
        if (ctas_per_sm) *ctas_per_sm = bm == 1 ? cicy::mg_batch_clusters(b->mg) : bc;
        if (seconds) *seconds = best;
    });
}

cicy_status cicy_batch_solve(cicy_batch* b, double* seconds) {
    if (!b) return CICY_E_INPUT;
    return batch_guard(b->device, [&] {
        const double t = timed_solve(b);
        if (seconds) *seconds = t;
    });
}

cicy_status cicy_batch_results(cicy_batch* b, int64_t* iterations, double* rel_residual, int32_t* flags) {
    if (!b) return CICY_E_INPUT;
    return batch_guard(b->device, [&] {
        std::vector<long long> it(b->count);
        CICY_CUDA(cudaMemcpyAsync(it.data(), b->iterations.get(), sizeof(long long) * b->count, cudaMemcpyDeviceToHost, b->stream));
        if (rel_residual) CICY_CUDA(cudaMemcpyAsync(rel_residual, b->rel.get(), sizeof(double) * b->count, cudaMemcpyDeviceToHost, b->stream));
        if (flags) CICY_CUDA(cudaMemcpyAsync(flags, b->flags.get(), sizeof(int) * b->count, cudaMemcpyDeviceToHost, b->stream));
        CICY_CUDA(cudaStreamSynchronize(b->stream));
        if (b->method == 2 && (int)b->seq_iterations.size() == b->count) {
            for (int i = 0; i < b->count; i++) it[i] = b->seq_iterations[i];
        } else if (b->method == 1) {
            std::vector<double> st;
            cicy::mg_batch_stats(b->mg, st, b->stream);
            for (int i = 0; i < b->count; i++) {
                it[i] = (long long)st[4 * i];
                if (flags) flags[i] = std::sqrt(st[4 * i + 1]) <= st[4 * i + 2] ? 1 : (it[i] >= b->iter_factor * b->inputs[i].n ? 2 : 0);
            }
        }
        if (iterations)
            for (int i = 0; i < b->count; i++) iterations[i] = it[i];
    });
}

}  // extern "C"
