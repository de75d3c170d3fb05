// Learned preconditioner: a small graph network that weights the couplings a
// chain block-Jacobi leaves out, building the sparse approximate inverse
//
//     M^-1 = T^-1 + T^-1 E_w T^-1,   E_w[i][k] = w_ik |a_ik| for couplings outside T
//
// (T: the chain blocks; the second-order Neumann term of (T - E)^-1 with one
// learned weight 0 < w_ik < 1 per coupling; T + E_w stays diagonally dominant,
// so M is SPD).  The network (width 32, three message-passing layers):
//
//   node features  ((log d_i - mean) / std, log(1 + deg_i))
//   entry features lc = log|a_ik| - (log d_i + log d_k) / 2 (relative log
//                  conductance), jf = 1 for a tunnelling junction (not two
//                  consecutive nodes of one CNT chain)
//   layer 0        H = bf16(relu(f W_in + b_in))
//   layers 1..3    G = bf16(H U_l) and H W_l on the tensor cores (BF16 in, FP32
//                  accumulate); gate_ik = sigmoid(p0 lc + p1 jf + p2);
//                  M_i = (1/deg_i) sum_k gate_ik G_k; H = bf16(H + relu(H W_l + M + b_l))
//   edge output    w_ik = sigmoid(sum_j v_j H_ij H_kj + q0 lc_ik + q1)  (symmetric)
//
// Training (hand-written backward, FP32; the preconditioner part in FP64)
// minimises, over probe vectors u with r = A u and z = M^-1 r, the residual
// left by one optimally scaled preconditioned Richardson step,
// L = 1 - (r.Az)^2 / (|r|^2 |Az|^2).  Parameters are one flat FP32 vector in
// the order W_in, b_in, (U_l, W_l, b_l, p_l) for l = 0..2, v, q.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "cicy_internal.h"
#include "csr_check.cuh"
#include "ctx.cuh"
#include "solver.cuh"

namespace cicy {

namespace {

constexpr int kW = 32;                       // hidden width
constexpr int kLayers = 3;
constexpr int kLayerParams = 2 * kW * kW + kW + 3;
constexpr int kOffWin = 0, kOffBin = 2 * kW;
constexpr int kOffLayer0 = kOffBin + kW;
constexpr int kOffV = kOffLayer0 + kLayers * kLayerParams;
constexpr int kOffQ = kOffV + kW;
constexpr int kParams = kOffQ + 2;
constexpr int kOffU = 0, kOffW = kW * kW, kOffB = 2 * kW * kW, kOffP = 2 * kW * kW + kW;  // inside a layer

int grid_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148LL * 16) b = 148LL * 16;
    return (int)b;
}

int warps_grid(long long items, int threads = 256) {  // one warp per item, grid-stride
    return grid_for(items * 32, threads);
}

__device__ __forceinline__ float bfr(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float sigm(float x) { return 1.0f / (1.0f + expf(-x)); }
__device__ __forceinline__ float wsum(float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------------------
// Features
__global__ void k_diag_deg(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                           double* __restrict__ diag, double* __restrict__ logd, float* __restrict__ deg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0;
        int c = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            if (ci[k] == i) d = v[k];
            else c++;
        }
        diag[i] = d;
        logd[i] = log(d);
        deg[i] = (float)c;
    }
}

// mean and standard deviation of log d (one CTA, deterministic order)
__global__ void k_mean_std(int n, const double* __restrict__ x, double* __restrict__ out) {
    __shared__ double s1[32], s2[32];
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a += x[i];
        b += x[i] * x[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) { s1[threadIdx.x >> 5] = a; s2[threadIdx.x >> 5] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double A = 0, B = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { A += s1[w]; B += s2[w]; }
        const double mu = A / n;
        const double var = fmax(B / n - mu * mu, 0.0);
        out[0] = mu;
        out[1] = var > 0 ? sqrt(var) : 1.0;
    }
}

__global__ void k_node_feat(int n, const double* __restrict__ logd, const float* __restrict__ deg, const double* __restrict__ ms,
                            float* __restrict__ f, float* __restrict__ invdeg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        f[2 * i] = (float)((logd[i] - ms[0]) / ms[1]);
        f[2 * i + 1] = log1pf(deg[i]);
        invdeg[i] = deg[i] > 0 ? 1.0f / deg[i] : 0.0f;
    }
}

__global__ void k_chain_id(int nc, const int32_t* __restrict__ cs, const int32_t* __restrict__ cl, int32_t* __restrict__ id) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
        for (int k = 0; k < cl[c]; k++) id[cs[c] + k] = c;
}

__global__ void k_blk_of_row(int n, const int32_t* __restrict__ is_start, const int32_t* __restrict__ scan, int32_t* __restrict__ blk) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) blk[i] = scan[i] + is_start[i] - 1;
}

// Per entry: relative log conductance, junction flag, outside-the-blocks flag,
// and the index of the transposed entry (columns ascending in every row).
__global__ void k_entry_feat(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                             const double* __restrict__ logd, const int32_t* __restrict__ chain, const int32_t* __restrict__ blk,
                             float* __restrict__ lc, float* __restrict__ jf, uint8_t* __restrict__ offb, int32_t* __restrict__ tr,
                             int* status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            const int c = ci[k];
            const bool off = c != i;
            const double a = fabs(v[k]);
            lc[k] = (off && a > 0) ? (float)(log(a) - 0.5 * (logd[i] + logd[c])) : 0.0f;
            const bool seg = chain[i] == chain[c] && chain[i] >= 0 && (c == i + 1 || c == i - 1);
            jf[k] = (off && !seg) ? 1.0f : 0.0f;
            offb[k] = (off && blk[i] != blk[c]) ? 1 : 0;
            int lo = rp[c], hi = rp[c + 1] - 1, t = -1;
            while (lo <= hi) {
                const int mid = (lo + hi) >> 1;
                if (ci[mid] == i) { t = mid; break; }
                if (ci[mid] < i) lo = mid + 1; else hi = mid - 1;
            }
            if (t < 0) { atomicCAS(status, 0, (int)DEV_INPUT); t = k; }  // not symmetric: reported, entry maps to itself
            tr[k] = t;
        }
    }
}

// ---------------------------------------------------------------------------
// Forward
__global__ void k_layer0(int n, const float* __restrict__ f, const float* __restrict__ P, float* __restrict__ A0,
                         __nv_bfloat16* __restrict__ H) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * kW; e += gridDim.x * blockDim.x) {
        const int i = e / kW, j = e - i * kW;
        const float a = f[2 * i] * bfr(P[kOffWin + j]) + f[2 * i + 1] * bfr(P[kOffWin + kW + j]) + P[kOffBin + j];
        A0[e] = a;
        H[e] = __float2bfloat16_rn(fmaxf(a, 0.0f));
    }
}

// Y[n x 32] = X[n x 32] (bf16) * W[32 x 32] (fp32 master weights rounded to bf16), FP32
// accumulate, on the 5th-generation tensor cores: one CTA of 4 warps per 128-row tile, the
// tile and W^T staged in shared memory in the canonical K-major no-swizzle layout (core
// matrices of 8 rows x 16 bytes: element (row, k) at ((row / 8) * 4 + k / 8) * 128 +
// (row % 8) * 16 + (k % 8) * 2 bytes, so the K step is 128 bytes (LBO) and an 8-row group 512
// bytes (SBO)), two tcgen05.mma of M = 128, N = 32, K = 16 issued by one thread into a 32-column
// TMEM accumulator, completion by tcgen05.commit on an mbarrier (bounded wait), and each warp
// reading its 32 accumulator lanes back with tcgen05.ld (one row of 32 FP32 per thread).
constexpr int kGemmRows = 128;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ int umma_off(int row, int k) { return ((row >> 3) * 4 + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2; }

// shared-memory matrix descriptor: start address, LBO 128 B, SBO 512 B, descriptor version 1,
// no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) | (1ull << 46);
}

__global__ void __launch_bounds__(kGemmRows) k_gemm32(int n, const __nv_bfloat16* __restrict__ X, const float* __restrict__ W,
                                                      float* __restrict__ Yf, __nv_bfloat16* __restrict__ Yb, int* status) {
    __shared__ __align__(1024) unsigned char sA[kGemmRows * kW * 2];
    __shared__ __align__(1024) unsigned char sB[kW * kW * 2];
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ uint32_t tmem_base;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    for (int e = t; e < kW * kW; e += kGemmRows) {  // B = W^T, K-major
        const int k = e / kW, j = e % kW;
        *reinterpret_cast<__nv_bfloat16*>(sB + umma_off(j, k)) = __float2bfloat16_rn(W[e]);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)), "r"(kW));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (t == 0) asm volatile("mbarrier.init.shared.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    // kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N = 32, M = 128
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kW >> 3) << 17) | ((uint32_t)(kGemmRows >> 4) << 24);
    uint32_t phase = 0;
    const int ntiles = (n + kGemmRows - 1) / kGemmRows;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int r = tile * kGemmRows + t;
        const uint4* src = reinterpret_cast<const uint4*>(X + (size_t)r * kW);
        for (int kc = 0; kc < kW / 8; kc++)
            *reinterpret_cast<uint4*>(sA + umma_off(t, kc * 8)) = r < n ? src[kc] : make_uint4(0, 0, 0, 0);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic-proxy stores -> the MMA's async proxy
        __syncthreads();
        if (t == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int ks = 0; ks < kW / 16; ks++) {
                const uint64_t da = umma_desc(a0 + ks * 256), db = umma_desc(b0 + ks * 256);
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"((uint32_t)ks));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&mbar)) : "memory");
        }
        uint32_t done = 0;
        for (long long it = 0; it < (1ll << 26) && !done; it++)
            asm volatile("{\n\t.reg .pred q;\n\tmbarrier.try_wait.parity.shared.b64 q, [%1], %2;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
                         : "=r"(done) : "r"(smem_u32(&mbar)), "r"(phase) : "memory");
        if (!done && t == 0) atomicCAS(status, 0, (int)DEV_TIMEOUT);
        phase ^= 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t d[32];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                     "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                     : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
                       "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
                       "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]),
                       "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
                     : "r"(tmem + ((uint32_t)(warp * 32) << 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int row = tile * kGemmRows + warp * 32 + lane;
        if (row < n) {
            if (Yf)
                for (int j = 0; j < kW; j++) Yf[(size_t)row * kW + j] = __uint_as_float(d[j]);
            if (Yb)
                for (int j = 0; j < kW; j++) Yb[(size_t)row * kW + j] = __float2bfloat16_rn(__uint_as_float(d[j]));
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kW));
}

// Message passing + update of one layer: one warp per node, lane = feature.
__global__ void k_layer(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const float* __restrict__ lc,
                        const float* __restrict__ jf, const float* __restrict__ invdeg, const float* __restrict__ P,
                        const __nv_bfloat16* __restrict__ H, const __nv_bfloat16* __restrict__ G, const float* __restrict__ HW,
                        float* __restrict__ A, __nv_bfloat16* __restrict__ Hn) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const float p0 = P[kOffP], p1 = P[kOffP + 1], p2 = P[kOffP + 2], bj = P[kOffB + lane];
    for (int i = warp; i < n; i += nwarps) {
        float m = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            const int c = ci[k];
            if (c == i) continue;
            const float gate = sigm(p0 * lc[k] + p1 * jf[k] + p2);
            m += gate * __bfloat162float(G[c * kW + lane]);
        }
        m *= invdeg[i];
        const float a = HW[i * kW + lane] + m + bj;
        A[i * kW + lane] = a;
        Hn[i * kW + lane] = __float2bfloat16_rn(__bfloat162float(H[i * kW + lane]) + fmaxf(a, 0.0f));
    }
}

// Edge output on the couplings outside the blocks (0 elsewhere).
__global__ void k_edge_out(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const float* __restrict__ lc,
                           const uint8_t* __restrict__ offb, const float* __restrict__ P, const __nv_bfloat16* __restrict__ H,
                           float* __restrict__ w) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const float vj = P[kOffV + lane], q0 = P[kOffQ], q1 = P[kOffQ + 1];
    for (int i = warp; i < n; i += nwarps) {
        const float hi = vj * __bfloat162float(H[i * kW + lane]);
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            if (!offb[k]) {
                if (lane == 0) w[k] = 0.0f;
                continue;
            }
            const float o = wsum(hi * __bfloat162float(H[ci[k] * kW + lane])) + q0 * lc[k] + q1;
            if (lane == 0) w[k] = sigm(o);
        }
    }
}

// ---------------------------------------------------------------------------
// Preconditioner pieces (FP64)
__global__ void k_spmv(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                       const double* __restrict__ x, double* __restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++) s += v[k] * x[ci[k]];
        y[i] = s;
    }
}

__global__ void k_tapply(int n, const double* __restrict__ tinv, const int32_t* __restrict__ off, const int32_t* __restrict__ base,
                         const int32_t* __restrict__ m, const double* __restrict__ x, double* __restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0;
        const int o = off[i], b = base[i];
        for (int j = 0; j < m[i]; j++) s += tinv[o + j] * x[b + j];
        y[i] = s;
    }
}

// u_i = sum over couplings outside the blocks of w_ik |a_ik| y_k  (a_ik <= 0: -a_ik)
__global__ void k_ew_apply(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                           const float* __restrict__ w, const uint8_t* __restrict__ offb, const double* __restrict__ y,
                           double* __restrict__ u) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++)
            if (offb[k]) s += (double)w[k] * (-v[k]) * y[ci[k]];
        u[i] = s;
    }
}

// out = a x + y; out may be y (in-place updates), so neither is restrict-qualified.
__global__ void k_axpy(int n, double a, const double* __restrict__ x, const double* y, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = a * x[i] + y[i];
}

// Dot products r.q, r.r, q.q: per-CTA partials, then one thread sums them in order.
__global__ void k_dots3(int n, const double* __restrict__ r, const double* __restrict__ q, double* __restrict__ part) {
    __shared__ double s[3][32];
    double a = 0, b = 0, c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        a += r[i] * q[i];
        b += r[i] * r[i];
        c += q[i] * q[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0) { s[0][threadIdx.x >> 5] = a; s[1][threadIdx.x >> 5] = b; s[2][threadIdx.x >> 5] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double A = 0, B = 0, C = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { A += s[0][w]; B += s[1][w]; C += s[2][w]; }
        part[3 * blockIdx.x] = A;
        part[3 * blockIdx.x + 1] = B;
        part[3 * blockIdx.x + 2] = C;
    }
}

// loss of one probe and the coefficients of dL/dq = alpha r + beta q
__global__ void k_probe_loss(int nb, const double* __restrict__ part, double* __restrict__ coef, double* __restrict__ loss) {
    if (blockIdx.x || threadIdx.x) return;
    double rq = 0, rr = 0, qq = 0;
    for (int b = 0; b < nb; b++) { rq += part[3 * b]; rr += part[3 * b + 1]; qq += part[3 * b + 2]; }
    const double den = rr * qq;
    coef[0] = -2 * rq / den;
    coef[1] = 2 * rq * rq / (den * qq);
    loss[0] += 1 - rq * rq / den;
}

__global__ void k_combine(int n, const double* __restrict__ coef, const double* __restrict__ r, const double* __restrict__ q,
                          double* __restrict__ out) {
    const double a = coef[0], b = coef[1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = a * r[i] + b * q[i];
}

__global__ void k_dw(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                     const uint8_t* __restrict__ offb, const double* __restrict__ lam, const double* __restrict__ y,
                     double* __restrict__ dw) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; k++)
            if (offb[k]) dw[k] += lam[i] * (-v[k]) * y[ci[k]];
}

__global__ void k_do(int nnz, double scale, const double* __restrict__ dw, const float* __restrict__ w, const uint8_t* __restrict__ offb,
                     float* __restrict__ dout) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x)
        dout[k] = offb[k] ? (float)(dw[k] * scale) * w[k] * (1.0f - w[k]) : 0.0f;
}

// ---------------------------------------------------------------------------
// Backward of the network (FP32)
__global__ void k_edge_bwd(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const float* __restrict__ lc,
                           const int32_t* __restrict__ tr, const float* __restrict__ dout, const float* __restrict__ P,
                           const __nv_bfloat16* __restrict__ H, float* __restrict__ dH, float* __restrict__ grad) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const float vj = P[kOffV + lane];
    float gv = 0, gq0 = 0, gq1 = 0;
    for (int i = warp; i < n; i += nwarps) {
        const float hi = __bfloat162float(H[i * kW + lane]);
        float dh = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            const float d1 = dout[k];
            const float d2 = dout[tr[k]];
            if (d1 == 0.0f && d2 == 0.0f) continue;
            const float hk = __bfloat162float(H[ci[k] * kW + lane]);
            dh += (d1 + d2) * vj * hk;
            gv += d1 * hi * hk;
            gq0 += d1 * lc[k];
            gq1 += d1;
        }
        dH[i * kW + lane] = dh;
    }
    atomicAdd(&grad[kOffV + lane], gv);
    if (lane == 0) {
        atomicAdd(&grad[kOffQ], gq0);
        atomicAdd(&grad[kOffQ + 1], gq1);
    }
}

// dA = dH (A > 0), dM = dA / deg; db += sum dA
__global__ void k_layer_bwd1(int n, const float* __restrict__ A, const float* __restrict__ dH, const float* __restrict__ invdeg,
                             float* __restrict__ dA, float* __restrict__ dM, float* __restrict__ gb) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    float acc = 0;
    for (int i = warp; i < n; i += nwarps) {
        const float d = A[i * kW + lane] > 0.0f ? dH[i * kW + lane] : 0.0f;
        dA[i * kW + lane] = d;
        dM[i * kW + lane] = d * invdeg[i];
        acc += d;
    }
    atomicAdd(&gb[lane], acc);
}

// dG_a = sum_c gate_ac dM_c ; dp += dgate gate (1 - gate) (lc, jf, 1) with dgate_ac = dM_a . G_c
__global__ void k_layer_bwd2(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const float* __restrict__ lc,
                             const float* __restrict__ jf, const float* __restrict__ P, const __nv_bfloat16* __restrict__ G,
                             const float* __restrict__ dM, float* __restrict__ dG, float* __restrict__ gp) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    const float p0 = P[kOffP], p1 = P[kOffP + 1], p2 = P[kOffP + 2];
    float a0 = 0, a1 = 0, a2 = 0;
    for (int i = warp; i < n; i += nwarps) {
        const float dmi = dM[i * kW + lane];
        float dg = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            const int c = ci[k];
            if (c == i) continue;
            const float gate = sigm(p0 * lc[k] + p1 * jf[k] + p2);
            dg += gate * dM[c * kW + lane];
            const float dgate = wsum(dmi * __bfloat162float(G[c * kW + lane]));
            const float dpre = dgate * gate * (1.0f - gate);
            a0 += dpre * lc[k];
            a1 += dpre * jf[k];
            a2 += dpre;
        }
        dG[i * kW + lane] = dg;
    }
    if (lane == 0) {
        atomicAdd(&gp[0], a0);
        atomicAdd(&gp[1], a1);
        atomicAdd(&gp[2], a2);
    }
}

// dH_l = dH_{l+1} + dA W^T + dG U^T ; dW += H^T dA ; dU += H^T dG  (weights as bf16)
__global__ void __launch_bounds__(256) k_dense_bwd(int n, const __nv_bfloat16* __restrict__ H, const float* __restrict__ dA,
                                                   const float* __restrict__ dG, const float* __restrict__ P, const float* __restrict__ dHin,
                                                   float* __restrict__ dHout, float* __restrict__ gW, float* __restrict__ gU) {
    __shared__ float Wb[kW * kW], Ub[kW * kW], aW[kW * kW], aU[kW * kW];
    for (int e = threadIdx.x; e < kW * kW; e += blockDim.x) {
        Wb[e] = bfr(P[kOffW + e]);
        Ub[e] = bfr(P[kOffU + e]);
        aW[e] = 0;
        aU[e] = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    float accW[kW], accU[kW];
    for (int a = 0; a < kW; a++) { accW[a] = 0; accU[a] = 0; }
    for (int i = warp; i < n; i += nwarps) {
        const float da = dA[i * kW + lane], dg = dG[i * kW + lane];
        const float h = __bfloat162float(H[i * kW + lane]);
        float s = dHin[i * kW + lane];
        for (int m = 0; m < kW; m++) {
            const float dam = __shfl_sync(0xffffffffu, da, m), dgm = __shfl_sync(0xffffffffu, dg, m);
            s += dam * Wb[lane * kW + m] + dgm * Ub[lane * kW + m];
            const float ha = __shfl_sync(0xffffffffu, h, m);  // H[i][m]
            accW[m] += ha * da;                                // dW[m][lane]
            accU[m] += ha * dg;
        }
        dHout[i * kW + lane] = s;
    }
    for (int a = 0; a < kW; a++) {
        atomicAdd(&aW[a * kW + lane], accW[a]);
        atomicAdd(&aU[a * kW + lane], accU[a]);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kW * kW; e += blockDim.x) {
        atomicAdd(&gW[e], aW[e]);
        atomicAdd(&gU[e], aU[e]);
    }
}

__global__ void k_layer0_bwd(int n, const float* __restrict__ f, const float* __restrict__ A0, const float* __restrict__ dH,
                             float* __restrict__ grad) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    float g0 = 0, g1 = 0, gb = 0;
    for (int i = warp; i < n; i += nwarps) {
        const float d = A0[i * kW + lane] > 0.0f ? dH[i * kW + lane] : 0.0f;
        g0 += f[2 * i] * d;
        g1 += f[2 * i + 1] * d;
        gb += d;
    }
    atomicAdd(&grad[kOffWin + lane], g0);
    atomicAdd(&grad[kOffWin + kW + lane], g1);
    atomicAdd(&grad[kOffBin + lane], gb);
}

__global__ void k_adam(int n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, float lr,
                       float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = 0.9f * m[i] + 0.1f * gi;
        const float vi = 0.999f * v[i] + 0.001f * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
int gnn_param_count() { return kParams; }

void gnn_set_system(GnnState& g, int n, int nnz, const int32_t* rp, const int32_t* ci, const double* val, int nchains,
                    const int32_t* cs, const int32_t* cl, cudaStream_t s, int64_t& launches) {
    g.n = n;
    g.nnz = nnz;
    g.rp = rp;
    g.ci = ci;
    g.val = val;
    g.status.ensure(1);
    CICY_CUDA(cudaMemsetAsync(g.status.get(), 0, sizeof(int), s));
    g.diag.ensure(n + 1);
    g.logd.ensure(n + 1);
    g.deg.ensure(n + 1);
    g.ms.ensure(2);
    g.f.ensure(2 * (size_t)n + 2);
    g.invdeg.ensure(n + 1);
    g.chain.ensure(n + 1);
    g.blk.ensure(n + 1);
    g.lc.ensure(nnz + 1);
    g.jf.ensure(nnz + 1);
    g.offb.ensure(nnz + 1);
    g.tr.ensure(nnz + 1);
    k_diag_deg<<<grid_for(n), 256, 0, s>>>(n, rp, ci, val, g.diag.get(), g.logd.get(), g.deg.get());
    k_mean_std<<<1, 1024, 0, s>>>(n, g.logd.get(), g.ms.get());
    k_node_feat<<<grid_for(n), 256, 0, s>>>(n, g.logd.get(), g.deg.get(), g.ms.get(), g.f.get(), g.invdeg.get());
    CICY_CUDA(cudaMemsetAsync(g.chain.get(), 0xff, sizeof(int32_t) * (n + 1), s));
    k_chain_id<<<grid_for(nchains), 256, 0, s>>>(nchains, cs, cl, g.chain.get());
    launches += 4;
    SolverSystem ss;
    ss.n = n;
    ss.nnz = nnz;
    ss.rp = rp;
    ss.ci = ci;
    ss.val = val;
    ss.diag = g.diag.get();
    build_block_preconditioner(g.sw, ss, nchains, cs, cl, nullptr, nullptr, false, s, launches);
    k_blk_of_row<<<grid_for(n), 256, 0, s>>>(n, g.sw.is_start.get(), g.sw.start_scan.get(), g.blk.get());
    k_entry_feat<<<grid_for(n), 256, 0, s>>>(n, rp, ci, val, g.logd.get(), g.chain.get(), g.blk.get(), g.lc.get(), g.jf.get(),
                                             g.offb.get(), g.tr.get(), g.status.get());
    launches += 2;
    int st = 0;
    CICY_CUDA(cudaMemcpyAsync(&st, g.status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    if (st) throw Fail{CICY_E_INPUT, "learned preconditioner: the matrix is not structurally symmetric with ascending columns"};
    const size_t nw = (size_t)n * kW + kW;
    g.A0.ensure(nw);
    g.HW.ensure(nw);
    for (int l = 0; l <= kLayers; l++) g.H[l].ensure(nw);
    for (int l = 0; l < kLayers; l++) {
        g.G[l].ensure(nw);
        g.A[l].ensure(nw);
    }
    g.w.ensure(nnz + 1);
    CICY_LAUNCH_CHECK();
}

void gnn_forward(GnnState& g, const float* P, cudaStream_t s, int64_t& launches) {
    const int n = g.n;
    k_layer0<<<grid_for((long long)n * kW), 256, 0, s>>>(n, g.f.get(), P, g.A0.get(), g.H[0].get());
    launches++;
    const int gemm_grid = std::max(1, std::min(148 * 4, ceil_div(n, kGemmRows)));
    g.status.ensure(1);
    for (int l = 0; l < kLayers; l++) {
        const float* Pl = P + kOffLayer0 + l * kLayerParams;
        k_gemm32<<<gemm_grid, kGemmRows, 0, s>>>(n, g.H[l].get(), Pl + kOffU, nullptr, g.G[l].get(), g.status.get());
        k_gemm32<<<gemm_grid, kGemmRows, 0, s>>>(n, g.H[l].get(), Pl + kOffW, g.HW.get(), nullptr, g.status.get());
        k_layer<<<warps_grid(n), 256, 0, s>>>(n, g.rp, g.ci, g.lc.get(), g.jf.get(), g.invdeg.get(), Pl, g.H[l].get(), g.G[l].get(),
                                              g.HW.get(), g.A[l].get(), g.H[l + 1].get());
        launches += 3;
    }
    k_edge_out<<<warps_grid(n), 256, 0, s>>>(n, g.rp, g.ci, g.lc.get(), g.offb.get(), P, g.H[kLayers].get(), g.w.get());
    launches++;
    CICY_LAUNCH_CHECK();
}

// z = T^-1 r + T^-1 E_w T^-1 r; y keeps T^-1 r
static void spai_apply(GnnState& g, const double* r, double* y, double* u, double* z, cudaStream_t s, int64_t& launches) {
    const int n = g.n;
    k_tapply<<<grid_for(n), 256, 0, s>>>(n, g.sw.tinv.get(), g.sw.row_off.get(), g.sw.row_base.get(), g.sw.row_m.get(), r, y);
    k_ew_apply<<<grid_for(n), 256, 0, s>>>(n, g.rp, g.ci, g.val, g.w.get(), g.offb.get(), y, u);
    k_tapply<<<grid_for(n), 256, 0, s>>>(n, g.sw.tinv.get(), g.sw.row_off.get(), g.sw.row_base.get(), g.sw.row_m.get(), u, z);
    k_axpy<<<grid_for(n), 256, 0, s>>>(n, 1.0, y, z, z);
    launches += 4;
}

double gnn_loss_grad(GnnState& g, const float* P, int K, const double* probes, float* grad, cudaStream_t s, int64_t& launches) {
    const int n = g.n, nnz = g.nnz;
    gnn_forward(g, P, s, launches);
    g.vr.ensure(n + 1); g.vy.ensure(n + 1); g.vu.ensure(n + 1); g.vz.ensure(n + 1); g.vq.ensure(n + 1);
    g.vd.ensure(n + 1); g.vl.ensure(n + 1);
    g.dw.ensure(nnz + 1);
    g.dout.ensure(nnz + 1);
    const int nbd = std::min(grid_for(n), 256);
    g.part.ensure(3 * (size_t)nbd + 3);
    g.coef.ensure(4);
    CICY_CUDA(cudaMemsetAsync(g.dw.get(), 0, sizeof(double) * (nnz + 1), s));
    CICY_CUDA(cudaMemsetAsync(g.coef.get(), 0, sizeof(double) * 4, s));
    for (int p = 0; p < K; p++) {
        const double* u0 = probes + (size_t)p * n;
        k_spmv<<<grid_for(n), 256, 0, s>>>(n, g.rp, g.ci, g.val, u0, g.vr.get());
        spai_apply(g, g.vr.get(), g.vy.get(), g.vu.get(), g.vz.get(), s, launches);
        k_spmv<<<grid_for(n), 256, 0, s>>>(n, g.rp, g.ci, g.val, g.vz.get(), g.vq.get());
        k_dots3<<<nbd, 256, 0, s>>>(n, g.vr.get(), g.vq.get(), g.part.get());
        k_probe_loss<<<1, 32, 0, s>>>(nbd, g.part.get(), g.coef.get(), g.coef.get() + 2);
        k_combine<<<grid_for(n), 256, 0, s>>>(n, g.coef.get(), g.vr.get(), g.vq.get(), g.vd.get());  // dL/dq
        k_spmv<<<grid_for(n), 256, 0, s>>>(n, g.rp, g.ci, g.val, g.vd.get(), g.vu.get());             // dL/dz
        k_tapply<<<grid_for(n), 256, 0, s>>>(n, g.sw.tinv.get(), g.sw.row_off.get(), g.sw.row_base.get(), g.sw.row_m.get(), g.vu.get(),
                                             g.vl.get());                                              // lambda
        k_dw<<<grid_for(n), 256, 0, s>>>(n, g.rp, g.ci, g.val, g.offb.get(), g.vl.get(), g.vy.get(), g.dw.get());
        launches += 8;
    }
    k_do<<<grid_for(nnz), 256, 0, s>>>(nnz, 1.0 / K, g.dw.get(), g.w.get(), g.offb.get(), g.dout.get());
    launches++;
    // ---- backward through the network ----
    CICY_CUDA(cudaMemsetAsync(grad, 0, sizeof(float) * kParams, s));
    const size_t nw = (size_t)n * kW + kW;
    g.dH0.ensure(nw); g.dH1.ensure(nw); g.dA.ensure(nw); g.dM.ensure(nw); g.dG.ensure(nw);
    k_edge_bwd<<<warps_grid(n), 256, 0, s>>>(n, g.rp, g.ci, g.lc.get(), g.tr.get(), g.dout.get(), P, g.H[kLayers].get(), g.dH0.get(),
                                             grad);
    launches++;
    float* dh = g.dH0.get();
    float* dh2 = g.dH1.get();
    const int dense_grid = std::min(148, std::max(1, ceil_div(n, 8 * 16)));
    for (int l = kLayers - 1; l >= 0; l--) {
        const float* Pl = P + kOffLayer0 + l * kLayerParams;
        float* gl = grad + kOffLayer0 + l * kLayerParams;
        k_layer_bwd1<<<warps_grid(n), 256, 0, s>>>(n, g.A[l].get(), dh, g.invdeg.get(), g.dA.get(), g.dM.get(), gl + kOffB);
        k_layer_bwd2<<<warps_grid(n), 256, 0, s>>>(n, g.rp, g.ci, g.lc.get(), g.jf.get(), Pl, g.G[l].get(), g.dM.get(), g.dG.get(),
                                                   gl + kOffP);
        k_dense_bwd<<<dense_grid, 256, 0, s>>>(n, g.H[l].get(), g.dA.get(), g.dG.get(), Pl, dh, dh2, gl + kOffW, gl + kOffU);
        launches += 3;
        std::swap(dh, dh2);
    }
    k_layer0_bwd<<<warps_grid(n), 256, 0, s>>>(n, g.f.get(), g.A0.get(), dh, grad);
    launches++;
    double h[4];
    CICY_CUDA(cudaMemcpyAsync(h, g.coef.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    CICY_LAUNCH_CHECK();
    return h[2] / K;
}

// u <- u - 0.9 T^-1 A u, `sweeps` times, for each of K probe vectors
void gnn_smooth_probes(GnnState& g, int K, double* u, int sweeps, cudaStream_t s, int64_t& launches) {
    const int n = g.n;
    g.vr.ensure(n + 1);
    g.vy.ensure(n + 1);
    for (int p = 0; p < K; p++) {
        double* up = u + (size_t)p * n;
        for (int it = 0; it < sweeps; it++) {
            k_spmv<<<grid_for(n), 256, 0, s>>>(n, g.rp, g.ci, g.val, up, g.vr.get());
            k_tapply<<<grid_for(n), 256, 0, s>>>(n, g.sw.tinv.get(), g.sw.row_off.get(), g.sw.row_base.get(), g.sw.row_m.get(), g.vr.get(),
                                                 g.vy.get());
            k_axpy<<<grid_for(n), 256, 0, s>>>(n, -0.9, g.vy.get(), up, up);
            launches += 3;
        }
    }
    CICY_LAUNCH_CHECK();
}

void gnn_adam(float* p, const float* gr, float* m, float* v, int n, int step, float lr, cudaStream_t s) {
    const float c1 = 1.0f - powf(0.9f, (float)step), c2 = 1.0f - powf(0.999f, (float)step);
    k_adam<<<grid_for(n), 256, 0, s>>>(n, p, gr, m, v, lr, c1, c2);
    CICY_LAUNCH_CHECK();
}

// Edge weights of the learned preconditioner for the system being solved.
const float* learned_edge_weights(Ctx& c, const SolverSystem& ss, int n_chains, cudaStream_t s) {
    if (c.gnn_params.n != (size_t)kParams) throw Fail{CICY_E_STATE, "learned preconditioner selected but no parameters were set"};
    gnn_set_system(c.gnn, ss.n, ss.nnz, ss.rp, ss.ci, ss.val, n_chains, c.chain_start.get(), c.chain_len.get(), s, c.launches);
    gnn_forward(c.gnn, c.gnn_params.get(), s, c.launches);
    return c.gnn.w.get();
}

}  // namespace cicy

// ---------------------------------------------------------------------------
// C ABI of the training entry points
struct cicy_gnn {
    int device = 0;
    cicy::GnnState g;
    cicy::DBuf<int> check;  // structure flags of the last cicy_gnn_set_system
    int64_t launches = 0;
};

namespace cicy {
namespace {
__global__ void k_check_system(int n, int nnz, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, int nchains,
                               const int32_t* __restrict__ cs, const int32_t* __restrict__ cl, int* __restrict__ bad) {
    const int f = check_structure_part(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, n, nnz, rp, ci, nchains, cs, cl);
    if (f) atomicOr(bad, f);
}
}  // namespace
}  // namespace cicy

namespace {

template <class F>
cicy_status gnn_guard(int device, F&& f) {
    try {
        CICY_CUDA(cudaSetDevice(device));
        f();
        return CICY_OK;
    } catch (const cicy::Fail& e) {
        cicy::set_host_error(e.msg);
        return e.status;
    }
}

}  // namespace

extern "C" {

int32_t cicy_gnn_param_count(void) { return cicy::gnn_param_count(); }

cicy_status cicy_gnn_create(cicy_gnn** out, int device) {
    if (!out) return CICY_E_INPUT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        cicy::set_host_error("cicy_gnn_create: no such CUDA device");
        return CICY_E_DEVICE;
    }
    *out = new cicy_gnn;
    (*out)->device = device;
    return CICY_OK;
}

cicy_status cicy_gnn_destroy(cicy_gnn* g) {
    if (g) {
        cudaSetDevice(g->device);
        delete g;
    }
    return CICY_OK;
}

cicy_status cicy_gnn_set_system(cicy_gnn* g, const cicy_gnn_system* sys, void* stream) {
    if (!g || !sys || sys->n <= 0 || sys->nnz <= 0 || !sys->row_ptr || !sys->col_ind || !sys->values || sys->n_chains <= 0 ||
        !sys->chain_start || !sys->chain_len) {
        cicy::set_host_error("cicy_gnn_set_system: invalid system");
        return CICY_E_INPUT;
    }
    return gnn_guard(g->device, [&] {
        // the feature and message kernels use the column indices and chains as addresses: check them first
        cudaStream_t s = (cudaStream_t)stream;
        g->check.ensure(1);
        CICY_CUDA(cudaMemsetAsync(g->check.get(), 0, sizeof(int), s));
        cicy::k_check_system<<<std::min((std::max(sys->nnz, sys->n) + 255) / 256, 148 * 8), 256, 0, s>>>(
            sys->n, sys->nnz, sys->row_ptr, sys->col_ind, sys->n_chains, sys->chain_start, sys->chain_len, g->check.get());
        CICY_LAUNCH_CHECK();
        int bad = 0;
        CICY_CUDA(cudaMemcpyAsync(&bad, g->check.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaStreamSynchronize(s));
        if (bad) throw cicy::Fail{CICY_E_INPUT, "cicy_gnn_set_system: " + cicy::structure_error(bad)};
        cicy::gnn_set_system(g->g, sys->n, sys->nnz, sys->row_ptr, sys->col_ind, sys->values, sys->n_chains, sys->chain_start,
                             sys->chain_len, s, g->launches);
    });
}

cicy_status cicy_gnn_forward(cicy_gnn* g, const float* params, float* w, void* stream) {
    if (!g || !params || g->g.n <= 0) {
        cicy::set_host_error("cicy_gnn_forward: no system or parameters");
        return CICY_E_INPUT;
    }
    return gnn_guard(g->device, [&] {
        cudaStream_t s = (cudaStream_t)stream;
        cicy::gnn_forward(g->g, params, s, g->launches);
        if (w) CICY_CUDA(cudaMemcpyAsync(w, g->g.w.get(), sizeof(float) * g->g.nnz, cudaMemcpyDeviceToDevice, s));
        CICY_CUDA(cudaStreamSynchronize(s));
    });
}

cicy_status cicy_gnn_loss_grad(cicy_gnn* g, const float* params, int32_t n_probes, const double* probes, double* loss, float* grad,
                               void* stream) {
    if (!g || !params || !probes || !grad || n_probes <= 0 || g->g.n <= 0) {
        cicy::set_host_error("cicy_gnn_loss_grad: invalid arguments");
        return CICY_E_INPUT;
    }
    return gnn_guard(g->device, [&] {
        const double L = cicy::gnn_loss_grad(g->g, params, n_probes, probes, grad, (cudaStream_t)stream, g->launches);
        if (loss) *loss = L;
    });
}

cicy_status cicy_gnn_smooth_probes(cicy_gnn* g, int32_t n_probes, double* probes, int32_t sweeps, void* stream) {
    if (!g || !probes || n_probes <= 0 || sweeps < 0 || g->g.n <= 0) {
        cicy::set_host_error("cicy_gnn_smooth_probes: invalid arguments");
        return CICY_E_INPUT;
    }
    return gnn_guard(g->device, [&] {
        cicy::gnn_smooth_probes(g->g, n_probes, probes, sweeps, (cudaStream_t)stream, g->launches);
        CICY_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    });
}

cicy_status cicy_gnn_adam(float* params, const float* grad, float* m, float* v, int32_t n, int32_t step, float lr, void* stream) {
    if (!params || !grad || !m || !v || n <= 0 || step < 1) {
        cicy::set_host_error("cicy_gnn_adam: invalid arguments");
        return CICY_E_INPUT;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    return gnn_guard(dev, [&] { cicy::gnn_adam(params, grad, m, v, n, step, lr, (cudaStream_t)stream); });
}

}  // extern "C"
