// Cluster-resident preconditioned CG (sm_100a thread-block cluster + DSMEM).
//
// One cluster of kClusterCtas CTAs (non-portable size 16) solves one system
// with everything in shared memory: each CTA owns a contiguous range of rows
// (aligned to preconditioner blocks), holds its rows of the full symmetric CSR,
// the vectors x, r, z, p, q and the LDL^T factors of its preconditioner blocks.
// The SpMV reads z of rows owned by other CTAs through distributed shared
// memory (cluster.map_shared_rank); dot products are reduced by writing each
// CTA's partial into every CTA's shared memory followed by the hardware
// cluster barrier, so there is no global-memory round trip and no spin loop on
// the iteration's critical path.  Same recurrence, stopping test and FP64
// true-residual refinement as k_pcg (solver.cu); the block preconditioner is
// applied by per-block LDL^T sweeps in shared memory (Jacobi = blocks of one).
#include <algorithm>
#include <cmath>
#include <cooperative_groups.h>

#include "solver.cuh"

namespace cg = cooperative_groups;

namespace cicy {

namespace {

constexpr int kClusterThreads = 512;

int grid_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)b;
}

// LDL^T factors of each preconditioner block: lfac[k] (multiplier of row k-1,
// 0 at a block start) and ipiv[k] = 1/pivot; Jacobi blocks have lfac = 0.
// Learned scalings as in k_block_inverse.
__global__ void k_block_factors(int nb, int n, const int32_t* __restrict__ blk_row, const int32_t* __restrict__ rp,
                                const int32_t* __restrict__ ci, const double* __restrict__ v, const double* __restrict__ diag,
                                const float* __restrict__ node_scale, const float* __restrict__ edge_scale,
                                double* __restrict__ lfac, double* __restrict__ ipiv) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int r0 = blk_row[b];
        const int m = ((b + 1 < nb) ? blk_row[b + 1] : n) - r0;
        double e_prev = 0, piv_prev = 0;
        bool singular = false;
        for (int k = 0; k < m; k++) {
            const int i = r0 + k;
            double e = 0;
            if (k + 1 < m)
                for (int kk = rp[i]; kk < rp[i + 1]; kk++)
                    if (ci[kk] == i + 1) { e = v[kk]; break; }
            double coup = fabs(e) + fabs(e_prev);
            double s = node_scale ? (double)node_scale[i] : 1.0;
            double d = coup + s * (diag[i] - coup);
            if (edge_scale && k + 1 < m) e *= (double)edge_scale[i];
            double l = (k == 0) ? 0.0 : e_prev / piv_prev;
            double piv = d - l * e_prev;
            singular |= !(piv > 1e-13 * fabs(d));
            lfac[i] = l;
            ipiv[i] = 1.0 / piv;
            e_prev = e;
            piv_prev = piv;
        }
        if (singular)
            for (int k = 0; k < m; k++) {
                lfac[r0 + k] = 0.0;
                ipiv[r0 + k] = 1.0 / diag[r0 + k];
            }
    }
}

// Per-CTA sizes for the shared-memory layout: rows, non-zeros, first block.
__global__ void k_cta_stats(int C, const int32_t* __restrict__ cta_row, const int32_t* __restrict__ rp, int nblk,
                            const int32_t* __restrict__ blk_row, int32_t* __restrict__ out) {
    int b = threadIdx.x;
    if (b > C) return;
    const int r = cta_row[b];
    int lo = 0, hi = nblk;  // first block with start >= r
    while (lo < hi) {
        int m = (lo + hi) >> 1;
        if (blk_row[m] < r) lo = m + 1; else hi = m;
    }
    out[b] = lo;                 // first block of CTA b
    out[C + 1 + b] = rp[r];      // first non-zero of CTA b
}

struct ClusterArgs {
    int n, C;
    const int32_t* rp;
    const int32_t* ci;
    const double* val;
    const double* b;
    double* x;
    const double* lfac;
    const double* ipiv;
    const int32_t* cta_row;
    const int32_t* cta_blk;
    const int32_t* blk_row;
    int nblk;
    int nr_max, nnz_max, nb_max;
    double tol;
    long long max_iter;
    int max_restarts;
    double* stats;
};

struct Smem {
    double *r, *z, *p, *q, *x, *lf, *ip, *val, *slotA, *slotB, *red;
    int32_t *rp, *code, *blk;
};

__device__ __forceinline__ Smem carve(unsigned char* base, const ClusterArgs& a) {
    Smem s;
    double* d = reinterpret_cast<double*>(base);
    const int nr = a.nr_max;
    s.r = d; d += nr;
    s.z = d; d += nr;
    s.p = d; d += nr;
    s.q = d; d += nr;
    s.x = d; d += nr;
    s.lf = d; d += nr;
    s.ip = d; d += nr;
    s.val = d; d += a.nnz_max;
    s.slotA = d; d += 2 * 16;
    s.slotB = d; d += 16;
    s.red = d; d += 72;
    int32_t* i = reinterpret_cast<int32_t*>(d);
    s.rp = i; i += nr + 1;
    s.code = i; i += a.nnz_max;
    s.blk = i; i += a.nb_max + 1;
    return s;
}

__device__ __forceinline__ double2 block_sum2(double a, double b, double* red) {
    a = warp_sum(a);
    b = warp_sum(b);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { red[w] = a; red[32 + w] = b; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        double x = lane < nw ? red[lane] : 0.0, y = lane < nw ? red[32 + lane] : 0.0;
        x = warp_sum(x);
        y = warp_sum(y);
        if (lane == 0) { red[64] = x; red[65] = y; }
    }
    __syncthreads();
    double2 r = make_double2(red[64], red[65]);
    __syncthreads();
    return r;
}

// Write this CTA's partials into slot[rank] of every CTA, barrier, sum slots in rank order.
__device__ __forceinline__ double2 cluster_sum2(cg::cluster_group& cl, double* slot, int nval, double a, double b, double* red,
                                                int C, unsigned rank) {
    double2 v = block_sum2(a, b, red);
    if (threadIdx.x < C) {
        double* dst = cl.map_shared_rank(slot, threadIdx.x);
        dst[nval * rank] = v.x;
        if (nval > 1) dst[nval * rank + 1] = v.y;
    }
    cl.sync();
    double s0 = 0, s1 = 0;
    for (int k = 0; k < C; k++) {
        s0 += slot[nval * k];
        if (nval > 1) s1 += slot[nval * k + 1];
    }
    return make_double2(s0, s1);
}

// z = M^-1 r on this CTA's blocks (one thread per block, LDL^T sweep in shared memory).
__device__ __forceinline__ void precond(const Smem& s, int nblk_local, int nr) {
    for (int bi = threadIdx.x; bi < nblk_local; bi += blockDim.x) {
        const int b0 = s.blk[bi], b1 = s.blk[bi + 1];
        double y = s.r[b0];
        s.z[b0] = y;
        for (int k = b0 + 1; k < b1; k++) {
            y = s.r[k] - s.lf[k] * y;
            s.z[k] = y;
        }
        double zk = s.z[b1 - 1] * s.ip[b1 - 1];
        s.z[b1 - 1] = zk;
        for (int k = b1 - 2; k >= b0; k--) {
            zk = s.z[k] * s.ip[k] - s.lf[k + 1] * zk;
            s.z[k] = zk;
        }
    }
}

__global__ void __launch_bounds__(kClusterThreads) k_pcg_cluster(ClusterArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const int C = a.C;
    Smem s = carve(smem, a);
    const int r_lo = a.cta_row[rank], r_hi = a.cta_row[rank + 1], nr = r_hi - r_lo;
    const int nz0 = a.rp[r_lo];
    const int nnz = a.rp[r_hi] - nz0;
    const int blk0 = a.cta_blk[rank], nblk = a.cta_blk[rank + 1] - blk0;
    __shared__ int s_cta_row[17];
    if (threadIdx.x <= C) s_cta_row[threadIdx.x] = a.cta_row[threadIdx.x];
    // ---- load this CTA's slice
    for (int i = threadIdx.x; i <= nr; i += blockDim.x) s.rp[i] = a.rp[r_lo + i] - nz0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) s.blk[i] = a.blk_row[blk0 + i] - r_lo;
    if (threadIdx.x == 0) s.blk[nblk] = nr;
    __syncthreads();
    for (int k = threadIdx.x; k < nnz; k += blockDim.x) {
        const int col = a.ci[nz0 + k];
        int lo = 0, hi = C;  // owner: last CTA with cta_row <= col
        while (hi - lo > 1) {
            int m = (lo + hi) >> 1;
            if (s_cta_row[m] <= col) lo = m; else hi = m;
        }
        s.code[k] = (lo << 16) | (col - s_cta_row[lo]);
        s.val[k] = a.val[nz0 + k];
    }
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        s.x[i] = a.x[r_lo + i];
        s.lf[i] = a.lfac[r_lo + i];
        s.ip[i] = a.ipiv[r_lo + i];
    }
    __syncthreads();
    // remote views of z and x
    double* zr[16];
    double* xr[16];
    for (int k = 0; k < C; k++) {
        zr[k] = cl.map_shared_rank(s.z, k);
        xr[k] = cl.map_shared_rank(s.x, k);
    }
    cl.sync();  // every CTA has loaded x before anyone reads it remotely
    // ---- r = b - A x0, z = M^-1 r, partials
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        double acc = 0;
        for (int k = s.rp[i]; k < s.rp[i + 1]; k++) {
            const int c = s.code[k];
            acc += s.val[k] * xr[c >> 16][c & 0xffff];
        }
        s.r[i] = a.b[r_lo + i] - acc;
    }
    __syncthreads();
    precond(s, nblk, nr);
    __syncthreads();
    double rr_l = 0, rz_l = 0;
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        rr_l += s.r[i] * s.r[i];
        rz_l += s.r[i] * s.z[i];
    }
    double2 t = cluster_sum2(cl, s.slotA, 2, rr_l, rz_l, s.red, C, rank);
    double rr = t.x, rz = t.y;
    const double R0 = a.tol * sqrt(rr);
    double beta = 0, rr_new = rr;
    long long k = 0;
    int restarts = 0;
    bool fresh = true;
    while (true) {
        // ---- A: w = A z, q = w + beta q, p = z + beta p, partial p.q
        double pq_l = 0;
        for (int i = threadIdx.x; i < nr; i += blockDim.x) {
            double w = 0;
            for (int kk = s.rp[i]; kk < s.rp[i + 1]; kk++) {
                const int c = s.code[kk];
                w += s.val[kk] * zr[c >> 16][c & 0xffff];
            }
            const double qi = fresh ? w : w + beta * s.q[i];
            const double pi = fresh ? s.z[i] : s.z[i] + beta * s.p[i];
            s.q[i] = qi;
            s.p[i] = pi;
            pq_l += pi * qi;
        }
        const double pq = cluster_sum2(cl, s.slotB, 1, pq_l, 0.0, s.red, C, rank).x;
        fresh = false;
        k++;
        // ---- B: x += alpha p, r -= alpha q, z = M^-1 r, partials r.r, r.z
        const double alpha = rz / pq;
        for (int i = threadIdx.x; i < nr; i += blockDim.x) {
            s.x[i] += alpha * s.p[i];
            s.r[i] -= alpha * s.q[i];
        }
        __syncthreads();
        precond(s, nblk, nr);
        __syncthreads();
        rr_l = 0;
        rz_l = 0;
        for (int i = threadIdx.x; i < nr; i += blockDim.x) {
            rr_l += s.r[i] * s.r[i];
            rz_l += s.r[i] * s.z[i];
        }
        t = cluster_sum2(cl, s.slotA, 2, rr_l, rz_l, s.red, C, rank);
        rr_new = t.x;
        beta = t.y / rz;
        rz = t.y;
        if (sqrt(rr_new) <= R0) {
            if (restarts >= a.max_restarts) break;
            cl.sync();  // every CTA has read slotA before it is written again below
            // FP64 true residual from x of all CTAs (complete after the barrier above)
            for (int i = threadIdx.x; i < nr; i += blockDim.x) {
                double acc = 0;
                for (int kk = s.rp[i]; kk < s.rp[i + 1]; kk++) {
                    const int c = s.code[kk];
                    acc += s.val[kk] * xr[c >> 16][c & 0xffff];
                }
                s.r[i] = a.b[r_lo + i] - acc;
            }
            __syncthreads();
            precond(s, nblk, nr);
            __syncthreads();
            rr_l = 0;
            rz_l = 0;
            for (int i = threadIdx.x; i < nr; i += blockDim.x) {
                rr_l += s.r[i] * s.r[i];
                rz_l += s.r[i] * s.z[i];
            }
            t = cluster_sum2(cl, s.slotA, 2, rr_l, rz_l, s.red, C, rank);
            rr_new = t.x;
            rz = t.y;
            restarts++;
            if (sqrt(rr_new) <= R0) break;
            fresh = true;
        }
        if (k >= a.max_iter) break;
    }
    for (int i = threadIdx.x; i < nr; i += blockDim.x) a.x[r_lo + i] = s.x[i];
    if (rank == 0 && threadIdx.x == 0) {
        a.stats[0] = (double)k;
        a.stats[1] = rr_new;
        a.stats[2] = R0;
        a.stats[3] = (double)restarts;
    }
    cl.sync();  // no CTA exits while others may still read its shared memory
}

size_t smem_bytes(int nr, int nnz, int nb) {
    return sizeof(double) * (7 * (size_t)nr + nnz + 48 + 72) + sizeof(int32_t) * ((size_t)nr + 1 + nnz + nb + 1) + 64;
}

}  // namespace

bool pcg_solve_cluster(SolverWork& w, const SolverSystem& sys, bool block_precond, const float* node_scale,
                       const float* edge_scale, int nchains, const int32_t* chain_start, const int32_t* chain_len, double tol,
                       long long max_iter, cudaStream_t s, int64_t& launches, PcgStats& st) {
    const int n = sys.n;
    const int C = kClusterCtas;
    st = PcgStats{};
    if (n <= 0) return true;
    if (n < 4 * C || n >= (1 << 16) * C) return false;
    static int attr_state = 0;  // 0 unknown, 1 ok, -1 unsupported
    if (attr_state == 0) {
        cudaError_t e1 = cudaFuncSetAttribute(k_pcg_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaError_t e2 = cudaFuncSetAttribute(k_pcg_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, kClusterSmemMax);
        attr_state = (e1 == cudaSuccess && e2 == cudaSuccess) ? 1 : -1;
        cudaGetLastError();
    }
    if (attr_state < 0) return false;
    // preconditioner blocks: chain blocks (<= kBlockMax) or single rows (Jacobi)
    w.total.ensure(2);
    w.is_start.ensure(n + 1);
    w.start_scan.ensure(n + 1);
    if (block_precond) {
        CICY_CUDA(cudaMemsetAsync(w.is_start.get(), 0, sizeof(int32_t) * (n + 1), s));
        launch_block_marks(nchains, chain_start, chain_len, w.is_start.get(), s);
    } else {
        k_fill_ones<<<grid_for(n + 1), 256, 0, s>>>(n, w.is_start.get());
    }
    exclusive_scan_i32(w.is_start.get(), w.start_scan.get(), n, w.total.get(), w.scan_tmp, s, launches);
    int nblk = 0;
    CICY_CUDA(cudaMemcpyAsync(&nblk, w.total.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    w.blk_row.ensure(nblk + 1);
    launch_block_fill(n, w.is_start.get(), w.start_scan.get(), w.blk_row.get(), s);
    w.lfac.ensure(n);
    w.ipiv.ensure(n);
    k_block_factors<<<grid_for(nblk, 128), 128, 0, s>>>(nblk, n, w.blk_row.get(), sys.rp, sys.ci, sys.val, sys.diag, node_scale,
                                                       edge_scale, w.lfac.get(), w.ipiv.get());
    w.cta_row.ensure(C + 1);
    launch_cta_rows(C, n, w.is_start.get(), w.cta_row.get(), s);
    w.cta_stats.ensure(2 * (C + 1));
    k_cta_stats<<<1, 32, 0, s>>>(C, w.cta_row.get(), sys.rp, nblk, w.blk_row.get(), w.cta_stats.get());
    launches += 5;
    int h_row[17], h_st[34];
    CICY_CUDA(cudaMemcpyAsync(h_row, w.cta_row.get(), sizeof(int) * (C + 1), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaMemcpyAsync(h_st, w.cta_stats.get(), sizeof(int) * 2 * (C + 1), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    int nr_max = 0, nnz_max = 0, nb_max = 0;
    for (int b = 0; b < C; b++) {
        int nr = h_row[b + 1] - h_row[b];
        int nb = (b + 1 < C ? h_st[b + 1] : nblk) - h_st[b];
        int nz = (b + 1 < C ? h_st[C + 1 + b + 1] : sys.nnz) - h_st[C + 1 + b];
        nr_max = std::max(nr_max, nr);
        nnz_max = std::max(nnz_max, nz);
        nb_max = std::max(nb_max, nb);
    }
    if (nr_max >= (1 << 16)) return false;
    const size_t smem = smem_bytes(nr_max, nnz_max, nb_max);
    if (smem > (size_t)kClusterSmemMax) return false;
    w.stats.ensure(4);
    CICY_CUDA(cudaMemsetAsync(w.stats.get(), 0, sizeof(double) * 4, s));
    ClusterArgs a{};
    a.n = n; a.C = C;
    a.rp = sys.rp; a.ci = sys.ci; a.val = sys.val; a.b = sys.b; a.x = sys.x;
    a.lfac = w.lfac.get(); a.ipiv = w.ipiv.get();
    a.cta_row = w.cta_row.get(); a.cta_blk = w.cta_stats.get(); a.blk_row = w.blk_row.get(); a.nblk = nblk;
    a.nr_max = nr_max; a.nnz_max = nnz_max; a.nb_max = nb_max;
    a.tol = tol; a.max_iter = max_iter; a.max_restarts = 24;
    a.stats = w.stats.get();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, (void*)k_pcg_cluster, &cfg) != cudaSuccess || nclusters < 1) {
        cudaGetLastError();
        return false;
    }
    cudaEvent_t e0, e1;
    CICY_CUDA(cudaEventCreate(&e0));
    CICY_CUDA(cudaEventCreate(&e1));
    CICY_CUDA(cudaEventRecord(e0, s));
    CICY_CUDA(cudaLaunchKernelEx(&cfg, k_pcg_cluster, a));
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
    st.ctas = C;
    st.cluster = true;
    return true;
}

}  // namespace cicy
