// Cluster-resident preconditioned CG (sm_100a thread-block cluster + DSMEM).
//
// One cluster of kClusterCtas CTAs (non-portable size 16) solves one system
// with everything in shared memory.  Each CTA owns a contiguous range of rows
// (aligned to preconditioner blocks) and holds its rows of the full symmetric
// CSR (columns renumbered to local indices), the vectors x, r, z, p, q, the
// LDL^T factors of its preconditioner blocks, and a halo: a copy of the z
// entries of other CTAs' rows its rows reference.  The owner of a row pushes
// its new z value into every consumer's halo with distributed-shared-memory
// stores right after computing it, so the SpMV reads local shared memory only
// and no remote load sits on an iteration's critical path.  Dot products are
// reduced by storing each CTA's partial into every CTA's shared memory; the
// hardware cluster barrier that follows also publishes the halo pushes.  Two
// cluster barriers per iteration, no global-memory round trip, no spin loop.
//
// Same recurrence, stopping test and FP64 true-residual refinement as k_pcg
// (solver.cu); the block preconditioner is applied by one LDL^T sweep per block
// in shared memory (Jacobi = blocks of one row).
#include <algorithm>
#include <cmath>
#include <cooperative_groups.h>

#include "solver.cuh"
#include "trace.cuh"

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

__device__ __forceinline__ int owner_of(const int32_t* __restrict__ cta_row, int C, int i) {
    int lo = 0, hi = C;  // last CTA with cta_row <= i
    while (hi - lo > 1) {
        int m = (lo + hi) >> 1;
        if (cta_row[m] <= i) lo = m; else hi = m;
    }
    return lo;
}

// LDL^T factors of each preconditioner block: lfac[k] (multiplier of row k-1,
// 0 at a block start) and ipiv[k] = 1/pivot; Jacobi blocks have lfac = 0.
// Learned scalings as in k_block_inverse (solver.cu).
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
        if (singular)  // a CNT decoupled from the rest of the system: diagonal instead
            for (int k = 0; k < m; k++) {
                lfac[r0 + k] = 0.0;
                ipiv[r0 + k] = 1.0 / diag[r0 + k];
            }
    }
}

// Per CTA: first preconditioner block and first non-zero.
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
    out[b] = lo;
    out[C + 1 + b] = rp[r];
}

// Halo: mark[c * n + col] = 1 when a row of CTA c references column col of another CTA.
__global__ void k_halo_mark(int n, int C, const int32_t* __restrict__ cta_row, const int32_t* __restrict__ rp,
                            const int32_t* __restrict__ ci, int32_t* __restrict__ mark) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = owner_of(cta_row, C, i);
        const int lo = cta_row[c], hi = cta_row[c + 1];
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            const int col = ci[k];
            if (col < lo || col >= hi) mark[(long long)c * n + col] = 1;
        }
    }
}

__global__ void k_halo_ptr(int n, int C, const int32_t* __restrict__ mscan, int total, int32_t* __restrict__ halo_ptr) {
    for (int c = threadIdx.x; c <= C; c += blockDim.x) halo_ptr[c] = (c == C) ? total : mscan[(long long)c * n];
}

// Local column codes: own rows -> col - row_lo, halo -> nr_max + slot.
__global__ void k_halo_codes(int n, int C, int nr_max, const int32_t* __restrict__ cta_row, const int32_t* __restrict__ rp,
                             const int32_t* __restrict__ ci, const int32_t* __restrict__ mscan, const int32_t* __restrict__ halo_ptr,
                             uint16_t* __restrict__ code) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = owner_of(cta_row, C, i);
        const int lo = cta_row[c], hi = cta_row[c + 1];
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            const int col = ci[k];
            int v;
            if (col >= lo && col < hi) v = col - lo;
            else v = nr_max + (mscan[(long long)c * n + col] - halo_ptr[c]);
            code[k] = (uint16_t)v;
        }
    }
}

// Send lists: for each halo entry (consumer c, slot) of a column owned by CTA o,
// an entry in o's list: local row | slot << 16 | c << 32.
__global__ void k_send_count(int n, int C, const int32_t* __restrict__ cta_row, const int32_t* __restrict__ mark, int32_t* cnt) {
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)C * n;
         idx += (long long)gridDim.x * blockDim.x)
        if (mark[idx]) atomicAdd(&cnt[owner_of(cta_row, C, (int)(idx % n))], 1);
}

__global__ void k_send_fill(int n, int C, const int32_t* __restrict__ cta_row, const int32_t* __restrict__ mark,
                            const int32_t* __restrict__ mscan, const int32_t* __restrict__ halo_ptr, int32_t* cursor,
                            unsigned long long* __restrict__ send) {
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)C * n;
         idx += (long long)gridDim.x * blockDim.x) {
        if (!mark[idx]) continue;
        const int c = (int)(idx / n), col = (int)(idx % n);
        const int o = owner_of(cta_row, C, col);
        const unsigned long long row_local = (unsigned long long)(col - cta_row[o]);
        const unsigned long long slot = (unsigned long long)(mscan[idx] - halo_ptr[c]);
        const int pos = atomicAdd(&cursor[o], 1);
        send[pos] = row_local | (slot << 16) | ((unsigned long long)c << 32);
    }
}

struct ClusterArgs {
    int n, C;
    const int32_t* rp;
    const uint16_t* code;
    const double* val;
    const double* b;
    double* x;
    const double* lfac;
    const double* ipiv;
    const int32_t* cta_row;
    const int32_t* cta_blk;
    const int32_t* blk_row;
    const int32_t* send_ptr;
    const unsigned long long* send;
    int nr_max, nnz_max, nb_max, h_max, s_max;
    double tol;
    long long max_iter;
    int max_restarts;
    double* stats;
};

struct Smem {
    double *r, *zf, *p, *q, *x, *lf, *ip, *val, *slotA, *slotB, *red;
    unsigned long long* send;
    int32_t *rp, *blk;
    uint16_t* code;
};

__host__ __device__ inline size_t smem_layout(int nr, int nnz, int nb, int h, int sn, Smem* s, unsigned char* base) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (bytes + 15) / 16 * 16;
        return base ? (void*)(base + o) : nullptr;
    };
    double* r = (double*)take(sizeof(double) * nr);
    double* zf = (double*)take(sizeof(double) * (nr + h));
    double* p = (double*)take(sizeof(double) * nr);
    double* q = (double*)take(sizeof(double) * nr);
    double* x = (double*)take(sizeof(double) * nr);
    double* lf = (double*)take(sizeof(double) * nr);
    double* ip = (double*)take(sizeof(double) * nr);
    double* val = (double*)take(sizeof(double) * nnz);
    double* slotA = (double*)take(sizeof(double) * 32);
    double* slotB = (double*)take(sizeof(double) * 32);  // two doubles per CTA, like slotA
    double* red = (double*)take(sizeof(double) * 72);
    unsigned long long* send = (unsigned long long*)take(sizeof(unsigned long long) * sn);
    int32_t* rp = (int32_t*)take(sizeof(int32_t) * (nr + 1));
    int32_t* blk = (int32_t*)take(sizeof(int32_t) * (nb + 1));
    uint16_t* code = (uint16_t*)take(sizeof(uint16_t) * nnz);
    if (s) {
        s->r = r; s->zf = zf; s->p = p; s->q = q; s->x = x; s->lf = lf; s->ip = ip; s->val = val;
        s->slotA = slotA; s->slotB = slotB; s->red = red; s->send = send; s->rp = rp; s->blk = blk; s->code = code;
    }
    return off;
}

// Cluster-wide sum, split in two: store the block partials into every CTA's slots ...
__device__ __forceinline__ void cluster_store2(cg::cluster_group& cl, double* slot, double a, double b, double* red, int C,
                                               unsigned rank) {
    a = warp_sum(a);
    b = warp_sum(b);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) { red[w] = a; red[32 + w] = b; }
    __syncthreads();
    if (w == 0) {
        double s0 = lane < nw ? red[lane] : 0.0, s1 = lane < nw ? red[32 + lane] : 0.0;
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        s0 = __shfl_sync(0xffffffffu, s0, 0);
        s1 = __shfl_sync(0xffffffffu, s1, 0);
        if (lane < C) {
            double* dst = cl.map_shared_rank(slot, lane);
            dst[2 * rank] = s0;
            dst[2 * rank + 1] = s1;
        }
    }
}

// ... and, after the cluster barrier, sum them in rank order.
__device__ __forceinline__ double2 cluster_slots2(const double* slot, int C) {
    const int lane = threadIdx.x & 31;
    double s0 = lane < C ? slot[2 * lane] : 0.0;
    double s1 = lane < C ? slot[2 * lane + 1] : 0.0;
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    return make_double2(__shfl_sync(0xffffffffu, s0, 0), __shfl_sync(0xffffffffu, s1, 0));
}

// z = M^-1 r on this CTA's blocks (one thread per block, LDL^T sweep in shared memory).
__device__ __forceinline__ void precond(const Smem& s, int nblk) {
    for (int bi = threadIdx.x; bi < nblk; bi += blockDim.x) {
        const int b0 = s.blk[bi], b1 = s.blk[bi + 1];
        double y = s.r[b0];
        s.zf[b0] = y;
        for (int k = b0 + 1; k < b1; k++) {
            y = s.r[k] - s.lf[k] * y;
            s.zf[k] = y;
        }
        double zk = s.zf[b1 - 1] * s.ip[b1 - 1];
        s.zf[b1 - 1] = zk;
        for (int k = b1 - 2; k >= b0; k--) {
            zk = s.zf[k] * s.ip[k] - s.lf[k + 1] * zk;
            s.zf[k] = zk;
        }
    }
}

// Push v[row] of this CTA's rows into the halos of the CTAs that reference them.
__device__ __forceinline__ void push_halo(const Smem& s, int nsend, const double* v, double* const* remote_zf, int nr_max) {
    for (int e = threadIdx.x; e < nsend; e += blockDim.x) {
        const unsigned long long t = s.send[e];
        const int row = (int)(t & 0xffff), slot = (int)((t >> 16) & 0xffff), dst = (int)(t >> 32);
        remote_zf[dst][nr_max + slot] = v[row];
    }
}

__global__ void __launch_bounds__(kClusterThreads) k_pcg_cluster(ClusterArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double* remote_zf[16];
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const int C = a.C, NR = a.nr_max;
    Smem s;
    smem_layout(a.nr_max, a.nnz_max, a.nb_max, a.h_max, a.s_max, &s, smem);
    const int r_lo = a.cta_row[rank], r_hi = a.cta_row[rank + 1], nr = r_hi - r_lo;
    const int nz0 = a.rp[r_lo];
    const int nnz = a.rp[r_hi] - nz0;
    const int blk0 = a.cta_blk[rank], nblk = a.cta_blk[rank + 1] - blk0;
    const int snd0 = a.send_ptr[rank], nsend = a.send_ptr[rank + 1] - snd0;
    if (threadIdx.x < C) remote_zf[threadIdx.x] = cl.map_shared_rank(s.zf, threadIdx.x);
    // ---- load this CTA's slice
    for (int i = threadIdx.x; i <= nr; i += blockDim.x) s.rp[i] = a.rp[r_lo + i] - nz0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) s.blk[i] = a.blk_row[blk0 + i] - r_lo;
    if (threadIdx.x == 0) s.blk[nblk] = nr;
    for (int k = threadIdx.x; k < nnz; k += blockDim.x) {
        s.code[k] = a.code[nz0 + k];
        s.val[k] = a.val[nz0 + k];
    }
    for (int e = threadIdx.x; e < nsend; e += blockDim.x) s.send[e] = a.send[snd0 + e];
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        s.x[i] = a.x[r_lo + i];
        s.lf[i] = a.lfac[r_lo + i];
        s.ip[i] = a.ipiv[r_lo + i];
    }
    cl.sync();  // all slices loaded, remote_zf set, before any push
    // ---- r = b - A x0 (x of other CTAs through the halo), z = M^-1 r, push z, partials
    push_halo(s, nsend, s.x, remote_zf, NR);
    cl.sync();
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        double acc = 0;
        for (int k = s.rp[i]; k < s.rp[i + 1]; k++) {
            const int c = s.code[k];
            acc += s.val[k] * (c < NR ? s.x[c] : s.zf[c]);
        }
        s.r[i] = a.b[r_lo + i] - acc;
    }
    cl.sync();  // every CTA has read its x halo before the z pushes below overwrite it
    precond(s, nblk);
    __syncthreads();
    push_halo(s, nsend, s.zf, remote_zf, NR);
    double rr_l = 0, rz_l = 0;
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        rr_l += s.r[i] * s.r[i];
        rz_l += s.r[i] * s.zf[i];
    }
    // Scalars are formed once per CTA by warp 0 and broadcast through shared memory
    // (sc[]): the FP64 pipe of the cluster's 16 SMs is the scarce resource, so no
    // thread repeats the divisions.  sc: 0 alpha, 1 beta, 2 rz, 3 rr_new, 4 R0^2, 5 converged.
    double* sc = s.red + 64;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    cluster_store2(cl, s.slotA, rr_l, rz_l, s.red, C, rank);
    cl.sync();
    if (warp == 0) {
        double2 t0 = cluster_slots2(s.slotA, C);
        if (lane == 0) {
            sc[2] = t0.y;
            sc[3] = t0.x;
            const double R0 = a.tol * sqrt(t0.x);
            sc[4] = R0 * R0;
        }
    }
    __syncthreads();
    const double R0sq = sc[4];
    double beta = 0;
    long long k = 0;
    int restarts = 0;
    bool fresh = true;
    while (true) {
        // ---- A: w = A z (all operands local), q = w + beta q, p = z + beta p, partial p.q
        double pq_l = 0;
        for (int i = threadIdx.x; i < nr; i += blockDim.x) {
            double w = 0;
            const int k0 = s.rp[i], k1 = s.rp[i + 1];
            for (int kk = k0; kk < k1; kk++) w += s.val[kk] * s.zf[s.code[kk]];
            const double qi = fresh ? w : w + beta * s.q[i];
            const double pi = fresh ? s.zf[i] : s.zf[i] + beta * s.p[i];
            s.q[i] = qi;
            s.p[i] = pi;
            pq_l += pi * qi;
        }
        cluster_store2(cl, s.slotB, pq_l, 0.0, s.red, C, rank);
        cl.sync();
        if (warp == 0) {
            double2 t1 = cluster_slots2(s.slotB, C);
            if (lane == 0) sc[0] = sc[2] / t1.x;  // alpha = rz / pq
        }
        __syncthreads();
        fresh = false;
        k++;
        // ---- B: x += alpha p, r -= alpha q, z = M^-1 r, push z, partials r.r, r.z
        const double alpha = sc[0];
        for (int i = threadIdx.x; i < nr; i += blockDim.x) s.r[i] -= alpha * s.q[i];
        __syncthreads();
        precond(s, nblk);
        __syncthreads();
        push_halo(s, nsend, s.zf, remote_zf, NR);
        rr_l = 0;
        rz_l = 0;
        for (int i = threadIdx.x; i < nr; i += blockDim.x) {
            rr_l += s.r[i] * s.r[i];
            rz_l += s.r[i] * s.zf[i];
        }
        cluster_store2(cl, s.slotA, rr_l, rz_l, s.red, C, rank);
        cl.barrier_arrive();
        for (int i = threadIdx.x; i < nr; i += blockDim.x) s.x[i] += alpha * s.p[i];  // overlaps the barrier
        cl.barrier_wait();
        if (warp == 0) {
            double2 t2 = cluster_slots2(s.slotA, C);
            if (lane == 0) {
                sc[1] = t2.y / sc[2];  // beta = rz_new / rz
                sc[2] = t2.y;
                sc[3] = t2.x;
                sc[5] = (t2.x <= R0sq) ? 1.0 : 0.0;
            }
        }
        __syncthreads();
        beta = sc[1];
        if (sc[5] != 0.0) {
            if (restarts >= a.max_restarts) break;
            cl.sync();  // every CTA has read slotA and is done with its halo before both are rewritten
            push_halo(s, nsend, s.x, remote_zf, NR);
            cl.sync();
            for (int i = threadIdx.x; i < nr; i += blockDim.x) {  // FP64 true residual
                double acc = 0;
                for (int kk = s.rp[i]; kk < s.rp[i + 1]; kk++) {
                    const int c = s.code[kk];
                    acc += s.val[kk] * (c < NR ? s.x[c] : s.zf[c]);
                }
                s.r[i] = a.b[r_lo + i] - acc;
            }
            cl.sync();  // every CTA has read its x halo before the z pushes below overwrite it
            precond(s, nblk);
            __syncthreads();
            push_halo(s, nsend, s.zf, remote_zf, NR);
            rr_l = 0;
            rz_l = 0;
            for (int i = threadIdx.x; i < nr; i += blockDim.x) {
                rr_l += s.r[i] * s.r[i];
                rz_l += s.r[i] * s.zf[i];
            }
            cluster_store2(cl, s.slotA, rr_l, rz_l, s.red, C, rank);
            cl.sync();
            if (warp == 0) {
                double2 t3 = cluster_slots2(s.slotA, C);
                if (lane == 0) {
                    sc[2] = t3.y;
                    sc[3] = t3.x;
                    sc[5] = (t3.x <= R0sq) ? 1.0 : 0.0;
                }
            }
            __syncthreads();
            restarts++;
            if (sc[5] != 0.0) break;
            fresh = true;
        }
        if (k >= a.max_iter) break;
    }
    for (int i = threadIdx.x; i < nr; i += blockDim.x) a.x[r_lo + i] = s.x[i];
    if (rank == 0 && threadIdx.x == 0) {
        a.stats[0] = (double)k;
        a.stats[1] = sc[3];
        a.stats[2] = sqrt(R0sq);
        a.stats[3] = (double)restarts;
    }
    cl.sync();  // no CTA exits while others may still access its shared memory
}

}  // namespace

bool pcg_solve_cluster(SolverWork& w, const SolverSystem& sys, bool block_precond, const float* node_scale,
                       const float* edge_scale, int nchains, const int32_t* chain_start, const int32_t* chain_len, double tol,
                       long long max_iter, cudaStream_t s, int64_t& launches, PcgStats& st) {
    const int n = sys.n;
    const int C = kClusterCtas;
    st = PcgStats{};
    if (n <= 0) return true;
    if (n < 4 * C || n >= (1 << 16) * C / 2) return false;
    static int attr_state = 0;  // 0 unknown, 1 ok, -1 unsupported
    if (attr_state == 0) {
        cudaError_t e1 = cudaFuncSetAttribute(k_pcg_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaError_t e2 = cudaFuncSetAttribute(k_pcg_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, kClusterSmemMax);
        attr_state = (e1 == cudaSuccess && e2 == cudaSuccess) ? 1 : -1;
        cudaGetLastError();
    }
    if (attr_state < 0) return false;
    TraceSeq tr(s);
    // ---- preconditioner blocks: chain blocks (<= kBlockMax) or single rows (Jacobi)
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
    tr.mark("cluster.factors");
    // ---- halo
    const long long cn = (long long)C * n;
    w.halo_mark.ensure(cn + 1);
    w.halo_scan.ensure(cn + 1);
    CICY_CUDA(cudaMemsetAsync(w.halo_mark.get(), 0, sizeof(int32_t) * (cn + 1), s));
    k_halo_mark<<<grid_for(n), 256, 0, s>>>(n, C, w.cta_row.get(), sys.rp, sys.ci, w.halo_mark.get());
    exclusive_scan_i32(w.halo_mark.get(), w.halo_scan.get(), (int)cn, w.total.get(), w.scan_tmp, s, launches);
    launches += 5;
    int h_row[17], h_st[34], h_total = 0, h_hp[17];
    CICY_CUDA(cudaMemcpyAsync(&h_total, w.total.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaMemcpyAsync(h_row, w.cta_row.get(), sizeof(int) * (C + 1), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaMemcpyAsync(h_st, w.cta_stats.get(), sizeof(int) * 2 * (C + 1), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    w.halo_ptr.ensure(C + 1);
    k_halo_ptr<<<1, 32, 0, s>>>(n, C, w.halo_scan.get(), h_total, w.halo_ptr.get());
    launches++;
    CICY_CUDA(cudaMemcpyAsync(h_hp, w.halo_ptr.get(), sizeof(int) * (C + 1), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    int nr_max = 0, nnz_max = 0, nb_max = 0, hmax = 0;
    for (int b = 0; b < C; b++) {
        nr_max = std::max(nr_max, h_row[b + 1] - h_row[b]);
        nnz_max = std::max(nnz_max, h_st[C + 2 + b] - h_st[C + 1 + b]);
        nb_max = std::max(nb_max, h_st[b + 1] - h_st[b]);
        hmax = std::max(hmax, h_hp[b + 1] - h_hp[b]);
    }
    if (nr_max + hmax >= (1 << 16)) return false;
    // send lists
    w.send_cnt.ensure(C + 1);
    w.send_ptr.ensure(C + 1);
    CICY_CUDA(cudaMemsetAsync(w.send_cnt.get(), 0, sizeof(int32_t) * (C + 1), s));
    k_send_count<<<grid_for(cn), 256, 0, s>>>(n, C, w.cta_row.get(), w.halo_mark.get(), w.send_cnt.get());
    exclusive_scan_i32(w.send_cnt.get(), w.send_ptr.get(), C + 1, nullptr, w.scan_tmp, s, launches);
    int h_sp[17];
    CICY_CUDA(cudaMemcpyAsync(h_sp, w.send_ptr.get(), sizeof(int) * (C + 1), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaMemcpyAsync(w.send_cnt.get(), w.send_ptr.get(), sizeof(int32_t) * (C + 1), cudaMemcpyDeviceToDevice, s));
    w.send.ensure(std::max(h_total, 1));
    k_send_fill<<<grid_for(cn), 256, 0, s>>>(n, C, w.cta_row.get(), w.halo_mark.get(), w.halo_scan.get(), w.halo_ptr.get(),
                                            w.send_cnt.get(), w.send.get());
    w.code.ensure(std::max(sys.nnz, 1));
    k_halo_codes<<<grid_for(n), 256, 0, s>>>(n, C, nr_max, w.cta_row.get(), sys.rp, sys.ci, w.halo_scan.get(), w.halo_ptr.get(),
                                            w.code.get());
    launches += 4;
    CICY_CUDA(cudaStreamSynchronize(s));
    tr.mark("cluster.halo");
    int smax = 0;
    for (int b = 0; b < C; b++) smax = std::max(smax, h_sp[b + 1] - h_sp[b]);
    const size_t smem = smem_layout(nr_max, nnz_max, nb_max, hmax, smax, nullptr, nullptr);
    if (smem > (size_t)kClusterSmemMax) return false;
    w.stats.ensure(4);
    CICY_CUDA(cudaMemsetAsync(w.stats.get(), 0, sizeof(double) * 4, s));
    ClusterArgs a{};
    a.n = n; a.C = C;
    a.rp = sys.rp; a.code = w.code.get(); a.val = sys.val; a.b = sys.b; a.x = sys.x;
    a.lfac = w.lfac.get(); a.ipiv = w.ipiv.get();
    a.cta_row = w.cta_row.get(); a.cta_blk = w.cta_stats.get(); a.blk_row = w.blk_row.get();
    a.send_ptr = w.send_ptr.get(); a.send = w.send.get();
    a.nr_max = nr_max; a.nnz_max = nnz_max; a.nb_max = nb_max; a.h_max = hmax; a.s_max = smax;
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
    tr.mark("cluster.layout");
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, (void*)k_pcg_cluster, &cfg) != cudaSuccess || nclusters < 1) {
        cudaGetLastError();
        return false;
    }
    tr.mark("cluster.occupancy");
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
