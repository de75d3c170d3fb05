// Preconditioned CG for DEA systems (see solver.cu).
#pragma once

#include <cuda_bf16.h>

#include <vector>

#include "dev_common.cuh"

namespace cicy {

constexpr int kBlockMax = 32;  // largest block of the chain block-Jacobi preconditioner
constexpr int kClusterCtas = 16;                // CTAs of the cluster-resident solver (non-portable cluster size)
constexpr int kClusterSmemMax = 232448 - 1024;  // dynamic shared memory per CTA it may use
enum PrecondKind : int { PRECOND_KIND_JACOBI = 0, PRECOND_KIND_BLOCK = 1, PRECOND_KIND_SPAI = 2 };

// A free-node system in full symmetric CSR (diagonal included).
struct SolverSystem {
    int n = 0, nnz = 0;
    const int32_t* rp = nullptr;
    const int32_t* ci = nullptr;
    const double* val = nullptr;
    const double* diag = nullptr;
    const double* b = nullptr;
    double* x = nullptr;  // in: initial guess, out: solution
};

struct PcgArgs {
    int n;
    const int32_t* rp;
    const int32_t* ci;
    const double* val;
    const float* val32;   // mixed: conductances g = -a off the diagonal, 0 on it
    const float* rs32;    // mixed: row sums of A (the conductance to prescribed nodes)
    const double* b;
    double* x;
    double* r;
    double *z, *p, *q;
    double* p2;           // mixed: second buffer of the search direction
    const double* minv;
    const float* minv32;
    const double* tinv;
    const float* tinv32;
    const int32_t *row_off, *row_base, *row_m;
    const int32_t* cta_row;
    const float* ew;  // learned weights of the couplings outside the blocks (SPAI), 0 elsewhere
    double* y;        // SPAI: T^-1 r
    double* u;        // SPAI: E_w T^-1 r
    double* partA;
    double* partB;
    double* stats;
    GridBarrier bar;
    int* err;
    double tol;
    long long max_iter;
    int max_restarts;
    double inner_drop;
};

struct PcgStats {
    long long iterations = 0;
    int restarts = 0;
    int ctas = 0;
    int levels = 0;  // multigrid levels (0: one-level preconditioner)
    bool cluster = false;
    double seconds = 0;
};

// ---- chain-aggregation multigrid (solver_mg.cu) ----
constexpr int kMgMaxLevels = 16;
constexpr int kMgDenseMax = 128;  // coarsest levels up to this size get a dense inverse

// One level as the solve kernel sees it.  Level 0 is the system's own CSR
// (diagonal included); levels >= 1 hold off-diagonal CSR plus `diag`.
struct MgLevel {
    int n;
    const int32_t* rp;
    const int32_t* ci;
    const double* val;
    const double* diag;
    const double* l1inv;
    const int32_t* agg;   // row -> aggregate on level l+1 (coarsest: nullptr)
    const int32_t* mptr;  // aggregate J of level l+1 -> its rows of level l: midx[mptr[J] .. mptr[J+1])
    const int32_t* midx;
    const int32_t* cagg;    // per nonzero: aggregate of its column (levels < coarsest)
    const int32_t* ra_ptr;  // rows of P^T A_l, one per aggregate of level l+1 (levels 1 .. coarsest-1)
    const int32_t* ra_col;
    const double* ra_val;
    double* r;
    double* z;
    double* zf;
};

struct MgWork {
    struct Lvl {
        int n = 0, nnz = 0;
        const int32_t* rp_ptr = nullptr;
        const int32_t* ci_ptr = nullptr;
        const double* val_ptr = nullptr;
        DBuf<int32_t> rp, ci, agg, mptr, midx, cagg, ra_ptr, ra_col;
        DBuf<double> val, diag, l1inv, rs, r, z, zf, ra_val;
        // fused rows for the clustered solve kernel: restriction into level l+1 (members on
        // r_l, P^T A_l on z_l) and prolongation-smoother rows of level l (A_l on z_l and on P zc)
        DBuf<int32_t> rr_ptr, rr_col, pq_ptr, pq_col;
        DBuf<double> rr_val, pq_val;
        DBuf<double> r_cl, z_cl, zf_cl;  // per-cluster copies of the levels each cluster solves alone
    };
    std::vector<Lvl> L;
    std::vector<MgLevel> host_lv;
    DBuf<MgLevel> dev_lv;
    DBuf<double> cinv, z0, wtmp, sval, gj_panel;
    DBuf<unsigned long long> gj_sync;  // grid Gauss-Jordan: barrier counter, largest diagonal (bits)
    DBuf<int32_t> gj_err;
    DBuf<unsigned long long> bar;
    DBuf<uint64_t> keys;
    DBuf<uint32_t> vals;
    DBuf<int32_t> flag, pos, head, uidx, mate, best, rep, total, scan_tmp, long_rows;
    RadixScratch radix;
    // smoothed level-1 prolongator (fused hierarchy): Q = P - w D^-1 A_1 P and the sparse
    // products built from it (T = A_1 P, Q^T, W = A_1 Q, Q^T A_1), plus the gather scratch
    struct Smoothed {
        DBuf<int32_t> tp, tc, qtp, qti, wp, wc, ap, ac, seg, ulen, longr;
        DBuf<double> tv, qv, qpv, qtv, wv, wpv, av, y, v, gv, gv2, ov, ov2;
        DBuf<uint64_t> gkey, okey;
    } sa;
    int levels = 0;
    bool dense = false;
    bool fused = false;  // fused rows built (build_mg_hierarchy with fused = true)
    bool smooth = true;  // with fused: level 1's prolongator smoothed (coarsen_smoothed)
    DBuf<int32_t> cl_fail;
    DBuf<unsigned char> sec_lv;  // device descriptors of the clustered kernel
};

struct SolverWork {
    DBuf<double> r, z, p, p2, q, minv, tinv, part, stats, lfac, ipiv;
    DBuf<float> val32, rs32, minv32, tinv32;
    DBuf<int32_t> is_start, start_scan, blk_row, blk_msq, blk_off, row_off, row_base, row_m, cta_row, total, scan_tmp, cta_stats;
    DBuf<int32_t> halo_mark, halo_scan, halo_ptr, send_cnt, send_ptr;
    DBuf<unsigned long long> send;
    DBuf<uint16_t> code;
    DBuf<unsigned int> barrier;
    int n_blocks = 0;
    long long spin_limit = kSpinLimit;  // polls of a grid-barrier wait before it gives up (DEV_TIMEOUT)
    MgWork mg;
    DBuf<double> y, u;
};

// ---- learned preconditioner (learned.cu) ----
struct GnnState {
    int n = 0, nnz = 0;
    const int32_t* rp = nullptr;
    const int32_t* ci = nullptr;
    const double* val = nullptr;
    SolverWork sw;  // chain blocks of the system
    DBuf<int> status;
    DBuf<double> diag, logd, ms, vr, vy, vu, vz, vq, vd, vl, dw, part, coef;
    DBuf<float> deg, f, invdeg, lc, jf, A0, HW, w, dout, dH0, dH1, dA, dM, dG;
    DBuf<float> A[3];
    DBuf<__nv_bfloat16> H[4], G[3];
    DBuf<int32_t> chain, blk, tr;
    DBuf<uint8_t> offb;
};

int gnn_param_count();
// Features, chain blocks and buffers for one system (full symmetric CSR, columns ascending).
void gnn_set_system(GnnState& g, int n, int nnz, const int32_t* rp, const int32_t* ci, const double* val, int nchains,
                    const int32_t* cs, const int32_t* cl, cudaStream_t s, int64_t& launches);
// Network forward: g.w holds the weight of every coupling outside the blocks (0 elsewhere).
void gnn_forward(GnnState& g, const float* params, cudaStream_t s, int64_t& launches);
// Mean loss over K probe vectors (K x n, FP64) and its gradient (overwrites grad).
double gnn_loss_grad(GnnState& g, const float* params, int K, const double* probes, float* grad, cudaStream_t s, int64_t& launches);
void gnn_smooth_probes(GnnState& g, int K, double* u, int sweeps, cudaStream_t s, int64_t& launches);
void gnn_adam(float* p, const float* grad, float* m, float* v, int n, int step, float lr, cudaStream_t s);

__global__ void k_residual(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                           const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ r);
__global__ void k_fill_ones(int n, int32_t* __restrict__ a);

// Block-Jacobi over CNT chains (chains given as free-node ranges), optionally with
// learned per-node / per-edge scalings (nullptr: exact blocks).
void build_block_preconditioner(SolverWork& w, const SolverSystem& sys, int nchains, const int32_t* chain_start,
                                const int32_t* chain_len, const float* node_scale, const float* edge_scale, bool mixed,
                                cudaStream_t s, int64_t& launches);

void launch_block_marks(int nchains, const int32_t* chain_start, const int32_t* chain_len, int32_t* is_start, cudaStream_t s);
void launch_block_fill(int n, const int32_t* is_start, const int32_t* start_scan, int32_t* blk_row, cudaStream_t s);
void launch_cta_rows(int nb_cta, int n, const int32_t* is_start, int32_t* cta_row, cudaStream_t s);
void launch_jacobi_fp64(int n, const double* diag, double* minv, cudaStream_t s);
int max_coop_blocks_jacobi_fp64(int num_sms);
void launch_pcg_jacobi_fp64(PcgArgs& a, int nb, cudaStream_t s);

// Cluster-resident PCG (solver_cluster.cu).  Returns false, without touching x,
// when the system does not fit one cluster's shared memory.
bool pcg_solve_cluster(SolverWork& w, const SolverSystem& sys, bool block_precond, const float* node_scale,
                       const float* edge_scale, int nchains, const int32_t* chain_start, const int32_t* chain_len, double tol,
                       long long max_iter, cudaStream_t s, int64_t& launches, PcgStats& st);

// Multigrid hierarchy over the chain blocks of build_block_preconditioner (which
// must have run on the same system), then the MG-preconditioned CG solve.
// fused: also build the fused restriction / prolongation rows the clustered grid kernel
// reads (systems above the single-cluster size).
void build_mg_hierarchy(SolverWork& w, const SolverSystem& sys, cudaStream_t s, int64_t& launches, bool fused = false, bool smooth = true,
                        int* status = nullptr);
// Whether pcg_solve_mg takes the clustered grid kernel for a system of n rows (build the
// hierarchy with fused = this).
bool mg_fused_path(int n, bool allow_cluster);
// allow_cluster: one 16-CTA cluster with hardware barriers when it fits, else the grid-wide kernel.
void pcg_solve_mg(SolverWork& w, const SolverSystem& sys, double tol, long long max_iter, bool allow_cluster, int num_sms, int* status,
                  cudaStream_t s, int64_t& launches, PcgStats& st);

// precond PRECOND_KIND_SPAI needs the block preconditioner and `ew` (learned weights per entry).
// Batched MG solves (solver_mg.cu): device arrays of each system; chains partition the rows.
struct MgBatchInput {
    int n, nnz, nchains;
    const int32_t *rp, *ci;
    const double *val, *b, *x0;
    double* x;
    const int32_t *cs, *cl;
};
struct MgBatch;
MgBatch* mg_batch_build(const std::vector<MgBatchInput>& in, double tol, long long iter_factor, cudaStream_t s, int64_t& launches);
void mg_batch_enqueue(MgBatch* b, cudaStream_t s);
// per system: iterations, |r|^2 of the last test, tol |r0|, restarts
void mg_batch_stats(MgBatch* b, std::vector<double>& stats, cudaStream_t s);
int mg_batch_clusters(const MgBatch* b);
void mg_batch_free(MgBatch* b);

void pcg_solve(SolverWork& w, const SolverSystem& sys, int precond, bool mixed, double tol, long long max_iter, int num_sms,
               int* status, cudaStream_t s, int64_t& launches, PcgStats& st, const float* ew = nullptr);

}  // namespace cicy
