// Preconditioned CG for DEA systems (see solver.cu).
#pragma once

#include "dev_common.cuh"

namespace cicy {

constexpr int kBlockMax = 32;  // largest block of the chain block-Jacobi preconditioner
constexpr int kClusterCtas = 16;                // CTAs of the cluster-resident solver (non-portable cluster size)
constexpr int kClusterSmemMax = 232448 - 1024;  // dynamic shared memory per CTA it may use
enum PrecondKind : int { PRECOND_KIND_JACOBI = 0, PRECOND_KIND_BLOCK = 1 };

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
    const float* val32;
    const double* b;
    double* x;
    double* r;
    double *z, *p, *q;
    float *z32, *p32, *q32;
    const double* minv;
    const float* minv32;
    const double* tinv;
    const float* tinv32;
    const int32_t *row_off, *row_base, *row_m;
    const int32_t* cta_row;
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
    bool cluster = false;
    double seconds = 0;
};

struct SolverWork {
    DBuf<double> r, z, p, q, minv, tinv, part, stats, lfac, ipiv;
    DBuf<float> z32, p32, q32, val32, minv32, tinv32;
    DBuf<int32_t> is_start, start_scan, blk_row, blk_msq, blk_off, row_off, row_base, row_m, cta_row, total, scan_tmp, cta_stats;
    DBuf<int32_t> halo_mark, halo_scan, halo_ptr, send_cnt, send_ptr;
    DBuf<unsigned long long> send;
    DBuf<uint16_t> code;
    DBuf<unsigned int> barrier;
    int n_blocks = 0, block_entries = 0;
};

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

void pcg_solve(SolverWork& w, const SolverSystem& sys, int precond, bool mixed, double tol, long long max_iter, int num_sms,
               int* status, cudaStream_t s, int64_t& launches, PcgStats& st);

}  // namespace cicy
