// Allocation-free variant of the FP64 Jacobi-PCG solve (cicy_jacobi_pcg_static).
//
// Some callers cannot allocate device memory at solve time: code that must not
// let cudaMalloc/cudaFree synchronize the device or take the allocator's lock
// in the middle of a time-stepped loop that other streams share, and hosts that
// have handed all device memory to their own pool and forbid allocations by
// plug-ins.  For them this entry point takes the system, right-hand side and
// solution vector in the caller's device memory and keeps all of its scratch
// (CG vectors, per-CTA partial sums, the grid-barrier words, the result words)
// in one fixed file-scope device array.  The array is part of the loaded
// library: every GPU that loads it holds kStaticBytes (about 5.3 MB) until the
// process exits.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>

#include "cicy_internal.h"
#include "csr_check.cuh"
#include "solver.cuh"

namespace cicy {

namespace {

constexpr int kStaticMaxRows = 1 << 17;  // largest system (rows) the static scratch holds
constexpr int kStaticMaxCtas = 4096;

// byte offsets inside the static array (256-byte aligned segments)
constexpr size_t align256(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t kVecBytes = align256(sizeof(double) * kStaticMaxRows);
constexpr size_t kOffR = 0;
constexpr size_t kOffZ = kOffR + kVecBytes;
constexpr size_t kOffP = kOffZ + kVecBytes;
constexpr size_t kOffQ = kOffP + kVecBytes;
constexpr size_t kOffMinv = kOffQ + kVecBytes;
constexpr size_t kOffPart = kOffMinv + kVecBytes;
constexpr size_t kOffStats = kOffPart + align256(sizeof(double) * 4 * kStaticMaxCtas);
constexpr size_t kOffBarrier = kOffStats + 256;
constexpr size_t kOffCtaRow = kOffBarrier + 256;
constexpr size_t kStaticBytes = kOffCtaRow + align256(sizeof(int32_t) * (kStaticMaxCtas + 1));

static __device__ __align__(256) unsigned char g_pcg_scratch[kStaticBytes];

std::mutex g_mu;
unsigned char* g_scratch_addr[64] = {nullptr};  // device address of g_pcg_scratch, per device

// Device address of the static array on the current device, looked up on the
// first call on each device and kept for the life of the process (a device
// reset or a re-created primary context invalidates it).
cicy_status scratch_address(int dev, unsigned char** out, std::string& err) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev < 0 || dev >= 64) {
        err = "device index out of range";
        return CICY_E_INPUT;
    }
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_pcg_scratch);
        if (e != cudaSuccess || !p) {
            err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return CICY_E_DEVICE;
        }
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[dev];
    return CICY_OK;
}

// Structure check of the caller's CSR before any kernel uses its indices as
// addresses: every read stays within row_ptr[n + 1] and col_ind[nnz].
__global__ void k_check_structure(int n, int nnz, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                  int* __restrict__ flags) {
    const int f = check_structure_part(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, n, nnz, rp, ci, 0, nullptr,
                                       nullptr);
    if (f) atomicOr(flags, f);
}

__global__ void k_diag_inverse(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                               double* __restrict__ minv, int* __restrict__ bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++)
            if (ci[k] == i) d += v[k];
        if (!(d != 0.0)) atomicExch(bad, (int)DEV_ZERO_DIAG);
        minv[i] = 1.0 / d;
    }
}

__global__ void k_uniform_rows(int nb, int n, int32_t* __restrict__ cta_row) {
    for (int b = threadIdx.x; b <= nb; b += blockDim.x) cta_row[b] = (int)((long long)b * n / nb);
}

}  // namespace

}  // namespace cicy

extern "C" cicy_status cicy_jacobi_pcg_static(int32_t n, int32_t nnz, const int32_t* row_ptr, const int32_t* col_ind,
                                               const double* values, const double* b, double* x, double tol, int64_t max_iter,
                                               void* stream, int64_t* iterations, double* rel_residual) {
    using namespace cicy;
    std::string err;
    if (n <= 0 || nnz < n || !row_ptr || !col_ind || !values || !b || !x || !(tol > 0) || max_iter <= 0) {
        set_host_error("cicy_jacobi_pcg_static: invalid arguments");
        return CICY_E_INPUT;
    }
    if (n > kStaticMaxRows) {
        set_host_error("cicy_jacobi_pcg_static: " + std::to_string(n) + " rows exceed the static scratch limit of " +
                       std::to_string(kStaticMaxRows) + " rows");
        return CICY_E_CAPACITY;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        set_host_error("cicy_jacobi_pcg_static: no current CUDA device");
        return CICY_E_DEVICE;
    }
    unsigned char* base = nullptr;
    cicy_status st = scratch_address(dev, &base, err);
    if (st != CICY_OK) {
        set_host_error("cicy_jacobi_pcg_static: " + err);
        return st;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int sms = 0, coop = 0;
    for (auto q : {std::make_pair(&sms, cudaDevAttrMultiProcessorCount), std::make_pair(&coop, cudaDevAttrCooperativeLaunch)}) {
        const cudaError_t e = cudaDeviceGetAttribute(q.first, q.second, dev);
        if (e != cudaSuccess) {
            set_host_error(std::string("cicy_jacobi_pcg_static: cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
            return CICY_E_DEVICE;
        }
    }
    if (!coop || sms <= 0) {
        set_host_error("cicy_jacobi_pcg_static: device lacks cooperative launch");
        return CICY_E_DEVICE;
    }
    double* r = reinterpret_cast<double*>(base + kOffR);
    double* z = reinterpret_cast<double*>(base + kOffZ);
    double* p = reinterpret_cast<double*>(base + kOffP);
    double* q = reinterpret_cast<double*>(base + kOffQ);
    double* minv = reinterpret_cast<double*>(base + kOffMinv);
    double* part = reinterpret_cast<double*>(base + kOffPart);
    double* stats = reinterpret_cast<double*>(base + kOffStats);
    unsigned int* bar = reinterpret_cast<unsigned int*>(base + kOffBarrier);
    int* status = reinterpret_cast<int*>(base + kOffBarrier + 64);
    int* structure = reinterpret_cast<int*>(base + kOffBarrier + 128);
    int32_t* cta_row = reinterpret_cast<int32_t*>(base + kOffCtaRow);
    try {
        int64_t launches = 0;
        const int cap = max_coop_blocks_jacobi_fp64(sms);
        const int nb = std::max(1, std::min({cap, sms, ceil_div(n, 256), kStaticMaxCtas}));
        // the array keeps the previous call's contents: reset what must start at zero
        // (stats, barrier, status and structure words)
        CICY_CUDA(cudaMemsetAsync(base + kOffStats, 0, 256 + 256, s));
        k_check_structure<<<std::min(ceil_div(std::max(n, nnz), 256), 148 * 8), 256, 0, s>>>(n, nnz, row_ptr, col_ind, structure);
        CICY_LAUNCH_CHECK();
        int hflags = 0;
        CICY_CUDA(cudaMemcpyAsync(&hflags, structure, sizeof(int), cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaStreamSynchronize(s));
        if (hflags) {
            set_host_error("cicy_jacobi_pcg_static: " + structure_error(hflags));
            return CICY_E_INPUT;
        }
        k_diag_inverse<<<std::min(ceil_div(n, 256), 148 * 8), 256, 0, s>>>(n, row_ptr, col_ind, values, minv, status);
        k_residual<<<std::min(ceil_div(n, 256), 148 * 8), 256, 0, s>>>(n, row_ptr, col_ind, values, x, b, r);
        k_uniform_rows<<<1, 256, 0, s>>>(nb, n, cta_row);
        CICY_LAUNCH_CHECK();
        PcgArgs a{};
        a.n = n;
        a.rp = row_ptr; a.ci = col_ind; a.val = values;
        a.b = b; a.x = x; a.r = r; a.z = z; a.p = p; a.q = q;
        a.minv = minv;
        a.cta_row = cta_row;
        a.partA = part; a.partB = part + 2 * nb;
        a.stats = stats;
        a.bar = GridBarrier{bar, bar + 1};
        a.err = status;
        a.tol = tol;
        a.max_iter = max_iter;
        a.max_restarts = 24;
        a.inner_drop = 0.0;
        launch_pcg_jacobi_fp64(a, nb, s);
        double hs[4];
        int hstatus = 0;
        CICY_CUDA(cudaMemcpyAsync(hs, stats, sizeof(hs), cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaMemcpyAsync(&hstatus, status, sizeof(int), cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaStreamSynchronize(s));
        (void)launches;
        if (hstatus == DEV_TIMEOUT) {
            set_host_error("cicy_jacobi_pcg_static: a bounded device wait gave up");
            return CICY_E_TIMEOUT;
        }
        if (hstatus == DEV_ZERO_DIAG) {
            set_host_error("cicy_jacobi_pcg_static: zero on the diagonal");
            return CICY_E_ZERO_DIAGONAL;
        }
        if (hstatus != 0) {
            set_host_error("cicy_jacobi_pcg_static: device status " + std::to_string(hstatus));
            return CICY_E_INTERNAL;
        }
        if (iterations) *iterations = (int64_t)hs[0];
        if (rel_residual) *rel_residual = hs[2] > 0 ? std::sqrt(hs[1]) / (hs[2] / tol) : 0.0;
    } catch (const Fail& f) {
        set_host_error("cicy_jacobi_pcg_static: " + f.msg);
        return f.status;
    }
    return CICY_OK;
}
