// Sparse matrix-vector product y = A x in full CSR, FP64: the SpMV of the DEA
// conjugate gradient (spM_V_SSS, Direct_Electrifying.cpp:1680-1735, on the
// symmetric-stored form there).  DEA rows are short (a CNT node couples to its
// two chain neighbours and a few junctions, ~3-4 entries), so one thread owns a
// row: a warp then streams one contiguous stretch of col_ind/values (each 32 B
// sector is fetched once through L1), reads row_ptr coalesced and gathers x,
// whose entries are mostly neighbours along the chains (L2 hits).  HBM-bound:
// algorithmic bytes per call = 12 nnz + 4 (n + 1) + 8 n (x) + 8 n (y).
#include "cicy_internal.h"
#include "dev_common.cuh"

namespace cicy {
namespace {

__global__ void __launch_bounds__(256) k_spmv_csr(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                                  const double* __restrict__ v, const double* __restrict__ x, double* __restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int b = __ldg(&rp[i]), e = __ldg(&rp[i + 1]);
        double s = 0;
        int k = b;
        for (; k + 1 < e; k += 2) {
            const int c0 = __ldg(&ci[k]), c1 = __ldg(&ci[k + 1]);
            const double v0 = __ldg(&v[k]), v1 = __ldg(&v[k + 1]);
            s += v0 * __ldg(&x[c0]);
            s += v1 * __ldg(&x[c1]);
        }
        if (k < e) s += __ldg(&v[k]) * __ldg(&x[__ldg(&ci[k])]);
        __stcs(&y[i], s);
    }
}

}  // namespace
}  // namespace cicy

extern "C" cicy_status cicy_spmv_csr(int32_t n, const int32_t* row_ptr, const int32_t* col_ind, const double* values, const double* x,
                                     double* y, void* stream) {
    if (n < 0 || (n > 0 && (!row_ptr || !col_ind || !values || !x || !y))) {
        cicy::set_host_error("cicy_spmv_csr: invalid arguments");
        return CICY_E_INPUT;
    }
    if (n == 0) return CICY_OK;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long blocks = std::min<long long>((n + 255) / 256, (long long)sms * 8);
    cicy::k_spmv_csr<<<(int)blocks, 256, 0, (cudaStream_t)stream>>>(n, row_ptr, col_ind, values, x, y);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        cicy::set_host_error(std::string("cicy_spmv_csr: ") + cudaGetErrorString(e));
        return CICY_E_DEVICE;
    }
    return CICY_OK;
}
