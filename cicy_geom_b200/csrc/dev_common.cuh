// Device-side building blocks shared by all kernels of libcicy_b200:
// error plumbing, grow-only device buffers, exclusive scan, a stable LSD radix
// sort of (u64 key, u32 value) pairs, a segmented sort for short segments and
// a bounded-spin grid barrier for persistent kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/cicy_b200.h"

namespace cicy {

constexpr int kWarp = 32;
// Upper bound on busy-wait polls of a grid barrier; far above any real wait
// (a co-resident cooperative launch reaches the barrier in microseconds).
constexpr long long kSpinLimit = 1LL << 28;
// Device status codes written by kernels (kept in DeviceStatus::code).
enum DevErr : int { DEV_OK = 0, DEV_TIMEOUT = 1, DEV_CAPACITY = 2, DEV_INPUT = 3, DEV_ZERO_DIAG = 4 };

struct Fail {
    cicy_status status;
    std::string msg;
};

#define CICY_CUDA(call)                                                                         \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            throw ::cicy::Fail{CICY_E_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

#define CICY_LAUNCH_CHECK() CICY_CUDA(cudaGetLastError())

// Grow-only device buffer; owns its allocation (freed on destruction, moves
// transfer it, copies are not allowed).
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t cap = 0;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), cap(o.cap), n(o.n) {
        o.p = nullptr;
        o.cap = o.n = 0;
    }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            cap = o.cap;
            n = o.n;
            o.p = nullptr;
            o.cap = o.n = 0;
        }
        return *this;
    }
    ~DBuf() { release(); }
    void ensure(size_t need) {
        n = need;
        if (need <= cap) return;
        if (p) cudaFree(p);
        p = nullptr;
        size_t c = need + need / 4 + 256;
        CICY_CUDA(cudaMalloc(&p, c * sizeof(T)));
        cap = c;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = n = 0;
    }
    T* get() const { return p; }
};

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// Exclusive scan of int32 counts (out may alias in). `total` (device) gets the sum.
void exclusive_scan_i32(const int32_t* in, int32_t* out, int n, int32_t* total, DBuf<int32_t>& tmp, cudaStream_t s,
                        int64_t& launches);
// Exclusive scan of int64 values.
void exclusive_scan_i64(const int64_t* in, int64_t* out, int n, int64_t* total, DBuf<int64_t>& tmp, cudaStream_t s,
                        int64_t& launches);

// Stable LSD radix sort of n pairs by the low `bits` bits of the key.
// Sorts (keys, vals) in place using (keys_tmp, vals_tmp) as ping-pong space.
struct RadixScratch {
    DBuf<uint64_t> keys_tmp;
    DBuf<uint32_t> vals_tmp;
    DBuf<int32_t> hist;
    DBuf<int32_t> scan_tmp;
};
void radix_sort_pairs(uint64_t* keys, uint32_t* vals, int n, int bits, RadixScratch& rs, cudaStream_t s, int64_t& launches);

// Sorts each segment [ptr[i], ptr[i+1]) of `keys` ascending (keys unique within a
// segment) into `out`, carrying nothing else: out holds the sorted keys.
// Segments longer than kSegSortMax set the capacity flag in *status.
constexpr int kSegSortMax = 8192;
void segmented_sort_u32(const int32_t* ptr, int n_seg, const uint32_t* keys, uint32_t* out, int32_t* large_list,
                        int32_t* large_count, int* status, cudaStream_t s, int64_t& launches);

int bits_for(uint64_t max_value);

// ---------------------------------------------------------------------------
// Grid-wide barrier for a cooperative (co-resident) launch with a bounded spin.
// Returns false, with *err set, if the wait gave up.
struct GridBarrier {
    unsigned int* count;
    unsigned int* gen;
    long long limit = kSpinLimit;  // polls before the wait gives up
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_sync(GridBarrier b, unsigned int nblocks, int* err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int g = ld_acquire_u32(b.gen);
        __threadfence();
        unsigned int arrived = atomicAdd(b.count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(b.count, 0u);
            __threadfence();
            atomicAdd(b.gen, 1u);
        } else {
            long long spins = 0;
            while (ld_acquire_u32(b.gen) == g) {
                if (++spins > b.limit || *((volatile int*)err) != 0) {
                    atomicCAS(err, 0, (int)DEV_TIMEOUT);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *((volatile int*)err) == 0;
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace cicy
