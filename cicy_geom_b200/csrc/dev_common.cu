// Scan, radix sort and segmented sort kernels (see dev_common.cuh).
#include "dev_common.cuh"

namespace cicy {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <class T>
__device__ T block_exclusive_sum(T v, T* smem_warp, T& block_total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    T incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) smem_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        T w = lane < nw ? smem_warp[lane] : T(0);
        T wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            T t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < nw) smem_warp[lane] = wi - w;
        if (lane == nw - 1) smem_warp[32] = wi;
    }
    __syncthreads();
    T res = smem_warp[wid] + incl - v;
    block_total = smem_warp[32];
    __syncthreads();
    return res;
}

template <class T>
__global__ void k_scan_reduce(const T* __restrict__ in, int n, T* __restrict__ bsum) {
    __shared__ T sw[33];
    long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    T s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        long long j = base + i;
        if (j < n) s += in[j];
    }
    T tot;
    block_exclusive_sum<T>(s, sw, tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

template <class T>
__global__ void k_scan_blocks(T* bsum, int nb, T* total) {
    __shared__ T sw[33];
    __shared__ T carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += blockDim.x) {
        int j = base + threadIdx.x;
        T v = j < nb ? bsum[j] : T(0);
        T tot;
        T ex = block_exclusive_sum<T>(v, sw, tot);
        if (j < nb) bsum[j] = ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <class T>
__global__ void k_scan_apply(const T* in, T* out, int n, const T* __restrict__ bsum) {
    __shared__ T sw[33];
    long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    T v[kScanItems];
    T s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        long long j = base + i;
        v[i] = j < n ? in[j] : T(0);
        s += v[i];
    }
    T tot;
    T ex = block_exclusive_sum<T>(s, sw, tot) + bsum[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        long long j = base + i;
        if (j < n) out[j] = ex;
        ex += v[i];
    }
}

// Scans of at most kScanSmallMax items in one launch: each of 1,024 threads holds a contiguous
// chunk of up to 16 items in registers (so out may alias in), one block-wide exclusive sum.
constexpr int kScanSmallItems = 16;
constexpr int kScanSmallMax = 1024 * kScanSmallItems;
template <class T>
__global__ void __launch_bounds__(1024) k_scan_small(const T* in, T* out, int n, T* total) {
    __shared__ T sw[33];
    const int ch = (n + 1023) / 1024;
    const int lo = min(n, (int)threadIdx.x * ch), hi = min(n, lo + ch);
    T v[kScanSmallItems];
    T s = 0;
#pragma unroll
    for (int i = 0; i < kScanSmallItems; i++) {
        v[i] = lo + i < hi ? in[lo + i] : T(0);
        s += v[i];
    }
    T tot;
    T ex = block_exclusive_sum<T>(s, sw, tot);
#pragma unroll
    for (int i = 0; i < kScanSmallItems; i++)
        if (lo + i < hi) {
            out[lo + i] = ex;
            ex += v[i];
        }
    if (threadIdx.x == 0 && total) *total = tot;
}

template <class T>
void exclusive_scan_impl(const T* in, T* out, int n, T* total, DBuf<T>& tmp, cudaStream_t s, int64_t& launches) {
    if (n <= 0) {
        if (total) CICY_CUDA(cudaMemsetAsync(total, 0, sizeof(T), s));
        return;
    }
    if (n <= kScanSmallMax) {
        k_scan_small<T><<<1, 1024, 0, s>>>(in, out, n, total);
        launches++;
        CICY_LAUNCH_CHECK();
        return;
    }
    int nb = ceil_div(n, kScanTile);
    tmp.ensure(nb + 1);
    k_scan_reduce<T><<<nb, kScanThreads, 0, s>>>(in, n, tmp.get());
    k_scan_blocks<T><<<1, 1024, 0, s>>>(tmp.get(), nb, total);
    k_scan_apply<T><<<nb, kScanThreads, 0, s>>>(in, out, n, tmp.get());
    launches += 3;
    CICY_LAUNCH_CHECK();
}

// ---------------- radix sort ----------------
constexpr int kRadixThreads = 256;            // 8 warps
constexpr int kRadixWarpItems = 256;          // items per warp per tile
constexpr int kRadixTile = kRadixWarpItems * (kRadixThreads / 32);  // 2048

__global__ void k_radix_hist(const uint64_t* __restrict__ keys, int n, int shift, int n_tiles, int32_t* __restrict__ hist) {
    __shared__ int32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * kRadixTile;
    for (int i = threadIdx.x; i < kRadixTile; i += kRadixThreads) {
        long long j = base + i;
        if (j < n) atomicAdd(&h[(keys[j] >> shift) & 0xff], 1);
    }
    __syncthreads();
    hist[(long long)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void k_radix_scatter(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint64_t* __restrict__ kout,
                                uint32_t* __restrict__ vout, int n, int shift, int n_tiles, const int32_t* __restrict__ offs) {
    __shared__ int32_t wcnt[8][256];
    __shared__ int32_t gofs[256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < 8 * 256; i += kRadixThreads) (&wcnt[0][0])[i] = 0;
    gofs[threadIdx.x] = offs[(long long)threadIdx.x * n_tiles + blockIdx.x];
    __syncthreads();
    const long long wbase = (long long)blockIdx.x * kRadixTile + (long long)w * kRadixWarpItems;
    // pass 1: per-warp digit counts
    for (int r = 0; r < kRadixWarpItems / 32; r++) {
        long long j = wbase + r * 32 + lane;
        if (j < n) atomicAdd(&wcnt[w][(kin[j] >> shift) & 0xff], 1);
    }
    __syncthreads();
    // exclusive prefix over warps, per digit (thread = digit)
    {
        int d = threadIdx.x;
        int acc = 0;
        for (int ww = 0; ww < 8; ww++) {
            int c = wcnt[ww][d];
            wcnt[ww][d] = acc;
            acc += c;
        }
    }
    __syncthreads();
    // pass 2: stable placement, rounds in order
    for (int r = 0; r < kRadixWarpItems / 32; r++) {
        long long j = wbase + r * 32 + lane;
        bool valid = j < n;
        unsigned vmask = __ballot_sync(0xffffffffu, valid);
        if (!vmask) break;
        uint64_t k = valid ? kin[j] : 0;
        uint32_t v = valid ? vin[j] : 0;
        int d = (int)((k >> shift) & 0xff);
        unsigned peers = __match_any_sync(0xffffffffu, valid ? d : 256 + lane);
        peers &= vmask;
        unsigned lt = (1u << lane) - 1u;
        int rank = __popc(peers & lt);
        int pos = 0;
        if (valid) pos = gofs[d] + wcnt[w][d] + rank;
        __syncwarp();
        if (valid && (peers & lt) == 0) wcnt[w][d] += __popc(peers);
        __syncwarp();
        if (valid) {
            kout[pos] = k;
            vout[pos] = v;
        }
    }
}

// ---------------- segmented sort ----------------
__global__ void k_segsort_warp(const int32_t* __restrict__ ptr, int n_seg, const uint32_t* __restrict__ keys,
                               uint32_t* __restrict__ out, int32_t* large_list, int32_t* large_count, int* status) {
    const int lane = threadIdx.x & 31;
    long long wg = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long sgi = wg; sgi < n_seg; sgi += nw) {
        int b = ptr[sgi], e = ptr[sgi + 1], len = e - b;
        if (len <= 1) {
            if (len == 1 && lane == 0) out[b] = keys[b];
            continue;
        }
        if (len > 32) {
            if (lane == 0) {
                if (len > kSegSortMax) atomicCAS(status, 0, (int)DEV_CAPACITY);
                else large_list[atomicAdd(large_count, 1)] = (int32_t)sgi;
            }
            continue;
        }
        uint32_t k = lane < len ? keys[b + lane] : 0xffffffffu;
        int rank = 0;
        for (int t = 0; t < len; t++) {
            uint32_t o = __shfl_sync(0xffffffffu, k, t);
            rank += (o < k) ? 1 : 0;
        }
        if (lane < len) out[b + rank] = k;
    }
}

__global__ void k_segsort_block(const int32_t* __restrict__ ptr, const uint32_t* __restrict__ keys, uint32_t* __restrict__ out,
                                const int32_t* large_list, const int32_t* large_count) {
    __shared__ uint32_t sk[kSegSortMax];
    int cnt = *large_count;
    for (int li = blockIdx.x; li < cnt; li += gridDim.x) {
        int sgi = large_list[li];
        int b = ptr[sgi], e = ptr[sgi + 1], len = e - b;
        for (int i = threadIdx.x; i < len; i += blockDim.x) sk[i] = keys[b + i];
        __syncthreads();
        for (int i = threadIdx.x; i < len; i += blockDim.x) {
            uint32_t k = sk[i];
            int rank = 0;
            for (int t = 0; t < len; t++) rank += (sk[t] < k) ? 1 : 0;
            out[b + rank] = k;
        }
        __syncthreads();
    }
}

}  // namespace

void exclusive_scan_i32(const int32_t* in, int32_t* out, int n, int32_t* total, DBuf<int32_t>& tmp, cudaStream_t s,
                        int64_t& launches) {
    exclusive_scan_impl<int32_t>(in, out, n, total, tmp, s, launches);
}

void exclusive_scan_i64(const int64_t* in, int64_t* out, int n, int64_t* total, DBuf<int64_t>& tmp, cudaStream_t s,
                        int64_t& launches) {
    exclusive_scan_impl<int64_t>(in, out, n, total, tmp, s, launches);
}

// Small sorts in one launch: one CTA of 32 warps runs every 8-bit pass.  Per pass each warp
// counts the digits of its contiguous segment, one CTA-wide scan turns the (digit, warp)
// counts into stable offsets, and each warp places its segment 32 keys at a time in order
// (ranks among equal digits by __match_any_sync), so the sort is a stable LSD radix sort like
// the multi-CTA one.  Launch-bound sorts (labels, cluster members) take one launch instead of
// five per pass.
constexpr int kRadixCtaThreads = 1024;
constexpr int kRadixCtaMax = 32768;  // largest n sorted this way
__global__ void __launch_bounds__(kRadixCtaThreads) k_radix_sort_cta(uint64_t* ka, uint32_t* va, uint64_t* kb, uint32_t* vb, int n,
                                                                     int passes, int* final_in_b) {
    __shared__ int32_t cnt[32][256];
    __shared__ int32_t tot[256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int seg = ((n + 31) / 32 + 31) & ~31;
    const int b0 = min(n, w * seg), b1 = min(n, b0 + seg);
    for (int p = 0; p < passes; p++) {
        const int shift = 8 * p;
        for (int i = threadIdx.x; i < 32 * 256; i += blockDim.x) (&cnt[0][0])[i] = 0;
        __syncthreads();
        for (int j = b0 + lane; j < b1; j += 32) atomicAdd(&cnt[w][(ka[j] >> shift) & 0xff], 1);
        __syncthreads();
        if (threadIdx.x < 256) {
            int acc = 0;
            for (int ww = 0; ww < 32; ww++) acc += cnt[ww][threadIdx.x];
            tot[threadIdx.x] = acc;
        }
        __syncthreads();
        for (int o = 1; o < 256; o <<= 1) {  // inclusive scan of the digit totals
            int v = 0;
            if (threadIdx.x < 256 && threadIdx.x >= o) v = tot[threadIdx.x - o];
            __syncthreads();
            if (threadIdx.x < 256) tot[threadIdx.x] += v;
            __syncthreads();
        }
        if (threadIdx.x < 256) {
            const int d = threadIdx.x;
            int acc = d > 0 ? tot[d - 1] : 0;
            for (int ww = 0; ww < 32; ww++) {
                const int c = cnt[ww][d];
                cnt[ww][d] = acc;
                acc += c;
            }
        }
        __syncthreads();
        for (int j0 = b0; j0 < b1; j0 += 32) {
            const int j = j0 + lane;
            const bool valid = j < b1;
            const unsigned vmask = __ballot_sync(0xffffffffu, valid);
            const uint64_t k = valid ? ka[j] : 0;
            const uint32_t v = valid ? va[j] : 0;
            const int d = (int)((k >> shift) & 0xff);
            unsigned peers = __match_any_sync(0xffffffffu, valid ? d : 256 + lane) & vmask;
            const unsigned lt = (1u << lane) - 1u;
            const int pos = valid ? cnt[w][d] + __popc(peers & lt) : 0;
            __syncwarp();
            if (valid && (peers & lt) == 0) cnt[w][d] += __popc(peers);
            __syncwarp();
            if (valid) {
                kb[pos] = k;
                vb[pos] = v;
            }
        }
        __syncthreads();
        uint64_t* tk = ka; ka = kb; kb = tk;
        uint32_t* tv = va; va = vb; vb = tv;
    }
    if (threadIdx.x == 0 && final_in_b) *final_in_b = passes & 1;
}

int bits_for(uint64_t v) {
    int b = 0;
    while (b < 64 && (v >> b) != 0) b++;
    return b < 1 ? 1 : b;
}

void radix_sort_pairs(uint64_t* keys, uint32_t* vals, int n, int bits, RadixScratch& rs, cudaStream_t s, int64_t& launches) {
    if (n <= 1) return;
    int passes = (bits + 7) / 8;
    if (n <= kRadixCtaMax) {
        rs.keys_tmp.ensure(n);
        rs.vals_tmp.ensure(n);
        k_radix_sort_cta<<<1, kRadixCtaThreads, 0, s>>>(keys, vals, rs.keys_tmp.get(), rs.vals_tmp.get(), n, passes, nullptr);
        launches++;
        CICY_LAUNCH_CHECK();
        if (passes & 1) {  // the result is in the scratch arrays
            CICY_CUDA(cudaMemcpyAsync(keys, rs.keys_tmp.get(), sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s));
            CICY_CUDA(cudaMemcpyAsync(vals, rs.vals_tmp.get(), sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
        }
        return;
    }
    int n_tiles = ceil_div(n, kRadixTile);
    rs.keys_tmp.ensure(n);
    rs.vals_tmp.ensure(n);
    rs.hist.ensure((size_t)256 * n_tiles);
    uint64_t* ka = keys;
    uint32_t* va = vals;
    uint64_t* kb = rs.keys_tmp.get();
    uint32_t* vb = rs.vals_tmp.get();
    for (int p = 0; p < passes; p++) {
        int shift = 8 * p;
        k_radix_hist<<<n_tiles, kRadixThreads, 0, s>>>(ka, n, shift, n_tiles, rs.hist.get());
        exclusive_scan_i32(rs.hist.get(), rs.hist.get(), 256 * n_tiles, nullptr, rs.scan_tmp, s, launches);
        k_radix_scatter<<<n_tiles, kRadixThreads, 0, s>>>(ka, va, kb, vb, n, shift, n_tiles, rs.hist.get());
        launches += 2;
        CICY_LAUNCH_CHECK();
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if (ka != keys) {
        CICY_CUDA(cudaMemcpyAsync(keys, ka, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s));
        CICY_CUDA(cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
    }
}

void segmented_sort_u32(const int32_t* ptr, int n_seg, const uint32_t* keys, uint32_t* out, int32_t* large_list,
                        int32_t* large_count, int* status, cudaStream_t s, int64_t& launches) {
    if (n_seg <= 0) return;
    CICY_CUDA(cudaMemsetAsync(large_count, 0, sizeof(int32_t), s));
    int blocks = std::min(ceil_div((long long)n_seg * 32, 256), 148 * 16);
    k_segsort_warp<<<blocks, 256, 0, s>>>(ptr, n_seg, keys, out, large_list, large_count, status);
    k_segsort_block<<<148 * 2, 256, 0, s>>>(ptr, keys, out, large_list, large_count);
    launches += 2;
    CICY_LAUNCH_CHECK();
}

}  // namespace cicy
