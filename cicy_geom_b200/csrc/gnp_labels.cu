// Labels of GNP and mixed CNT/GNP clusters on the device: the HK76 passes of
// Hoshen_Kopelman::Label_gnps_in_window (GNP-GNP contacts whose junction points
// are inside the sample, Hoshen_Kopelman.cpp:626-767) and Find_adjacent_labels
// (CNT-GNP contacts, :1989-2142), each followed by Cleanup_labels (:374-425).
//
// HK76 (:2908-2953) gives a contact between two unlabelled particles a new
// label, in contact order; Merge_labels (:2969-2989) keeps the smaller root;
// Cleanup_labels numbers the surviving roots in ascending order.  So a
// cluster's final label is the rank of its smallest raw label: the smallest
// label it already had before the pass, or else the label its first contact
// created (labels created in a pass are above all earlier ones and ascend with
// contact order).  On the device: union-find over the earlier labels and the
// unlabelled particles, a min per cluster of the key (earlier label, or the
// label count + contact ordinal), and a rank of the keys.
#include <algorithm>
#include <string>
#include <vector>

#include "cicy_internal.h"
#include "ctx.cuh"
#include "dev_common.cuh"
#include "uf.cuh"

namespace cicy {
namespace {

int label_blocks(long long n) { return (int)std::max(1LL, std::min((n + 255) / 256, 148LL * 16)); }

// Entity of particle p: its earlier label, or n_pre + p when unlabelled.
__device__ __forceinline__ int entity(const int32_t* __restrict__ pre, int n_pre, int p) { return pre[p] >= 0 ? pre[p] : n_pre + p; }

__global__ void k_lab_init(int n, int32_t* __restrict__ parent, unsigned long long* __restrict__ key) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        parent[i] = i;
        key[i] = ~0ull;
    }
}

__global__ void k_lab_unite(int m, const int32_t* __restrict__ u, const int32_t* __restrict__ v, const int32_t* __restrict__ pre, int n_pre,
                            int32_t* parent) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        uf_unite(parent, entity(pre, n_pre, u[i]), entity(pre, n_pre, v[i]));
}

__global__ void k_lab_roots(int n, const int32_t* __restrict__ parent, int32_t* __restrict__ root) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) root[i] = uf_root(parent, i);
}

// Keys: an earlier label keys its own cluster; contact i keys its cluster with n_pre + i.
__global__ void k_lab_keys(int n_pre, int m, const int32_t* __restrict__ u, const int32_t* __restrict__ pre, const int32_t* __restrict__ root,
                           unsigned long long* key) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_pre + m; i += gridDim.x * blockDim.x) {
        if (i < n_pre) atomicMin(&key[root[i]], (unsigned long long)i);
        else atomicMin(&key[root[entity(pre, n_pre, u[i - n_pre])]], (unsigned long long)i);
    }
}

__global__ void k_lab_flags(int n, const int32_t* __restrict__ root, const unsigned long long* __restrict__ key, int32_t* __restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flag[i] = (root[i] == i && key[i] != ~0ull) ? 1 : 0;
}

__global__ void k_lab_gather(int n, const int32_t* __restrict__ flag, const int32_t* __restrict__ pos, const unsigned long long* __restrict__ key,
                             uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) {
            keys[pos[i]] = key[i];
            vals[pos[i]] = (uint32_t)i;
        }
}

__global__ void k_lab_rank(int c, const uint32_t* __restrict__ vals, int32_t* __restrict__ rank) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) rank[vals[i]] = i;
}

__global__ void k_lab_out(int n, const int32_t* __restrict__ pre, int n_pre, const int32_t* __restrict__ root,
                          const unsigned long long* __restrict__ key, const int32_t* __restrict__ rank, int32_t* __restrict__ out) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int r = root[entity(pre, n_pre, p)];
        out[p] = key[r] == ~0ull ? -1 : rank[r];
    }
}

// A contact list whose particle indices are out of range.
__global__ void k_lab_check(int m, const int32_t* __restrict__ u, const int32_t* __restrict__ v, int n, int32_t* __restrict__ bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        if (u[i] < 0 || u[i] >= n || v[i] < 0 || v[i] >= n) atomicMin(bad, i);
}

}  // namespace

// Labels after an HK76 pass over contacts (u[i], v[i]) in order and Cleanup_labels:
// particles 0..n-1 with earlier proper labels pre[] (-1: none, else < n_pre).
// Device arrays; out[n] on the device; returns the number of labels.
int relabel(int n, const int32_t* pre, int n_pre, int m, const int32_t* u, const int32_t* v, int32_t* out, cudaStream_t s, int64_t& launches) {
    const long long E = (long long)n_pre + n;
    if (E >= (1LL << 31) - 1 || (long long)n_pre + m >= (1LL << 62)) throw Fail{CICY_E_CAPACITY, "relabel: too many particles"};
    DBuf<int32_t> parent, root, flag, pos, total, rank, bad;
    DBuf<unsigned long long> key;
    DBuf<int32_t> scan32;
    parent.ensure(E);
    root.ensure(E);
    key.ensure(E);
    flag.ensure(E);
    pos.ensure(E);
    rank.ensure(E);
    total.ensure(1);
    bad.ensure(1);
    if (m > 0) {
        const int32_t big = 0x7fffffff;
        CICY_CUDA(cudaMemcpyAsync(bad.get(), &big, sizeof(int32_t), cudaMemcpyHostToDevice, s));
        k_lab_check<<<label_blocks(m), 256, 0, s>>>(m, u, v, n, bad.get());
        int32_t hb = 0;
        CICY_CUDA(cudaMemcpyAsync(&hb, bad.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaStreamSynchronize(s));
        if (hb != big) throw Fail{CICY_E_INPUT, "relabel: contact " + std::to_string(hb) + " names a particle out of range"};
    }
    k_lab_init<<<label_blocks(E), 256, 0, s>>>((int)E, parent.get(), key.get());
    if (m > 0) k_lab_unite<<<label_blocks(m), 256, 0, s>>>(m, u, v, pre, n_pre, parent.get());
    k_lab_roots<<<label_blocks(E), 256, 0, s>>>((int)E, parent.get(), root.get());
    k_lab_keys<<<label_blocks((long long)n_pre + m), 256, 0, s>>>(n_pre, m, u, pre, root.get(), key.get());
    k_lab_flags<<<label_blocks(E), 256, 0, s>>>((int)E, root.get(), key.get(), flag.get());
    exclusive_scan_i32(flag.get(), pos.get(), (int)E, total.get(), scan32, s, launches);
    int C = 0;
    CICY_CUDA(cudaMemcpyAsync(&C, total.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    if (C > 0) {
        DBuf<uint64_t> keys;
        DBuf<uint32_t> vals;
        keys.ensure(C);
        vals.ensure(C);
        k_lab_gather<<<label_blocks(E), 256, 0, s>>>((int)E, flag.get(), pos.get(), key.get(), keys.get(), vals.get());
        RadixScratch rs;
        radix_sort_pairs(keys.get(), vals.get(), C, bits_for((uint64_t)n_pre + (uint64_t)m), rs, s, launches);
        k_lab_rank<<<label_blocks(C), 256, 0, s>>>(C, vals.get(), rank.get());
    }
    k_lab_out<<<label_blocks(n), 256, 0, s>>>(n, pre, n_pre, root.get(), key.get(), rank.get(), out);
    CICY_LAUNCH_CHECK();
    CICY_CUDA(cudaStreamSynchronize(s));
    launches += 8;
    return C;
}

void gnp_labels(const GnpPairs& pairs, int n_gnps, int n_labels_cnt, std::vector<int32_t>& labels, int& n_total) {
    std::vector<int32_t> u, v;
    for (size_t i = 0; i < pairs.a.size(); i++)
        if (pairs.outside[i] == 0) {  // both junction points inside the sample: HK76 (Hoshen_Kopelman.cpp:727-744)
            u.push_back(pairs.a[i]);
            v.push_back(pairs.b[i]);
        }
    labels.assign(n_gnps, -1);
    n_total = n_labels_cnt;
    if (n_gnps == 0) return;
    DBuf<int32_t> pre, du, dv, out;
    pre.ensure(n_gnps);
    du.ensure(std::max<size_t>(u.size(), 1));
    dv.ensure(std::max<size_t>(u.size(), 1));
    out.ensure(n_gnps);
    CICY_CUDA(cudaMemcpy(pre.get(), labels.data(), sizeof(int32_t) * n_gnps, cudaMemcpyHostToDevice));
    if (!u.empty()) {
        CICY_CUDA(cudaMemcpy(du.get(), u.data(), sizeof(int32_t) * u.size(), cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(dv.get(), v.data(), sizeof(int32_t) * v.size(), cudaMemcpyHostToDevice));
    }
    int64_t launches = 0;
    const int n_gnp_labels = relabel(n_gnps, pre.get(), 0, (int)u.size(), du.get(), dv.get(), out.get(), nullptr, launches);
    CICY_CUDA(cudaMemcpy(labels.data(), out.get(), sizeof(int32_t) * n_gnps, cudaMemcpyDeviceToHost));
    for (int32_t& l : labels)  // Renumber_gnp_labels (:427-440)
        if (l >= 0) l += n_labels_cnt;
    n_total = n_labels_cnt + n_gnp_labels;
}

namespace {
__global__ void k_mixed_contacts(int m, const int32_t* __restrict__ point, const int32_t* __restrict__ gnp, const int32_t* __restrict__ flag,
                                 int n_cnts, int32_t* __restrict__ u, int32_t* __restrict__ v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        u[i] = flag[point[i]];
        v[i] = n_cnts + gnp[i];
    }
}
}  // namespace

// Make_mixed_clusters' labels (:1925-1987): the context's CNT labels and CNT-GNP
// contacts with the given GNP labels; CNT labels in the context are replaced.
int run_mixed_labels(Ctx& c, const int32_t* labels_gnp, int n_gnps, int n_total_labels, int32_t* labels_cnt_out, int32_t* labels_gnp_out) {
    if (c.stage < 3) throw Fail{CICY_E_STATE, "cicy_mixed_labels: no CNT labels (run cicy_clusters)"};
    if (n_gnps < 0 || n_total_labels < c.n_labels) throw Fail{CICY_E_INPUT, "cicy_mixed_labels: invalid label counts"};
    for (int g = 0; g < n_gnps; g++)
        if (labels_gnp[g] < -1 || labels_gnp[g] >= n_total_labels) throw Fail{CICY_E_INPUT, "cicy_mixed_labels: a GNP label is out of range"};
    cudaStream_t s = c.stream;
    const int n = c.n_cnts + n_gnps, m = c.n_mix;
    DBuf<int32_t> pre, u, v, out;
    pre.ensure(std::max(n, 1));
    u.ensure(std::max(m, 1));
    v.ensure(std::max(m, 1));
    out.ensure(std::max(n, 1));
    if (c.n_cnts) CICY_CUDA(cudaMemcpyAsync(pre.get(), c.labels.get(), sizeof(int32_t) * c.n_cnts, cudaMemcpyDeviceToDevice, s));
    if (n_gnps) CICY_CUDA(cudaMemcpyAsync(pre.get() + c.n_cnts, labels_gnp, sizeof(int32_t) * n_gnps, cudaMemcpyHostToDevice, s));
    if (m > 0) {
        k_mixed_contacts<<<label_blocks(m), 256, 0, s>>>(m, c.mix_point.get(), c.mix_gnp.get(), c.flag.get(), c.n_cnts, u.get(), v.get());
        CICY_LAUNCH_CHECK();
    }
    int64_t launches = 0;
    const int n_clusters = n > 0 ? relabel(n, pre.get(), n_total_labels, m, u.get(), v.get(), out.get(), s, launches) : 0;
    c.launches += launches + 1;
    if (labels_cnt_out && c.n_cnts)
        CICY_CUDA(cudaMemcpyAsync(labels_cnt_out, out.get(), sizeof(int32_t) * c.n_cnts, cudaMemcpyDeviceToHost, s));
    if (labels_gnp_out && n_gnps)
        CICY_CUDA(cudaMemcpyAsync(labels_gnp_out, out.get() + c.n_cnts, sizeof(int32_t) * n_gnps, cudaMemcpyDeviceToHost, s));
    if (c.n_cnts) CICY_CUDA(cudaMemcpyAsync(c.labels.get(), out.get(), sizeof(int32_t) * c.n_cnts, cudaMemcpyDeviceToDevice, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    c.n_labels = n_clusters;
    return n_clusters;
}

}  // namespace cicy

// ---------------------------------------------------------------------------
extern "C" {

cicy_status cicy_gnp_labels(int device, const cicy_gnp_pairs* pairs, int32_t n_gnps, int32_t n_labels_cnt, int32_t* labels_gnp,
                            int32_t* n_total_labels) {
    if (!pairs || n_gnps < 0 || n_labels_cnt < 0 || (n_gnps > 0 && !labels_gnp) || !n_total_labels) {
        cicy::set_host_error("cicy_gnp_labels: invalid arguments");
        return CICY_E_INPUT;
    }
    for (size_t i = 0; i < pairs->pairs.a.size(); i++)
        if (pairs->pairs.a[i] >= n_gnps || pairs->pairs.b[i] >= n_gnps) {
            cicy::set_host_error("cicy_gnp_labels: a contact names a GNP beyond n_gnps");
            return CICY_E_INPUT;
        }
    try {
        CICY_CUDA(cudaSetDevice(device));
        std::vector<int32_t> lab;
        int total = 0;
        cicy::gnp_labels(pairs->pairs, n_gnps, n_labels_cnt, lab, total);
        std::copy(lab.begin(), lab.end(), labels_gnp);
        *n_total_labels = total;
    } catch (const cicy::Fail& e) {
        cicy::set_host_error(e.msg);
        return e.status;
    }
    return CICY_OK;
}

}  // extern "C"
