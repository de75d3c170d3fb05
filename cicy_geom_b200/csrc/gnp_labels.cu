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

// ---------------------------------------------------------------------------
// GNP point structures: Add_gnp_junction (Hoshen_Kopelman.cpp:1837-1923) and
// Compress_mixed_contacts / Add_mixed_junction (:2181-2306).
//
// Add_gnp_junction adds, contact by contact, the junction point on a and then
// the one on b to their GNP's point list; a point of an interpenetrating pair
// reuses the first point of that GNP's list within tol_gnp of it.  Only points
// of the same GNP interact, so on the device events (point a, point b of each
// linked contact, in order) are grouped by GNP with a stable sort and one thread
// per GNP replays its events; the new points are numbered by a scan in event
// order, as upstream's appends number them.
//
// Compress_mixed_contacts walks GNPs ascending, the CNTs in contact with each
// ascending and their contact points ascending, cutting runs at min_points
// past the run start and keeping each run's first point of least distance; its
// closest GNP point is appended (Add_mixed_junction).  On the device two stable
// radix sorts order the contacts by (GNP, CNT, point), one thread per (GNP,
// CNT) group counts and then writes its junctions at offsets from a scan.

namespace cicy {
namespace {

// Events of one GNP, replayed in order: reuse (initial point, or earlier new event) or new.
__global__ void k_gnp_events(int n_gnps, const int32_t* __restrict__ seg, const uint32_t* __restrict__ ev, const double* __restrict__ ep,
                             const int32_t* __restrict__ epen, const int32_t* __restrict__ iptr, const int32_t* __restrict__ iidx,
                             const double* __restrict__ ipts, double tol2, int32_t* __restrict__ is_new, int32_t* __restrict__ ref_init,
                             int32_t* __restrict__ ref_event) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n_gnps; g += gridDim.x * blockDim.x) {
        for (int k = seg[g]; k < seg[g + 1]; k++) {
            const uint32_t e = ev[k];
            const double px = ep[3 * e], py = ep[3 * e + 1], pz = ep[3 * e + 2];
            int hit_init = -1, hit_event = -1;
            if (epen[e]) {
                for (int j = iptr[g]; j < iptr[g + 1] && hit_init < 0; j++) {
                    const int q = iidx[j];
                    const double dx = px - ipts[3 * q], dy = py - ipts[3 * q + 1], dz = pz - ipts[3 * q + 2];
                    if (dx * dx + dy * dy + dz * dz < tol2) hit_init = q;
                }
                for (int j = seg[g]; j < k && hit_init < 0 && hit_event < 0; j++) {
                    const uint32_t f = ev[j];
                    if (!is_new[f]) continue;
                    const double dx = px - ep[3 * f], dy = py - ep[3 * f + 1], dz = pz - ep[3 * f + 2];
                    if (dx * dx + dy * dy + dz * dz < tol2) hit_event = (int)f;
                }
            }
            is_new[e] = (hit_init < 0 && hit_event < 0) ? 1 : 0;
            ref_init[e] = hit_init;
            ref_event[e] = hit_event;
        }
    }
}

__global__ void k_event_ids(int E, int n_init, const int32_t* __restrict__ is_new, const int32_t* __restrict__ pos,
                            const int32_t* __restrict__ ref_init, const int32_t* __restrict__ ref_event, int32_t* __restrict__ id) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x)
        id[e] = is_new[e] ? n_init + pos[e] : (ref_init[e] >= 0 ? ref_init[e] : n_init + pos[ref_event[e]]);
}

__global__ void k_seg_bounds(int n_seg, int n, const uint64_t* __restrict__ keys, int32_t* __restrict__ seg) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g <= n_seg; g += gridDim.x * blockDim.x) {
        int lo = 0, hi = n;  // first key >= g
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (keys[mid] < (uint64_t)g) lo = mid + 1;
            else hi = mid;
        }
        seg[g] = lo;
    }
}

// Mixed contacts in (GNP, CNT, point) order: one thread per (GNP, CNT) group.
struct MixGroups {
    int n;                       // contacts
    const uint32_t* order;       // contact numbers in (GNP, CNT, point) order
    const int32_t* head;         // group starts (positions in `order`), [n_groups + 1]
    const int32_t *point, *gnp, *flag;
    const double* dist;
    int min_points;
};

template <bool WRITE>
__global__ void k_mix_compress(MixGroups a, int n_groups, int32_t* __restrict__ count, const int32_t* __restrict__ off, int n_points_before,
                               int32_t* __restrict__ j_cnt_point, int32_t* __restrict__ j_cnt, int32_t* __restrict__ j_gnp_point,
                               int32_t* __restrict__ j_gnp, double* __restrict__ j_dist, int32_t* __restrict__ j_contact) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_groups; q += gridDim.x * blockDim.x) {
        const int b = a.head[q], e = a.head[q + 1];
        int k = 0;
        const int o = WRITE ? off[q] : 0;
        auto emit = [&](int contact, int P, double d) {
            if (WRITE) {
                j_cnt_point[o + k] = P;
                j_cnt[o + k] = a.flag[P];
                j_gnp_point[o + k] = n_points_before + o + k;
                j_gnp[o + k] = a.gnp[contact];
                j_dist[o + k] = d;
                j_contact[o + k] = contact;
            }
            k++;
        };
        uint32_t c = a.order[b];
        int Pj0 = a.point[c], Pj = Pj0;
        int cj = (int)c;
        double dmin = a.dist[c];
        for (int i = b + 1; i < e; i++) {
            c = a.order[i];
            const int P1 = a.point[c];
            const double d = a.dist[c];
            if (P1 - Pj0 >= a.min_points) {
                emit(cj, Pj, dmin);
                dmin = d;
                cj = (int)c;
                Pj = P1;
                Pj0 = P1;
            } else if (d < dmin) {
                dmin = d;
                cj = (int)c;
                Pj = P1;
            }
        }
        emit(cj, Pj, dmin);
        if (!WRITE) count[q] = k;
    }
}

__global__ void k_mix_group_keys(int n, const int32_t* __restrict__ point, const int32_t* __restrict__ gnp, const int32_t* __restrict__ flag,
                                 int n_cnts, int by_point, uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = vals[i];
        keys[i] = by_point ? (uint64_t)point[c] : (uint64_t)gnp[c] * (uint64_t)n_cnts + (uint64_t)flag[point[c]];
    }
}

__global__ void k_iota(int n, uint32_t* v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = (uint32_t)i;
}

__global__ void k_group_heads(int n, const uint64_t* __restrict__ keys, int32_t* __restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

__global__ void k_group_starts(int n, const int32_t* __restrict__ flag, const int32_t* __restrict__ pos, int32_t* __restrict__ head) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) head[pos[i]] = i;
}

__global__ void k_gather_closest(int m, const int32_t* __restrict__ contact, const double* __restrict__ closest, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        for (int d = 0; d < 3; d++) out[3 * i + d] = closest[3 * contact[i] + d];
}

}  // namespace

void gnp_junction_structures(const GnpPairs& pairs, int n_gnps, double tol_gnp2, const std::vector<double>& init_points,
                             const std::vector<int32_t>& init_ptr, const std::vector<int32_t>& init_idx, GnpStructures& out) {
    const int n_init = (int)(init_points.size() / 3);
    out = GnpStructures{};
    out.points = init_points;
    out.n_boundary = n_init;
    out.boundary_used.assign(n_init, 0);
    std::vector<int32_t> ev_gnp;
    std::vector<double> ev_pt;
    std::vector<int32_t> ev_pen;
    std::vector<int> kept;
    for (size_t i = 0; i < pairs.a.size(); i++) {
        if (pairs.outside[i] != 0) continue;
        kept.push_back((int)i);
        for (int s = 0; s < 2; s++) {
            ev_gnp.push_back(s == 0 ? pairs.a[i] : pairs.b[i]);
            const double* P = (s == 0 ? pairs.point_a.data() : pairs.point_b.data()) + 3 * i;
            ev_pt.insert(ev_pt.end(), {P[0], P[1], P[2]});
            ev_pen.push_back(pairs.penetrating[i]);
        }
    }
    const int E = (int)ev_gnp.size();
    std::vector<int32_t> ids(E);
    if (E > 0) {
        DBuf<uint64_t> keys;
        DBuf<uint32_t> vals;
        DBuf<int32_t> seg, epen, iptr, iidx, is_new, ref_i, ref_e, pos, total, id, scan32;
        DBuf<double> ep, ipts;
        keys.ensure(E); vals.ensure(E); seg.ensure(n_gnps + 1); epen.ensure(E); iptr.ensure(n_gnps + 1);
        iidx.ensure(std::max<size_t>(init_idx.size(), 1)); is_new.ensure(E); ref_i.ensure(E); ref_e.ensure(E); pos.ensure(E); total.ensure(1);
        id.ensure(E); ep.ensure(3 * (size_t)E); ipts.ensure(std::max<size_t>(init_points.size(), 1));
        std::vector<uint64_t> hk(ev_gnp.begin(), ev_gnp.end());
        CICY_CUDA(cudaMemcpy(keys.get(), hk.data(), sizeof(uint64_t) * E, cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(epen.get(), ev_pen.data(), sizeof(int32_t) * E, cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(ep.get(), ev_pt.data(), sizeof(double) * 3 * E, cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(iptr.get(), init_ptr.data(), sizeof(int32_t) * (n_gnps + 1), cudaMemcpyHostToDevice));
        if (!init_idx.empty()) CICY_CUDA(cudaMemcpy(iidx.get(), init_idx.data(), sizeof(int32_t) * init_idx.size(), cudaMemcpyHostToDevice));
        if (!init_points.empty())
            CICY_CUDA(cudaMemcpy(ipts.get(), init_points.data(), sizeof(double) * init_points.size(), cudaMemcpyHostToDevice));
        int64_t launches = 0;
        k_iota<<<label_blocks(E), 256>>>(E, vals.get());
        RadixScratch rs;
        radix_sort_pairs(keys.get(), vals.get(), E, bits_for((uint64_t)n_gnps), rs, nullptr, launches);  // stable: events of a GNP stay in order
        k_seg_bounds<<<label_blocks(n_gnps + 1), 256>>>(n_gnps, E, keys.get(), seg.get());
        k_gnp_events<<<label_blocks(n_gnps), 256>>>(n_gnps, seg.get(), vals.get(), ep.get(), epen.get(), iptr.get(), iidx.get(), ipts.get(), tol_gnp2,
                                                   is_new.get(), ref_i.get(), ref_e.get());
        exclusive_scan_i32(is_new.get(), pos.get(), E, total.get(), scan32, nullptr, launches);
        k_event_ids<<<label_blocks(E), 256>>>(E, n_init, is_new.get(), pos.get(), ref_i.get(), ref_e.get(), id.get());
        CICY_LAUNCH_CHECK();
        std::vector<int32_t> hn(E);
        CICY_CUDA(cudaMemcpy(ids.data(), id.get(), sizeof(int32_t) * E, cudaMemcpyDeviceToHost));
        CICY_CUDA(cudaMemcpy(hn.data(), is_new.get(), sizeof(int32_t) * E, cudaMemcpyDeviceToHost));
        out.launches = launches + 5;
        // the points and lists in upstream's append order (host bookkeeping of the device results)
        std::vector<std::vector<int32_t>> add(n_gnps);
        for (int e = 0; e < E; e++)
            if (hn[e]) {
                out.points.insert(out.points.end(), {ev_pt[3 * e], ev_pt[3 * e + 1], ev_pt[3 * e + 2]});
                add[ev_gnp[e]].push_back(ids[e]);
            }
        out.structure_ptr.assign(1, 0);
        for (int g = 0; g < n_gnps; g++) {
            out.structure_idx.insert(out.structure_idx.end(), init_idx.begin() + init_ptr[g], init_idx.begin() + init_ptr[g + 1]);
            out.structure_idx.insert(out.structure_idx.end(), add[g].begin(), add[g].end());
            out.structure_ptr.push_back((int32_t)out.structure_idx.size());
        }
    } else {
        out.structure_ptr = init_ptr;
        out.structure_idx = init_idx;
    }
    for (size_t k = 0; k < kept.size(); k++) {
        const int i = kept[k];
        out.junctions.insert(out.junctions.end(), {ids[2 * k], pairs.a[i], ids[2 * k + 1], pairs.b[i]});
        out.junction_dist.push_back(pairs.dist[i]);
        for (int s = 0; s < 2; s++)  // bp_flags of a reused boundary point (:1866-1876)
            if (ids[2 * k + s] < n_init) out.boundary_used[ids[2 * k + s]] = 1;
    }
}

int run_mixed_junctions(Ctx& c, int n_points_before, int min_points, std::vector<int32_t>& junctions, std::vector<double>& dist,
                        std::vector<double>& points) {
    if (min_points < 0 || n_points_before < 0) throw Fail{CICY_E_INPUT, "cicy_mixed_junctions: invalid arguments"};
    junctions.clear();
    dist.clear();
    points.clear();
    const int n = c.n_mix;
    if (n == 0) return 0;
    cudaStream_t s = c.stream;
    int n_gnps = 0;
    {
        std::vector<int32_t> g(n);
        CICY_CUDA(cudaMemcpyAsync(g.data(), c.mix_gnp.get(), sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaStreamSynchronize(s));
        for (int32_t v : g) n_gnps = std::max(n_gnps, v + 1);
    }
    DBuf<uint64_t> keys;
    DBuf<uint32_t> vals;
    DBuf<int32_t> flag, pos, total, head, count, off, scan32;
    keys.ensure(n); vals.ensure(n); flag.ensure(n); pos.ensure(n); total.ensure(1); head.ensure(n + 1);
    int64_t launches = 0;
    k_iota<<<label_blocks(n), 256, 0, s>>>(n, vals.get());
    // (GNP, CNT, point) order: sort by point, then stably by (GNP, CNT)
    k_mix_group_keys<<<label_blocks(n), 256, 0, s>>>(n, c.mix_point.get(), c.mix_gnp.get(), c.flag.get(), c.n_cnts, 1, keys.get(), vals.get());
    radix_sort_pairs(keys.get(), vals.get(), n, bits_for((uint64_t)std::max(c.n_points, 1)), c.rs, s, launches);
    k_mix_group_keys<<<label_blocks(n), 256, 0, s>>>(n, c.mix_point.get(), c.mix_gnp.get(), c.flag.get(), c.n_cnts, 0, keys.get(), vals.get());
    radix_sort_pairs(keys.get(), vals.get(), n, bits_for((uint64_t)n_gnps * (uint64_t)std::max(c.n_cnts, 1)), c.rs, s, launches);
    k_group_heads<<<label_blocks(n), 256, 0, s>>>(n, keys.get(), flag.get());
    exclusive_scan_i32(flag.get(), pos.get(), n, total.get(), scan32, s, launches);
    int G = 0;
    CICY_CUDA(cudaMemcpyAsync(&G, total.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    k_group_starts<<<label_blocks(n), 256, 0, s>>>(n, flag.get(), pos.get(), head.get());
    CICY_CUDA(cudaMemcpyAsync(head.get() + G, &n, sizeof(int32_t), cudaMemcpyHostToDevice, s));
    count.ensure(G + 1);
    off.ensure(G + 1);
    MixGroups a{n, vals.get(), head.get(), c.mix_point.get(), c.mix_gnp.get(), c.flag.get(), c.mix_dist.get(), min_points};
    k_mix_compress<false><<<label_blocks(G), 256, 0, s>>>(a, G, count.get(), nullptr, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    CICY_CUDA(cudaMemsetAsync(count.get() + G, 0, sizeof(int32_t), s));
    exclusive_scan_i32(count.get(), off.get(), G + 1, total.get(), scan32, s, launches);
    int J = 0;
    CICY_CUDA(cudaMemcpyAsync(&J, total.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    DBuf<int32_t> jp, jc, jgp, jg, jcontact;
    DBuf<double> jd, jq;
    jp.ensure(J); jc.ensure(J); jgp.ensure(J); jg.ensure(J); jcontact.ensure(J); jd.ensure(J); jq.ensure(3 * (size_t)J);
    k_mix_compress<true><<<label_blocks(G), 256, 0, s>>>(a, G, nullptr, off.get(), n_points_before, jp.get(), jc.get(), jgp.get(), jg.get(),
                                                        jd.get(), jcontact.get());
    k_gather_closest<<<label_blocks(J), 256, 0, s>>>(J, jcontact.get(), c.mix_closest.get(), jq.get());
    CICY_LAUNCH_CHECK();
    std::vector<int32_t> hp(J), hc(J), hgp(J), hg(J);
    dist.resize(J);
    points.resize(3 * (size_t)J);
    CICY_CUDA(cudaMemcpyAsync(hp.data(), jp.get(), sizeof(int32_t) * J, cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaMemcpyAsync(hc.data(), jc.get(), sizeof(int32_t) * J, cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaMemcpyAsync(hgp.data(), jgp.get(), sizeof(int32_t) * J, cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaMemcpyAsync(hg.data(), jg.get(), sizeof(int32_t) * J, cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaMemcpyAsync(dist.data(), jd.get(), sizeof(double) * J, cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaMemcpyAsync(points.data(), jq.get(), sizeof(double) * 3 * J, cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    for (int j = 0; j < J; j++) junctions.insert(junctions.end(), {hp[j], hc[j], hgp[j], hg[j]});
    c.launches += launches + 9;
    return J;
}

}  // namespace cicy

// ---------------------------------------------------------------------------
extern "C" {

cicy_status cicy_gnp_junction_structures(int device, const cicy_gnp_pairs* pairs, int32_t n_gnps, double tol_gnp2, int32_t n_init_points,
                                         const double* init_points, const int32_t* init_ptr, const int32_t* init_idx, cicy_gnp_points** out) {
    if (!pairs || !out || n_gnps < 0 || n_init_points < 0 || !(tol_gnp2 >= 0) || (n_init_points > 0 && !init_points) ||
        (init_ptr && init_ptr[n_gnps] > 0 && !init_idx)) {
        cicy::set_host_error("cicy_gnp_junction_structures: invalid arguments");
        return CICY_E_INPUT;
    }
    *out = nullptr;
    std::vector<int32_t> iptr(n_gnps + 1, 0), iidx;
    if (init_ptr) {
        for (int g = 0; g <= n_gnps; g++) iptr[g] = init_ptr[g];
        for (int g = 0; g < n_gnps; g++)
            if (iptr[g + 1] < iptr[g] || iptr[0] != 0) {
                cicy::set_host_error("cicy_gnp_junction_structures: structure offsets not ascending");
                return CICY_E_INPUT;
            }
        iidx.assign(init_idx, init_idx + iptr[n_gnps]);
        for (int32_t v : iidx)
            if (v < 0 || v >= n_init_points) {
                cicy::set_host_error("cicy_gnp_junction_structures: a structure names a point outside the initial points");
                return CICY_E_INPUT;
            }
    }
    const cicy::GnpPairs& q = pairs->pairs;
    for (size_t i = 0; i < q.a.size(); i++)
        if (q.a[i] >= n_gnps || q.b[i] >= n_gnps) {
            cicy::set_host_error("cicy_gnp_junction_structures: a contact names a GNP beyond n_gnps");
            return CICY_E_INPUT;
        }
    cicy_gnp_points* p = new cicy_gnp_points;
    try {
        CICY_CUDA(cudaSetDevice(device));
        std::vector<double> ipts(init_points, init_points + 3 * (size_t)n_init_points);
        cicy::gnp_junction_structures(q, n_gnps, tol_gnp2, ipts, iptr, iidx, p->s);
    } catch (const cicy::Fail& e) {
        cicy::set_host_error(e.msg);
        delete p;
        return e.status;
    }
    *out = p;
    return CICY_OK;
}

cicy_status cicy_gnp_points_view(const cicy_gnp_points* p, cicy_gnp_point_list* v) {
    if (!p || !v) return CICY_E_INPUT;
    const cicy::GnpStructures& s = p->s;
    v->n_points = (int64_t)(s.points.size() / 3);
    v->points = s.points.data();
    v->n_gnps = (int32_t)s.structure_ptr.size() - 1;
    v->structure_ptr = s.structure_ptr.data();
    v->structure_idx = s.structure_idx.data();
    v->n_junctions = (int64_t)s.junction_dist.size();
    v->junctions = s.junctions.data();
    v->junction_dist = s.junction_dist.data();
    v->n_boundary = s.n_boundary;
    v->boundary_used = s.boundary_used.data();
    return CICY_OK;
}

void cicy_gnp_points_free(cicy_gnp_points* p) { delete p; }

}  // extern "C"
