// GNP part of the contact grid (device): Contact_grid::Fill_sectioned_domain_gnps /
// Fill_sectioned_domain_single_gnp / Assign_point_to_regions_gnps
// (Contact_grid.cpp:297-512).  Each GNP in `inside` order is sampled on a
// regular grid of its volume (nx = max(40, 1 + (int)(l / lx)), the same for y,
// nz = max(2, 1 + (int)(t / lz)); points bilinear between its vertices in
// upstream's operation order); a point strictly inside the window adds the
// GNP to its region and to the neighbour regions its overlap flags name.  A
// region lists each GNP once, in `inside` order.
//
// One thread per sample point emits up to four keys region * n_inside + order
// (32 bits); a radix sort, a unique pass and a binary search per region give
// the CSR of region lists.  FP64 without contraction (this file is built with
// --fmad=false), so points, regions and flags equal upstream's.
//
// CNT-GNP contacts of the hybrid grid (Hoshen_Kopelman::Find_adjacent_labels,
// Hoshen_Kopelman.cpp:1989-2142): upstream visits, region by region, every GNP
// of the region against every CNT point of the region, and numbers a (point,
// GNP) pair's contact point when the pair first tests as a contact.  The test
// depends on the pair only, so the number is the rank of the pair's first
// visit among the contact pairs.  On the device every visit is one thread
// (ordinal = region offset + GNP slot x points + point slot); contact visits
// append (pair key, ordinal), a sort by pair key and a min per run give each
// pair's first ordinal, and a sort by that ordinal gives upstream's numbers.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cicy_internal.h"
#include "ctx.cuh"
#include "dev_common.cuh"
#include "gnp_geom.cuh"

namespace cicy {
namespace {

constexpr uint32_t kNoKey = 0xffffffffu;

struct GnpGridArgs {
    int n_inside;
    const int32_t* inside;    // GNP index of each order position
    const int64_t* pt_off;    // first sample point of each order position, [n_inside + 1]
    const int32_t* nxyz;      // nx, ny, nz per order position
    const double* vertices;   // [24 * n_gnps]
    double wmin[3], wmax[3];
    int nreg[3];
    double lreg[3];
    double overlap;
    long long n_points;
    uint64_t* keys;           // [4 * n_points]
};

__global__ void k_gnp_sample(GnpGridArgs a) {
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < a.n_points; s += (long long)gridDim.x * blockDim.x) {
        // order position of sample s (offsets ascend)
        int lo = 0, hi = a.n_inside - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.pt_off[mid] <= s) lo = mid;
            else hi = mid - 1;
        }
        const int ord = lo;
        const int nx = a.nxyz[3 * ord], ny = a.nxyz[3 * ord + 1], nz = a.nxyz[3 * ord + 2];
        const long long loc = s - a.pt_off[ord];
        const int k = (int)(loc / ((long long)nx * ny));
        const int j = (int)((loc / nx) % ny);
        const int i = (int)(loc % nx);
        const double* V = a.vertices + 24 * (size_t)a.inside[ord];
        const double lz = (double)k / (nz - 1), ly = (double)j / (ny - 1), lx = (double)i / (nx - 1);
        double p[3];
        for (int d = 0; d < 3; d++) {
            const double start1 = V[21 + d] + (V[9 + d] - V[21 + d]) * lz;   // vertices 7, 3
            const double end1 = V[12 + d] + (V[0 + d] - V[12 + d]) * lz;     // vertices 4, 0
            const double diff1 = end1 - start1;
            const double start2 = V[18 + d] + (V[6 + d] - V[18 + d]) * lz;   // vertices 6, 2
            const double end2 = V[15 + d] + (V[3 + d] - V[15 + d]) * lz;     // vertices 5, 1
            const double diff2 = end2 - start2;
            const double start_x = start1 + diff1 * ly;
            const double end_x = start2 + diff2 * ly;
            const double diff_x = end_x - start_x;
            p[d] = start_x + diff_x * lx;
        }
        uint64_t* out = a.keys + 4 * s;
        out[0] = out[1] = out[2] = out[3] = kNoKey;
        bool in = true;
        for (int d = 0; d < 3; d++) in &= !(p[d] <= a.wmin[d] || p[d] >= a.wmax[d]);
        if (!in) continue;
        int abc[3], f[3];
        for (int d = 0; d < 3; d++) {  // Calculate_region_coordinates, Calculate_overlapping_flags
            int c = (int)((p[d] - a.wmin[d]) / a.lreg[d]);
            c = c < 0 ? 0 : (c >= a.nreg[d] ? a.nreg[d] - 1 : c);
            abc[d] = c;
            const double x1 = (double)c * a.lreg[d] + a.wmin[d];
            const double x2 = x1 + a.lreg[d];
            f[d] = 0;
            if (c > 0 && p[d] >= x1 && p[d] <= x1 + a.overlap) f[d] = -1;
            else if (c < a.nreg[d] - 1 && p[d] >= x2 - a.overlap && p[d] <= x2) f[d] = 1;
        }
        const uint32_t n_in = (uint32_t)a.n_inside;
        auto key = [&](int x, int y, int z) {
            return (uint64_t)((uint32_t)(x + y * a.nreg[0] + z * a.nreg[0] * a.nreg[1]) * n_in + (uint32_t)ord);
        };
        out[0] = key(abc[0], abc[1], abc[2]);
        if (f[0]) out[1] = key(abc[0] + f[0], abc[1], abc[2]);
        if (f[1]) out[2] = key(abc[0], abc[1] + f[1], abc[2]);
        if (f[2]) out[3] = key(abc[0], abc[1], abc[2] + f[2]);
    }
}

__global__ void k_first_of_run(long long n, const uint64_t* __restrict__ keys, int32_t* __restrict__ flag) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        flag[i] = (keys[i] != kNoKey && (i == 0 || keys[i] != keys[i - 1])) ? 1 : 0;
}

__global__ void k_compact(long long n, const uint64_t* __restrict__ keys, const int32_t* __restrict__ flag,
                          const int32_t* __restrict__ pos, uint32_t* __restrict__ uniq) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (flag[i]) uniq[pos[i]] = (uint32_t)keys[i];
}

// ptr[t] = first unique key >= t * n_inside; idx = key - region * n_inside (the order position)
__global__ void k_region_ptr(int tot, int n_unique, uint32_t n_inside, const uint32_t* __restrict__ uniq, int32_t* __restrict__ ptr) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= tot; t += gridDim.x * blockDim.x) {
        const uint64_t target = (uint64_t)t * n_inside;
        int lo = 0, hi = n_unique;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((uint64_t)uniq[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        ptr[t] = lo;
    }
}

__global__ void k_region_idx(int n_unique, uint32_t n_inside, const int32_t* __restrict__ inside, const uint32_t* __restrict__ uniq,
                             int32_t* __restrict__ idx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_unique; i += gridDim.x * blockDim.x) idx[i] = inside[uniq[i] % n_inside];
}

int blocks_for(long long n) { return (int)std::max(1LL, std::min((n + 255) / 256, 148LL * 16)); }

// Closest GNP point to each query point (gnp_geom.cuh), one thread per query.
__global__ void k_gnp_closest(int n, const double* __restrict__ xyz, const int32_t* __restrict__ gnp, const double* __restrict__ V,
                              const double* __restrict__ F, double* __restrict__ dist, double* __restrict__ q, int32_t* __restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int g = gnp[i];
        gnp::P3 c;
        double d;
        flag[i] = gnp::closest_point(V + 24 * (size_t)g, F + 24 * (size_t)g, gnp::P3{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]}, c, d);
        dist[i] = d;
        q[3 * i] = c.x;
        q[3 * i + 1] = c.y;
        q[3 * i + 2] = c.z;
    }
}

// ---------------------------------------------------------------------------
// CNT-GNP contacts

struct MixArgs {
    int n_regions;
    const int64_t* visit_off;   // first visit ordinal of each region [n_regions + 1]
    const int32_t* gptr;        // GNP region lists (CSR)
    const int32_t* gidx;
    const int32_t* cptr;        // CNT region lists: slots of region t are cptr[t] .. cptr[t+1]
    const uint32_t* slot;       // traversal index of each slot
    const int32_t* trav_pt;     // point of each traversal index
    const double *x, *y, *z, *radii;
    const int32_t* flag;        // CNT of each point
    const double *V, *F;        // GNP vertices and face planes
    double vdw, tunnel;
    uint32_t n_gnps;
    long long n_visits;
    uint64_t* keys;             // pair key P * n_gnps + GNP of each contact visit
    uint32_t* ords;             // visit ordinal of each contact visit
    int32_t cap;
    int32_t* counters;          // [0] contact visits, [1] visits of a point inside a GNP
};

// Junction distance of Find_adjacent_labels; false when the point is no contact.
__device__ __forceinline__ bool mixed_junction(const MixArgs& a, int P, int G, gnp::P3& q, double& dj, bool& inside) {
    const int cnt = a.flag[P];
    double d;
    inside = gnp::closest_point(a.V + 24 * (size_t)G, a.F + 24 * (size_t)G, gnp::P3{a.x[P], a.y[P], a.z[P]}, q, d) == -1;
    if (inside) d = a.radii[cnt] + 3.0 * a.tunnel;  // ignored: no contact
    dj = d - a.radii[cnt];
    if (dj < a.vdw) dj = a.vdw;
    return dj - a.tunnel <= gnp::kZero;
}

__global__ void k_mix_visits(int R, const int32_t* __restrict__ gptr, const int32_t* __restrict__ cptr, int64_t* __restrict__ n) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= R; t += gridDim.x * blockDim.x)
        n[t] = t < R ? (int64_t)(gptr[t + 1] - gptr[t]) * (cptr[t + 1] - cptr[t]) : 0;
}

__global__ void k_mix_eval(MixArgs a) {
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < a.n_visits; o += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = a.n_regions - 1;  // last region whose first ordinal is <= o (a region with visits)
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.visit_off[mid] <= o) lo = mid;
            else hi = mid - 1;
        }
        const int t = lo;
        const long long loc = o - a.visit_off[t];
        const int np = a.cptr[t + 1] - a.cptr[t];
        const int G = a.gidx[a.gptr[t] + (int)(loc / np)];
        const int P = a.trav_pt[a.slot[a.cptr[t] + (int)(loc % np)]];
        gnp::P3 q;
        double dj;
        bool inside;
        const bool hit = mixed_junction(a, P, G, q, dj, inside);
        if (inside) atomicAdd(&a.counters[1], 1);
        if (hit) {
            const int pos = atomicAdd(&a.counters[0], 1);
            if (pos < a.cap) {
                a.keys[pos] = (uint64_t)P * a.n_gnps + (uint32_t)G;
                a.ords[pos] = (uint32_t)o;
            }
        }
    }
}

__global__ void k_mix_heads(int n, const uint64_t* __restrict__ keys, int32_t* __restrict__ head) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// One entry per pair: its first visit ordinal (sort key) and its pair key.
__global__ void k_mix_first(int n, const uint64_t* __restrict__ keys, const uint32_t* __restrict__ ords, const int32_t* __restrict__ head,
                            const int32_t* __restrict__ pos, uint64_t* __restrict__ first, uint32_t* __restrict__ uidx,
                            uint64_t* __restrict__ upair) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        uint32_t m = ords[i];
        for (int k = i + 1; k < n && keys[k] == keys[i]; k++) m = min(m, ords[k]);
        first[pos[i]] = m;
        uidx[pos[i]] = (uint32_t)pos[i];
        upair[pos[i]] = keys[i];
    }
}

// Contact number i (pairs in first-visit order): point, GNP, junction distance, closest GNP point.
__global__ void k_mix_out(MixArgs a, int n, const uint32_t* __restrict__ uidx, const uint64_t* __restrict__ upair,
                          int32_t* __restrict__ point, int32_t* __restrict__ gnp_out, double* __restrict__ dist, double* __restrict__ closest) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t k = upair[uidx[i]];
        const int P = (int)(k / a.n_gnps), G = (int)(k % a.n_gnps);
        gnp::P3 q;
        double dj;
        bool inside;
        mixed_junction(a, P, G, q, dj, inside);
        point[i] = P;
        gnp_out[i] = G;
        dist[i] = dj;
        closest[3 * i] = q.x;
        closest[3 * i + 1] = q.y;
        closest[3 * i + 2] = q.z;
    }
}

}  // namespace

int run_gnp_cnt_contacts(Ctx& c, const GnpSet& g, const GnpGrid& grid, const cicy_params& p, int inside_is_error) {
    if (c.stage < 2) throw Fail{CICY_E_STATE, "cicy_gnp_cnt_contacts: no contact grid"};
    for (int d = 0; d < 3; d++)
        if (grid.n_regions[d] != c.grid.n[d] || grid.l_regions[d] != c.grid.l[d])
            throw Fail{CICY_E_INPUT, "cicy_gnp_cnt_contacts: the GNP grid and the contact grid have different regions"};
    const int R = (int)c.grid.total;
    if ((int)grid.ptr.size() != R + 1 || grid.ptr[R] != (int32_t)grid.idx.size())
        throw Fail{CICY_E_INPUT, "cicy_gnp_cnt_contacts: GNP grid has no region lists"};
    for (int32_t gi : grid.idx)
        if (gi < 0 || gi >= g.n) throw Fail{CICY_E_INPUT, "cicy_gnp_cnt_contacts: GNP grid names a GNP outside the set"};
    if ((unsigned long long)std::max(c.n_points, 1) * (unsigned long long)std::max(g.n, 1) >= (1ULL << 63))
        throw Fail{CICY_E_CAPACITY, "cicy_gnp_cnt_contacts: points x GNPs too large"};
    cudaStream_t s = c.stream;
    c.n_mix = 0;
    if (grid.idx.empty() || c.n_slots == 0) return 0;
    DBuf<int32_t> gptr, gidx, counters, head, pos, total;
    DBuf<int64_t> nvis, off, tot64;
    DBuf<double> V, F;
    gptr.ensure(R + 1);
    gidx.ensure(grid.idx.size());
    V.ensure(24 * (size_t)g.n);
    F.ensure(24 * (size_t)g.n);
    CICY_CUDA(cudaMemcpyAsync(gptr.get(), grid.ptr.data(), sizeof(int32_t) * (R + 1), cudaMemcpyHostToDevice, s));
    CICY_CUDA(cudaMemcpyAsync(gidx.get(), grid.idx.data(), sizeof(int32_t) * grid.idx.size(), cudaMemcpyHostToDevice, s));
    CICY_CUDA(cudaMemcpyAsync(V.get(), g.vertices.data(), sizeof(double) * 24 * g.n, cudaMemcpyHostToDevice, s));
    CICY_CUDA(cudaMemcpyAsync(F.get(), g.planes.data(), sizeof(double) * 24 * g.n, cudaMemcpyHostToDevice, s));
    nvis.ensure(R + 1);
    off.ensure(R + 1);
    tot64.ensure(1);
    k_mix_visits<<<blocks_for(R + 1), 256, 0, s>>>(R, gptr.get(), c.region_ptr.get(), nvis.get());
    DBuf<int64_t> scan64;
    exclusive_scan_i64(nvis.get(), off.get(), R + 1, tot64.get(), scan64, s, c.launches);
    int64_t T = 0;
    CICY_CUDA(cudaMemcpyAsync(&T, tot64.get(), sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    if (T >= (1LL << 31)) throw Fail{CICY_E_CAPACITY, "cicy_gnp_cnt_contacts: 2^31 or more point-GNP visits"};
    if (T == 0) return 0;
    MixArgs a{};
    a.n_regions = R;
    a.visit_off = off.get();
    a.gptr = gptr.get();
    a.gidx = gidx.get();
    a.cptr = c.region_ptr.get();
    a.slot = c.slot_sorted.get();
    a.trav_pt = c.trav_pt.get();
    a.x = c.x.get(); a.y = c.y.get(); a.z = c.z.get();
    a.radii = c.radii.get();
    a.flag = c.flag.get();
    a.V = V.get();
    a.F = F.get();
    a.vdw = p.van_der_waals_dist;
    a.tunnel = p.tunneling_dist;
    a.n_gnps = (uint32_t)g.n;
    a.n_visits = T;
    counters.ensure(2);
    DBuf<uint64_t> keys;
    DBuf<uint32_t> ords;
    int32_t h[2] = {0, 0};
    // contact visits are a small share of all visits: start with a bounded buffer, rerun once at the exact size
    long long cap = std::min<long long>(T, 1LL << 22);
    for (int attempt = 0; attempt < 2; attempt++) {
        keys.ensure(cap);
        ords.ensure(cap);
        a.keys = keys.get();
        a.ords = ords.get();
        a.cap = (int32_t)cap;
        a.counters = counters.get();
        CICY_CUDA(cudaMemsetAsync(counters.get(), 0, sizeof(int32_t) * 2, s));
        k_mix_eval<<<blocks_for(T), 256, 0, s>>>(a);
        CICY_LAUNCH_CHECK();
        c.launches += 1;
        CICY_CUDA(cudaMemcpyAsync(h, counters.get(), sizeof(int32_t) * 2, cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaStreamSynchronize(s));
        if (h[0] <= cap) break;
        cap = h[0];
    }
    if (inside_is_error && h[1] > 0)
        throw Fail{CICY_E_INPUT, "Find_adjacent_labels: a CNT point in a mixed junction is inside a GNP"};
    const int n = h[0];
    if (n == 0) return 0;
    radix_sort_pairs(keys.get(), ords.get(), n, bits_for((uint64_t)c.n_points * (uint64_t)g.n), c.rs, s, c.launches);
    head.ensure(n);
    pos.ensure(n);
    total.ensure(1);
    k_mix_heads<<<blocks_for(n), 256, 0, s>>>(n, keys.get(), head.get());
    DBuf<int32_t> scan32;
    exclusive_scan_i32(head.get(), pos.get(), n, total.get(), scan32, s, c.launches);
    int U = 0;
    CICY_CUDA(cudaMemcpyAsync(&U, total.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    DBuf<uint64_t> first, upair;
    DBuf<uint32_t> uidx;
    first.ensure(U);
    upair.ensure(U);
    uidx.ensure(U);
    k_mix_first<<<blocks_for(n), 256, 0, s>>>(n, keys.get(), ords.get(), head.get(), pos.get(), first.get(), uidx.get(), upair.get());
    radix_sort_pairs(first.get(), uidx.get(), U, bits_for((uint64_t)T), c.rs, s, c.launches);
    c.mix_point.ensure(U);
    c.mix_gnp.ensure(U);
    c.mix_dist.ensure(U);
    c.mix_closest.ensure(3 * (size_t)U);
    k_mix_out<<<blocks_for(U), 256, 0, s>>>(a, U, uidx.get(), upair.get(), c.mix_point.get(), c.mix_gnp.get(), c.mix_dist.get(),
                                           c.mix_closest.get());
    CICY_LAUNCH_CHECK();
    c.launches += 4;
    CICY_CUDA(cudaStreamSynchronize(s));
    c.n_mix = U;
    return U;
}

void gnp_sectioned_domain(const GnpSet& g, const std::vector<int32_t>& inside, const cicy_cuboid& w, const double gs_min[3],
                          double overlap_cnt, double overlap_gnp, GnpGrid& out) {
    const int n_in = (int)inside.size();
    // region grid: Generate_contact_grid + Adjust_regions_if_needed (Contact_grid.cpp:18-102)
    const double len[3] = {w.len_x, w.len_y, w.len_z};
    for (int d = 0; d < 3; d++) {
        out.n_regions[d] = std::max(1, (int)(len[d] / gs_min[d]));
        out.l_regions[d] = gs_min[d];
    }
    const double ov = std::max(overlap_cnt, overlap_gnp);
    for (int d = 0; d < 3; d++)
        if (gs_min[d] < 2 * ov) {
            out.l_regions[d] = 2.0 * (ov + 1.0e-10);
            out.n_regions[d] = 1 + (int)(len[d] / out.l_regions[d]);
        }
    const long long tot = (long long)out.n_regions[0] * out.n_regions[1] * out.n_regions[2];
    if (tot >= (1LL << 31) || tot * (long long)std::max(n_in, 1) >= (long long)kNoKey)
        throw Fail{CICY_E_CAPACITY, "cicy_gnp_sectioned_domain: regions x GNPs must stay below 2^32"};
    for (int32_t gi : inside)
        if (gi < 0 || gi >= g.n) throw Fail{CICY_E_INPUT, "cicy_gnp_sectioned_domain: a GNP index is out of range"};
    // sample counts per GNP (host: the upstream integer arithmetic) and their offsets
    std::vector<int32_t> nxyz(3 * (size_t)std::max(n_in, 1));
    std::vector<int64_t> off(n_in + 1, 0);
    for (int o = 0; o < n_in; o++) {
        const int gi = inside[o];
        const int nx = std::max(40, 1 + (int)(g.l[gi] / out.l_regions[0]));
        const int ny = std::max(40, 1 + (int)(g.l[gi] / out.l_regions[1]));
        const int nz = std::max(2, 1 + (int)(g.t[gi] / out.l_regions[2]));
        nxyz[3 * o] = nx;
        nxyz[3 * o + 1] = ny;
        nxyz[3 * o + 2] = nz;
        off[o + 1] = off[o] + (int64_t)nx * ny * nz;
    }
    const long long P = off[n_in];
    if (4 * P >= (1LL << 31)) throw Fail{CICY_E_CAPACITY, "cicy_gnp_sectioned_domain: more than 2^29 sample points"};
    out.ptr.assign(tot + 1, 0);
    out.idx.clear();
    if (n_in == 0 || P == 0) return;
    cudaStream_t s = nullptr;
    int64_t launches = 0;
    DBuf<int32_t> d_inside, d_nxyz, d_flag, d_pos, d_ptr, d_idx, d_total;
    DBuf<int64_t> d_off;
    DBuf<double> d_vert;
    DBuf<uint64_t> d_keys;
    DBuf<uint32_t> d_vals, d_uniq;
    RadixScratch rs;
    DBuf<int32_t> scan_tmp;
    d_inside.ensure(n_in);
    d_nxyz.ensure(3 * (size_t)n_in);
    d_off.ensure(n_in + 1);
    d_vert.ensure(24 * (size_t)g.n);
    CICY_CUDA(cudaMemcpy(d_inside.get(), inside.data(), sizeof(int32_t) * n_in, cudaMemcpyHostToDevice));
    CICY_CUDA(cudaMemcpy(d_nxyz.get(), nxyz.data(), sizeof(int32_t) * 3 * n_in, cudaMemcpyHostToDevice));
    CICY_CUDA(cudaMemcpy(d_off.get(), off.data(), sizeof(int64_t) * (n_in + 1), cudaMemcpyHostToDevice));
    CICY_CUDA(cudaMemcpy(d_vert.get(), g.vertices.data(), sizeof(double) * 24 * g.n, cudaMemcpyHostToDevice));
    const long long K = 4 * P;
    d_keys.ensure(K);
    d_vals.ensure(K);
    GnpGridArgs a{};
    a.n_inside = n_in;
    a.inside = d_inside.get();
    a.pt_off = d_off.get();
    a.nxyz = d_nxyz.get();
    a.vertices = d_vert.get();
    a.wmin[0] = w.min_x; a.wmin[1] = w.min_y; a.wmin[2] = w.min_z;
    a.wmax[0] = w.max_x; a.wmax[1] = w.max_y; a.wmax[2] = w.max_z;
    for (int d = 0; d < 3; d++) {
        a.nreg[d] = out.n_regions[d];
        a.lreg[d] = out.l_regions[d];
    }
    a.overlap = overlap_gnp;
    a.n_points = P;
    a.keys = d_keys.get();
    k_gnp_sample<<<blocks_for(P), 256, 0, s>>>(a);
    CICY_LAUNCH_CHECK();
    CICY_CUDA(cudaMemsetAsync(d_vals.get(), 0, sizeof(uint32_t) * K, s));
    radix_sort_pairs(d_keys.get(), d_vals.get(), (int)K, 32, rs, s, launches);
    d_flag.ensure(K);
    d_pos.ensure(K);
    d_total.ensure(1);
    k_first_of_run<<<blocks_for(K), 256, 0, s>>>(K, d_keys.get(), d_flag.get());
    exclusive_scan_i32(d_flag.get(), d_pos.get(), (int)K, d_total.get(), scan_tmp, s, launches);
    int n_unique = 0;
    CICY_CUDA(cudaMemcpy(&n_unique, d_total.get(), sizeof(int32_t), cudaMemcpyDeviceToHost));
    d_uniq.ensure(std::max(n_unique, 1));
    k_compact<<<blocks_for(K), 256, 0, s>>>(K, d_keys.get(), d_flag.get(), d_pos.get(), d_uniq.get());
    d_ptr.ensure(tot + 1);
    d_idx.ensure(std::max(n_unique, 1));
    k_region_ptr<<<blocks_for(tot + 1), 256, 0, s>>>((int)tot, n_unique, (uint32_t)n_in, d_uniq.get(), d_ptr.get());
    k_region_idx<<<blocks_for(n_unique), 256, 0, s>>>(n_unique, (uint32_t)n_in, d_inside.get(), d_uniq.get(), d_idx.get());
    CICY_LAUNCH_CHECK();
    out.idx.resize(n_unique);
    CICY_CUDA(cudaMemcpy(out.ptr.data(), d_ptr.get(), sizeof(int32_t) * (tot + 1), cudaMemcpyDeviceToHost));
    if (n_unique) CICY_CUDA(cudaMemcpy(out.idx.data(), d_idx.get(), sizeof(int32_t) * n_unique, cudaMemcpyDeviceToHost));
    out.launches = launches + 6;
}

}  // namespace cicy

// ---------------------------------------------------------------------------
extern "C" {

cicy_status cicy_gnp_sectioned_domain(int device, const cicy_gnp_set* gnps, const int32_t* inside, int32_t n_inside,
                                      const cicy_cuboid* window, const double* gs_min, double overlap_cnt, double overlap_gnp,
                                      cicy_gnp_grid** out) {
    if (!gnps || !window || !gs_min || !out || n_inside < 0 || (n_inside > 0 && !inside) || !(gs_min[0] > 0) || !(gs_min[1] > 0) ||
        !(gs_min[2] > 0) || overlap_cnt < 0 || overlap_gnp < 0) {
        cicy::set_host_error("cicy_gnp_sectioned_domain: invalid arguments");
        return CICY_E_INPUT;
    }
    cicy_gnp_grid* g = new cicy_gnp_grid;
    try {
        CICY_CUDA(cudaSetDevice(device));
        std::vector<int32_t> in(inside, inside + n_inside);
        cicy::gnp_sectioned_domain(gnps->g, in, *window, gs_min, overlap_cnt, overlap_gnp, g->grid);
    } catch (const cicy::Fail& e) {
        cicy::set_host_error(e.msg);
        delete g;
        return e.status;
    }
    *out = g;
    return CICY_OK;
}

cicy_status cicy_gnp_grid_view(const cicy_gnp_grid* g, int32_t* n_regions, double* l_regions, const int32_t** ptr, const int32_t** idx,
                               int64_t* n_entries) {
    if (!g) return CICY_E_INPUT;
    for (int d = 0; d < 3; d++) {
        if (n_regions) n_regions[d] = g->grid.n_regions[d];
        if (l_regions) l_regions[d] = g->grid.l_regions[d];
    }
    if (ptr) *ptr = g->grid.ptr.data();
    if (idx) *idx = g->grid.idx.data();
    if (n_entries) *n_entries = (int64_t)g->grid.idx.size();
    return CICY_OK;
}

void cicy_gnp_grid_free(cicy_gnp_grid* g) { delete g; }

cicy_status cicy_gnp_point_distance(int device, const cicy_gnp_set* gnps, int32_t n, const double* xyz, const int32_t* gnp, double* dist,
                                    double* closest, int32_t* flag) {
    if (!gnps || n < 0 || (n > 0 && (!xyz || !gnp || !dist || !closest || !flag))) {
        cicy::set_host_error("cicy_gnp_point_distance: invalid arguments");
        return CICY_E_INPUT;
    }
    for (int i = 0; i < n; i++)
        if (gnp[i] < 0 || gnp[i] >= gnps->g.n) {
            cicy::set_host_error("cicy_gnp_point_distance: GNP index " + std::to_string(gnp[i]) + " out of range");
            return CICY_E_INPUT;
        }
    if (n == 0) return CICY_OK;
    try {
        CICY_CUDA(cudaSetDevice(device));
        const cicy::GnpSet& g = gnps->g;
        cicy::DBuf<double> d_xyz, d_v, d_f, d_dist, d_q;
        cicy::DBuf<int32_t> d_g, d_flag;
        d_xyz.ensure(3 * (size_t)n); d_g.ensure(n); d_v.ensure(24 * (size_t)g.n); d_f.ensure(24 * (size_t)g.n);
        d_dist.ensure(n); d_q.ensure(3 * (size_t)n); d_flag.ensure(n);
        CICY_CUDA(cudaMemcpy(d_xyz.get(), xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(d_g.get(), gnp, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(d_v.get(), g.vertices.data(), sizeof(double) * 24 * g.n, cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(d_f.get(), g.planes.data(), sizeof(double) * 24 * g.n, cudaMemcpyHostToDevice));
        cicy::k_gnp_closest<<<cicy::blocks_for(n), 256>>>(n, d_xyz.get(), d_g.get(), d_v.get(), d_f.get(), d_dist.get(), d_q.get(), d_flag.get());
        CICY_LAUNCH_CHECK();
        CICY_CUDA(cudaMemcpy(dist, d_dist.get(), sizeof(double) * n, cudaMemcpyDeviceToHost));
        CICY_CUDA(cudaMemcpy(closest, d_q.get(), sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
        CICY_CUDA(cudaMemcpy(flag, d_flag.get(), sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    } catch (const cicy::Fail& e) {
        cicy::set_host_error(e.msg);
        return e.status;
    }
    return CICY_OK;
}

}  // extern "C"
