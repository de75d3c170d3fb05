// GNP-GNP distances on the device (gnp_gjk.cuh: GJK, EPA for interpenetrating
// GNPs, Hoshen_Kopelman::Get_distance_between_GNPs) for explicit pairs, and the
// GNP-GNP contact pass of Hoshen_Kopelman::Label_gnps_in_window
// (Hoshen_Kopelman.cpp:626-767) over the GNP region lists, with the junction
// points of each contact (gnp_junction.cuh).
//
// Upstream visits, region by region, every pair j < k of the region's GNPs and
// measures a pair the first time it meets it (a visited set); a pair within
// the tunnelling cutoff goes on to the junction points and the labels.  The
// distance depends on the pair only, so the contacts in upstream's order are
// the pairs within the cutoff ranked by their first visit.  On the device every
// visit emits (pair key, visit ordinal); a radix sort by pair key and a min per
// run give each pair once with its first ordinal, one thread per pair runs GJK
// / EPA (its polytope in local memory), and a sort by ordinal of the pairs
// within the cutoff gives upstream's order.  FP64 without contraction (this
// file is built with --fmad=false), so distances and directions equal
// upstream's.
#include <algorithm>
#include <string>
#include <vector>

#include "cicy_internal.h"
#include "dev_common.cuh"
#include "gnp_gjk.cuh"
#include "gnp_junction.cuh"

namespace cicy {
namespace {

int pair_blocks(long long n, int threads) { return (int)std::max(1LL, std::min((n + threads - 1) / threads, 148LL * 32)); }

constexpr int kPairThreads = 128;  // one GJK / EPA per thread; ~10 KB of polytope in local memory each

// Distance of pair i (GNPs a[i], b[i]); results by pair.
__global__ void __launch_bounds__(kPairThreads) k_pair_distance(int n, const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                                                                const double* __restrict__ V, double vdw, double* __restrict__ dist,
                                                                double* __restrict__ dir, double* __restrict__ disp,
                                                                int32_t* __restrict__ pen, int32_t* __restrict__ status) {
    gnp::Polytope T;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0.0;
        gnp::P3 N{0.0, 0.0, 0.0}, m{0.0, 0.0, 0.0};
        bool p = false;
        status[i] = gnp::pair_distance(V + 24 * (size_t)a[i], V + 24 * (size_t)b[i], vdw, T, d, N, m, p);
        dist[i] = d;
        dir[3 * i] = N.x;
        dir[3 * i + 1] = N.y;
        dir[3 * i + 2] = N.z;
        disp[3 * i] = m.x;
        disp[3 * i + 1] = m.y;
        disp[3 * i + 2] = m.z;
        pen[i] = p ? 1 : 0;
    }
}

struct Box {
    double lo[3], hi[3];
};
Box box_of(const cicy_cuboid& c) { return Box{{c.min_x, c.min_y, c.min_z}, {c.max_x, c.max_y, c.max_z}}; }

// Junction step of Label_gnps_in_window for pair i (Hoshen_Kopelman.cpp:712-746):
// the second GNP moved apart when the pair interpenetrates, the two junction
// points, the point on the second GNP moved back, and which points lie outside
// the sample (1: a's, 2: b's).  Pairs with skip[i] set are left alone.
__global__ void __launch_bounds__(kPairThreads) k_pair_junction(int n, const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                                                                const double* __restrict__ V, const double* __restrict__ F,
                                                                const double* __restrict__ dist, const double* __restrict__ dir,
                                                                const double* __restrict__ disp, const int32_t* __restrict__ pen,
                                                                const int32_t* __restrict__ take, Box box, int allow3,
                                                                double* __restrict__ pa, double* __restrict__ pb,
                                                                int32_t* __restrict__ outside, int32_t* __restrict__ status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (take && !take[i]) continue;
        gnp::Cuboid8 A, B;
        gnp::load_cuboid(V + 24 * (size_t)a[i], F + 24 * (size_t)a[i], A);
        const gnp::P3 m{disp[3 * i], disp[3 * i + 1], disp[3 * i + 2]};
        if (pen[i]) gnp::moved_cuboid(V + 24 * (size_t)b[i], m, B);
        else gnp::load_cuboid(V + 24 * (size_t)b[i], F + 24 * (size_t)b[i], B);
        gnp::P3 PA{0.0, 0.0, 0.0}, PB{0.0, 0.0, 0.0};
        const int st = gnp::junction_points(A, B, gnp::P3{dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]}, dist[i], allow3 != 0, PA, PB);
        if (st == gnp::kJuncOk && pen[i]) PB = gnp::sub(PB, m);
        pa[3 * i] = PA.x; pa[3 * i + 1] = PA.y; pa[3 * i + 2] = PA.z;
        pb[3 * i] = PB.x; pb[3 * i + 1] = PB.y; pb[3 * i + 2] = PB.z;
        outside[i] = st == gnp::kJuncOk ? (gnp::outside_box(PA, box.lo, box.hi) ? 1 : 0) + (gnp::outside_box(PB, box.lo, box.hi) ? 2 : 0) : -1;
        status[i] = st;
    }
}

__global__ void k_region_pairs(int R, const int32_t* __restrict__ gptr, int64_t* __restrict__ n) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= R; t += gridDim.x * blockDim.x) {
        const int64_t m = t < R ? gptr[t + 1] - gptr[t] : 0;
        n[t] = m * (m - 1) / 2;
    }
}

// Visit o: the pair (j, k), j < k, of its region in upstream's j-major order.
__global__ void k_pair_visits(int R, long long T, const int64_t* __restrict__ off, const int32_t* __restrict__ gptr,
                              const int32_t* __restrict__ gidx, uint32_t n_gnps, uint64_t* __restrict__ keys, uint32_t* __restrict__ ords) {
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < T; o += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = R - 1;  // last region whose first ordinal is <= o (a region with pairs)
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (off[mid] <= o) lo = mid;
            else hi = mid - 1;
        }
        const int m = gptr[lo + 1] - gptr[lo];
        long long loc = o - off[lo];
        int j = 0;
        while (loc >= m - 1 - j) {
            loc -= m - 1 - j;
            j++;
        }
        const int k = j + 1 + (int)loc;
        const uint32_t g1 = (uint32_t)gidx[gptr[lo] + j], g2 = (uint32_t)gidx[gptr[lo] + k];
        const uint32_t ga = min(g1, g2), gb = max(g1, g2);
        keys[o] = (uint64_t)ga * n_gnps + gb;
        ords[o] = (uint32_t)o;
    }
}

__global__ void k_run_heads(int n, const uint64_t* __restrict__ keys, int32_t* __restrict__ head) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// One entry per pair: GNPs and first visit ordinal (a run of equal keys is one pair).
__global__ void k_pair_first(int n, const uint64_t* __restrict__ keys, const uint32_t* __restrict__ ords, const int32_t* __restrict__ head,
                             const int32_t* __restrict__ pos, uint32_t n_gnps, int32_t* __restrict__ pa, int32_t* __restrict__ pb,
                             uint32_t* __restrict__ first) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        uint32_t mn = ords[i];
        for (int k = i + 1; k < n && keys[k] == keys[i]; k++) mn = min(mn, ords[k]);
        pa[pos[i]] = (int32_t)(keys[i] / n_gnps);
        pb[pos[i]] = (int32_t)(keys[i] % n_gnps);
        first[pos[i]] = mn;
    }
}

__global__ void k_within(int n, const double* __restrict__ dist, double tunnel, int32_t* __restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flag[i] = dist[i] <= tunnel ? 1 : 0;
}

__global__ void k_contact_keys(int n, const int32_t* __restrict__ flag, const int32_t* __restrict__ pos, const uint32_t* __restrict__ first,
                               uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) {
            keys[pos[i]] = first[i];
            vals[pos[i]] = (uint32_t)i;
        }
}

const char* status_text(int s) {
    switch (s) {
        case gnp::kGjkNoConvergence: return "GJK reached 50 iterations";
        case gnp::kGjkBadSimplex: return "GJK met a simplex of invalid size";
        case gnp::kGjkCapacity: return "the EPA polytope outgrew its fixed capacity";
        case gnp::kGjkNoHorizon: return "the EPA support point sees no face";
        default: return "unknown";
    }
}

// Distances of explicit pairs on the device; throws on the first failing pair.
struct PairBufs {
    DBuf<int32_t> a, b, pen, status, outside, jstatus;
    DBuf<double> dist, dir, disp, pa, pb;
    void ensure(size_t n) {
        a.ensure(n); b.ensure(n); pen.ensure(n); status.ensure(n); outside.ensure(n); jstatus.ensure(n);
        dist.ensure(n); dir.ensure(3 * n); disp.ensure(3 * n); pa.ensure(3 * n); pb.ensure(3 * n);
    }
};

const char* junction_text(int s) {
    switch (s) {
        case gnp::kJuncBadSimplex: return "the closest features have a vertex count upstream rejects";
        case gnp::kJuncNoIntersection: return "an edge meets a face edge outside [0, 1]";
        case gnp::kJuncNoInsideVertex: return "no vertex of one face lies inside the other";
        case gnp::kJuncNoEdge: return "no face edge for the two-intersection average";
        case gnp::kJuncBadFace: return "a vertex sum names no face";
        default: return "unknown";
    }
}

void check_pair_status(int n, const int32_t* d_status, const int32_t* d_a, const int32_t* d_b) {
    std::vector<int32_t> st(n), a(n), b(n);
    CICY_CUDA(cudaMemcpy(st.data(), d_status, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; i++)
        if (st[i] != gnp::kGjkOk) {
            CICY_CUDA(cudaMemcpy(a.data(), d_a, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
            CICY_CUDA(cudaMemcpy(b.data(), d_b, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
            throw Fail{st[i] == gnp::kGjkCapacity ? CICY_E_CAPACITY : CICY_E_INPUT,
                       "Get_distance_between_GNPs: GNPs " + std::to_string(a[i]) + " and " + std::to_string(b[i]) + ": " +
                           status_text(st[i])};
        }
}

}  // namespace

void gnp_contact_pairs(const GnpSet& g, const GnpGrid& grid, double vdw, double tunnel, const cicy_cuboid& sample, bool allow_simplex3,
                       GnpPairs& out) {
    out = GnpPairs{};
    const int R = (int)grid.ptr.size() - 1;
    if (R < 0 || grid.ptr[R] != (int32_t)grid.idx.size()) throw Fail{CICY_E_INPUT, "cicy_gnp_contact_pairs: the GNP grid has no region lists"};
    for (int t = 0; t < R; t++)
        if (grid.ptr[t + 1] < grid.ptr[t] || grid.ptr[0] != 0) throw Fail{CICY_E_INPUT, "cicy_gnp_contact_pairs: region offsets not ascending"};
    for (int32_t gi : grid.idx)
        if (gi < 0 || gi >= g.n) throw Fail{CICY_E_INPUT, "cicy_gnp_contact_pairs: the GNP grid names a GNP outside the set"};
    if (grid.idx.empty()) return;
    if ((unsigned long long)g.n * (unsigned long long)g.n >= (1ULL << 63)) throw Fail{CICY_E_CAPACITY, "cicy_gnp_contact_pairs: too many GNPs"};
    cudaStream_t s = nullptr;
    int64_t launches = 0;
    DBuf<int32_t> gptr, gidx, head, pos, total, flag;
    DBuf<int64_t> npairs, off, tot64, scan64;
    DBuf<int32_t> scan32;
    DBuf<double> V, F;
    gptr.ensure(R + 1);
    gidx.ensure(grid.idx.size());
    V.ensure(24 * (size_t)g.n);
    F.ensure(24 * (size_t)g.n);
    CICY_CUDA(cudaMemcpy(F.get(), g.planes.data(), sizeof(double) * 24 * g.n, cudaMemcpyHostToDevice));
    CICY_CUDA(cudaMemcpy(gptr.get(), grid.ptr.data(), sizeof(int32_t) * (R + 1), cudaMemcpyHostToDevice));
    CICY_CUDA(cudaMemcpy(gidx.get(), grid.idx.data(), sizeof(int32_t) * grid.idx.size(), cudaMemcpyHostToDevice));
    CICY_CUDA(cudaMemcpy(V.get(), g.vertices.data(), sizeof(double) * 24 * g.n, cudaMemcpyHostToDevice));
    npairs.ensure(R + 1);
    off.ensure(R + 1);
    tot64.ensure(1);
    k_region_pairs<<<pair_blocks(R + 1, 256), 256, 0, s>>>(R, gptr.get(), npairs.get());
    exclusive_scan_i64(npairs.get(), off.get(), R + 1, tot64.get(), scan64, s, launches);
    int64_t T = 0;
    CICY_CUDA(cudaMemcpy(&T, tot64.get(), sizeof(int64_t), cudaMemcpyDeviceToHost));
    if (T >= (1LL << 31)) throw Fail{CICY_E_CAPACITY, "cicy_gnp_contact_pairs: 2^31 or more GNP pair visits"};
    if (T == 0) return;
    DBuf<uint64_t> keys;
    DBuf<uint32_t> ords;
    keys.ensure(T);
    ords.ensure(T);
    k_pair_visits<<<pair_blocks(T, 256), 256, 0, s>>>(R, T, off.get(), gptr.get(), gidx.get(), (uint32_t)g.n, keys.get(), ords.get());
    CICY_LAUNCH_CHECK();
    RadixScratch rs;
    radix_sort_pairs(keys.get(), ords.get(), (int)T, bits_for((uint64_t)g.n * (uint64_t)g.n), rs, s, launches);
    head.ensure(T);
    pos.ensure(T);
    total.ensure(1);
    k_run_heads<<<pair_blocks(T, 256), 256, 0, s>>>((int)T, keys.get(), head.get());
    exclusive_scan_i32(head.get(), pos.get(), (int)T, total.get(), scan32, s, launches);
    int U = 0;
    CICY_CUDA(cudaMemcpy(&U, total.get(), sizeof(int32_t), cudaMemcpyDeviceToHost));
    PairBufs pb;
    pb.ensure(U);
    DBuf<uint32_t> first;
    first.ensure(U);
    k_pair_first<<<pair_blocks(T, 256), 256, 0, s>>>((int)T, keys.get(), ords.get(), head.get(), pos.get(), (uint32_t)g.n, pb.a.get(),
                                                      pb.b.get(), first.get());
    k_pair_distance<<<pair_blocks(U, kPairThreads), kPairThreads, 0, s>>>(U, pb.a.get(), pb.b.get(), V.get(), vdw, pb.dist.get(), pb.dir.get(),
                                                                          pb.disp.get(), pb.pen.get(), pb.status.get());
    CICY_LAUNCH_CHECK();
    check_pair_status(U, pb.status.get(), pb.a.get(), pb.b.get());
    // pairs within the cutoff, in first-visit order
    flag.ensure(U);
    DBuf<int32_t> fpos;
    fpos.ensure(U);
    k_within<<<pair_blocks(U, 256), 256, 0, s>>>(U, pb.dist.get(), tunnel, flag.get());
    k_pair_junction<<<pair_blocks(U, kPairThreads), kPairThreads, 0, s>>>(U, pb.a.get(), pb.b.get(), V.get(), F.get(), pb.dist.get(), pb.dir.get(),
                                                                          pb.disp.get(), pb.pen.get(), flag.get(), box_of(sample),
                                                                          allow_simplex3 ? 1 : 0, pb.pa.get(), pb.pb.get(), pb.outside.get(),
                                                                          pb.jstatus.get());
    CICY_LAUNCH_CHECK();
    exclusive_scan_i32(flag.get(), fpos.get(), U, total.get(), scan32, s, launches);
    int C = 0;
    CICY_CUDA(cudaMemcpy(&C, total.get(), sizeof(int32_t), cudaMemcpyDeviceToHost));
    out.n_visits = T;
    out.n_pairs = U;
    out.launches = launches + 8;
    if (C == 0) return;
    DBuf<uint64_t> ckeys;
    DBuf<uint32_t> cvals;
    ckeys.ensure(C);
    cvals.ensure(C);
    k_contact_keys<<<pair_blocks(U, 256), 256, 0, s>>>(U, flag.get(), fpos.get(), first.get(), ckeys.get(), cvals.get());
    radix_sort_pairs(ckeys.get(), cvals.get(), C, bits_for((uint64_t)T), rs, s, launches);
    std::vector<uint32_t> order(C);
    std::vector<int32_t> a(U), b(U), pen(U);
    std::vector<double> dist(U), dir(3 * (size_t)U), disp(3 * (size_t)U), pa(3 * (size_t)U), pbv(3 * (size_t)U);
    std::vector<int32_t> outside(U), jst(U);
    CICY_CUDA(cudaMemcpy(pa.data(), pb.pa.get(), sizeof(double) * 3 * U, cudaMemcpyDeviceToHost));
    CICY_CUDA(cudaMemcpy(pbv.data(), pb.pb.get(), sizeof(double) * 3 * U, cudaMemcpyDeviceToHost));
    CICY_CUDA(cudaMemcpy(outside.data(), pb.outside.get(), sizeof(int32_t) * U, cudaMemcpyDeviceToHost));
    CICY_CUDA(cudaMemcpy(jst.data(), pb.jstatus.get(), sizeof(int32_t) * U, cudaMemcpyDeviceToHost));
    CICY_CUDA(cudaMemcpy(order.data(), cvals.get(), sizeof(uint32_t) * C, cudaMemcpyDeviceToHost));
    CICY_CUDA(cudaMemcpy(a.data(), pb.a.get(), sizeof(int32_t) * U, cudaMemcpyDeviceToHost));
    CICY_CUDA(cudaMemcpy(b.data(), pb.b.get(), sizeof(int32_t) * U, cudaMemcpyDeviceToHost));
    CICY_CUDA(cudaMemcpy(pen.data(), pb.pen.get(), sizeof(int32_t) * U, cudaMemcpyDeviceToHost));
    CICY_CUDA(cudaMemcpy(dist.data(), pb.dist.get(), sizeof(double) * U, cudaMemcpyDeviceToHost));
    CICY_CUDA(cudaMemcpy(dir.data(), pb.dir.get(), sizeof(double) * 3 * U, cudaMemcpyDeviceToHost));
    CICY_CUDA(cudaMemcpy(disp.data(), pb.disp.get(), sizeof(double) * 3 * U, cudaMemcpyDeviceToHost));
    out.launches = launches + 9;
    for (uint32_t i : order)  // upstream stops at the first pair whose junction step fails
        if (jst[i] != gnp::kJuncOk)
            throw Fail{CICY_E_INPUT, "Find_junction_points_for_gnps: GNPs " + std::to_string(a[i]) + " and " + std::to_string(b[i]) + ": " +
                                         junction_text(jst[i])};
    for (uint32_t i : order) {
        out.point_a.insert(out.point_a.end(), {pa[3 * i], pa[3 * i + 1], pa[3 * i + 2]});
        out.point_b.insert(out.point_b.end(), {pbv[3 * i], pbv[3 * i + 1], pbv[3 * i + 2]});
        out.outside.push_back(outside[i]);
        out.a.push_back(a[i]);
        out.b.push_back(b[i]);
        out.penetrating.push_back(pen[i]);
        out.dist.push_back(dist[i]);
        out.direction.insert(out.direction.end(), {dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]});
        out.displacement.insert(out.displacement.end(), {disp[3 * i], disp[3 * i + 1], disp[3 * i + 2]});
    }
}

}  // namespace cicy

// ---------------------------------------------------------------------------
extern "C" {

cicy_status cicy_gnp_pair_distance(int device, const cicy_gnp_set* gnps, int32_t n, const int32_t* a, const int32_t* b, double vdw, double* dist,
                                   double* direction, double* displacement, int32_t* penetrating) {
    if (!gnps || n < 0 || (n > 0 && (!a || !b || !dist || !direction || !displacement || !penetrating)) || !(vdw >= 0)) {
        cicy::set_host_error("cicy_gnp_pair_distance: invalid arguments");
        return CICY_E_INPUT;
    }
    for (int i = 0; i < n; i++)
        if (a[i] < 0 || a[i] >= gnps->g.n || b[i] < 0 || b[i] >= gnps->g.n) {
            cicy::set_host_error("cicy_gnp_pair_distance: GNP index out of range in pair " + std::to_string(i));
            return CICY_E_INPUT;
        }
    if (n == 0) return CICY_OK;
    try {
        CICY_CUDA(cudaSetDevice(device));
        const cicy::GnpSet& g = gnps->g;
        cicy::PairBufs pb;
        cicy::DBuf<double> V;
        pb.ensure(n);
        V.ensure(24 * (size_t)g.n);
        CICY_CUDA(cudaMemcpy(pb.a.get(), a, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(pb.b.get(), b, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(V.get(), g.vertices.data(), sizeof(double) * 24 * g.n, cudaMemcpyHostToDevice));
        cicy::k_pair_distance<<<cicy::pair_blocks(n, cicy::kPairThreads), cicy::kPairThreads>>>(
            n, pb.a.get(), pb.b.get(), V.get(), vdw, pb.dist.get(), pb.dir.get(), pb.disp.get(), pb.pen.get(), pb.status.get());
        CICY_LAUNCH_CHECK();
        cicy::check_pair_status(n, pb.status.get(), pb.a.get(), pb.b.get());
        CICY_CUDA(cudaMemcpy(dist, pb.dist.get(), sizeof(double) * n, cudaMemcpyDeviceToHost));
        CICY_CUDA(cudaMemcpy(direction, pb.dir.get(), sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
        CICY_CUDA(cudaMemcpy(displacement, pb.disp.get(), sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
        CICY_CUDA(cudaMemcpy(penetrating, pb.pen.get(), sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    } catch (const cicy::Fail& e) {
        cicy::set_host_error(e.msg);
        return e.status;
    }
    return CICY_OK;
}

cicy_status cicy_gnp_junction_points(int device, const cicy_gnp_set* gnps, int32_t n, const int32_t* a, const int32_t* b, double vdw,
                                     const cicy_cuboid* sample, int32_t allow_simplex3, double* point_a, double* point_b, int32_t* outside,
                                     int32_t* status) {
    if (!gnps || !sample || n < 0 || (n > 0 && (!a || !b || !point_a || !point_b || !outside || !status)) || !(vdw >= 0)) {
        cicy::set_host_error("cicy_gnp_junction_points: invalid arguments");
        return CICY_E_INPUT;
    }
    for (int i = 0; i < n; i++)
        if (a[i] < 0 || a[i] >= gnps->g.n || b[i] < 0 || b[i] >= gnps->g.n) {
            cicy::set_host_error("cicy_gnp_junction_points: GNP index out of range in pair " + std::to_string(i));
            return CICY_E_INPUT;
        }
    if (n == 0) return CICY_OK;
    try {
        CICY_CUDA(cudaSetDevice(device));
        const cicy::GnpSet& g = gnps->g;
        cicy::PairBufs pb;
        cicy::DBuf<double> V, F;
        pb.ensure(n);
        V.ensure(24 * (size_t)g.n);
        F.ensure(24 * (size_t)g.n);
        CICY_CUDA(cudaMemcpy(pb.a.get(), a, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(pb.b.get(), b, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(V.get(), g.vertices.data(), sizeof(double) * 24 * g.n, cudaMemcpyHostToDevice));
        CICY_CUDA(cudaMemcpy(F.get(), g.planes.data(), sizeof(double) * 24 * g.n, cudaMemcpyHostToDevice));
        const int blocks = cicy::pair_blocks(n, cicy::kPairThreads);
        cicy::k_pair_distance<<<blocks, cicy::kPairThreads>>>(n, pb.a.get(), pb.b.get(), V.get(), vdw, pb.dist.get(), pb.dir.get(), pb.disp.get(),
                                                             pb.pen.get(), pb.status.get());
        CICY_LAUNCH_CHECK();
        cicy::check_pair_status(n, pb.status.get(), pb.a.get(), pb.b.get());
        cicy::k_pair_junction<<<blocks, cicy::kPairThreads>>>(n, pb.a.get(), pb.b.get(), V.get(), F.get(), pb.dist.get(), pb.dir.get(), pb.disp.get(),
                                                             pb.pen.get(), nullptr, cicy::box_of(*sample), allow_simplex3 ? 1 : 0, pb.pa.get(),
                                                             pb.pb.get(), pb.outside.get(), pb.jstatus.get());
        CICY_LAUNCH_CHECK();
        CICY_CUDA(cudaMemcpy(point_a, pb.pa.get(), sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
        CICY_CUDA(cudaMemcpy(point_b, pb.pb.get(), sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
        CICY_CUDA(cudaMemcpy(outside, pb.outside.get(), sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        CICY_CUDA(cudaMemcpy(status, pb.jstatus.get(), sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    } catch (const cicy::Fail& e) {
        cicy::set_host_error(e.msg);
        return e.status;
    }
    return CICY_OK;
}

cicy_status cicy_gnp_contact_pairs(int device, const cicy_gnp_set* gnps, const cicy_gnp_grid* grid, double vdw, double tunnel,
                                   const cicy_cuboid* sample, int32_t allow_simplex3, cicy_gnp_pairs** out) {
    if (!gnps || !grid || !out || !sample || !(vdw >= 0) || !(tunnel >= 0)) {
        cicy::set_host_error("cicy_gnp_contact_pairs: invalid arguments");
        return CICY_E_INPUT;
    }
    *out = nullptr;
    cicy_gnp_pairs* p = new cicy_gnp_pairs;
    try {
        CICY_CUDA(cudaSetDevice(device));
        cicy::gnp_contact_pairs(gnps->g, grid->grid, vdw, tunnel, *sample, allow_simplex3 != 0, p->pairs);
    } catch (const cicy::Fail& e) {
        cicy::set_host_error(e.msg);
        delete p;
        return e.status;
    }
    *out = p;
    return CICY_OK;
}

cicy_status cicy_gnp_pairs_view(const cicy_gnp_pairs* p, cicy_gnp_pair_list* view) {
    if (!p || !view) return CICY_E_INPUT;
    const cicy::GnpPairs& q = p->pairs;
    view->n = (int64_t)q.a.size();
    view->n_visits = q.n_visits;
    view->n_pairs = q.n_pairs;
    view->a = q.a.data();
    view->b = q.b.data();
    view->penetrating = q.penetrating.data();
    view->dist = q.dist.data();
    view->direction = q.direction.data();
    view->displacement = q.displacement.data();
    view->point_a = q.point_a.data();
    view->point_b = q.point_b.data();
    view->outside = q.outside.data();
    return CICY_OK;
}

void cicy_gnp_pairs_free(cicy_gnp_pairs* p) { delete p; }

}  // extern "C"
