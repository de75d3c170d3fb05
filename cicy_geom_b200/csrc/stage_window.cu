// Network construction on the device, before the contact grid:
//  * the seeded CNT generator (the Philox-4x32-10 streams of the host generator,
//    one thread per CNT), and
//  * the window-0 extraction of a single-window run: Shells::Generate_shells /
//    Find_shell (Shells.cpp:21-149) and Cutoff_Wins::Trim_boundary_cnts
//    (Cutoff_Wins.cpp:82-276), Add_cnt_segment_to_structure (:298-467),
//    Substitute_boundary_point (:468-548), Where_is (:554-566),
//    Where_is_with_boundary (:683-743), Add_cnt_point_to_boundary_vectors
//    (:745-769) and Fill_cnts_inside (:803-831), CNT_wires branch.
//
// Upstream trims the CNTs of shell 0 one after another.  A CNT's trim reads and
// writes only its own points, so here one thread replays it per CNT; what is
// global in upstream's loop is rebuilt from counts:
//  * a CNT that leaves and re-enters the window is cut into pieces that take
//    new indices n_cnts, n_cnts + 1, ... in shell-0 order: the trim marks the
//    pieces' points with a placeholder flag (-m for the m-th segment) and an
//    exclusive scan of the pieces per CNT gives the indices afterwards;
//  * the pieces join shell 0 (their end points lie on the window) and upstream's
//    loop trims them again after all original CNTs: a second kernel replays that
//    pass per CNT over its own pieces, in order;
//  * the boundary point / CNT lists of each face are appended in processing
//    order: per (face, unit) counts in face-major order, one scan, a scatter,
//    and the CNT lists' "skip when equal to the last entry" as a run-length
//    compaction.
// FP64 without contraction (--fmad=false), so the coordinates equal the host
// restatement's bit for bit.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "cicy_internal.h"
#include "ctx.cuh"
#include "trace.cuh"
#include "window_trim.cuh"

namespace cicy {

namespace {

using namespace win;

__global__ void k_win_layout(int nc, const int32_t* __restrict__ cstart, const int32_t* __restrict__ clen,
                             const int32_t* __restrict__ expect, const int32_t* __restrict__ flag, int* __restrict__ err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x)
        if (!layout_ok(i, cstart, clen, expect, flag)) atomicCAS(err, 0, (int)WIN_LAYOUT);
}

__global__ void k_win_trim(int nc, WinGeom g, Pts p, const int32_t* __restrict__ cstart, const int32_t* __restrict__ clen,
                           int32_t* __restrict__ npieces, int32_t* __restrict__ first, int32_t* __restrict__ slots,
                           int64_t* __restrict__ ev, int32_t* __restrict__ nev, int* __restrict__ err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        const int e = trim_cnt(i, g, p, cstart, clen, npieces, first, slots, ev, nev);
        if (e) atomicCAS(err, 0, e);
    }
}

__global__ void k_win_pieces(int nc, WinGeom g, Pts p, const int32_t* __restrict__ npieces, const int32_t* __restrict__ pbase,
                             const int32_t* __restrict__ slots, const double* __restrict__ radii, int32_t* __restrict__ prun,
                             int32_t* __restrict__ pparent, int64_t* __restrict__ pev, int32_t* __restrict__ pnev,
                             double* __restrict__ rad_out, int* __restrict__ err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        const int e = trim_pieces(i, nc, g, p, npieces, pbase, slots, radii, prun, pparent, pev, pnev, rad_out);
        if (e) atomicCAS(err, 0, e);
    }
}

__global__ void k_win_flags(int nc, const int32_t* __restrict__ cstart, const int32_t* __restrict__ clen,
                            const int32_t* __restrict__ npieces, const int32_t* __restrict__ pbase, int32_t* __restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x)
        fix_flags(i, nc, cstart, clen, npieces, pbase, flag);
}

__global__ void k_win_face_counts(int nc, int npc, const int64_t* __restrict__ ev, const int32_t* __restrict__ nev,
                                  const int64_t* __restrict__ pev, const int32_t* __restrict__ pnev, int32_t* __restrict__ cnt) {
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < nc + npc; u += gridDim.x * blockDim.x)
        face_counts(u, nc, npc, ev, nev, pev, pnev, cnt);
}

__global__ void k_win_scatter(int nc, int npc, const int64_t* __restrict__ ev, const int32_t* __restrict__ nev,
                              const int64_t* __restrict__ pev, const int32_t* __restrict__ pnev, const int32_t* __restrict__ pbase,
                              const int32_t* __restrict__ off, int32_t* __restrict__ raw_p, int32_t* __restrict__ raw_c) {
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < nc + npc; u += gridDim.x * blockDim.x)
        scatter_events(u, nc, npc, ev, nev, pev, pnev, pbase, off, raw_p, raw_c);
}

struct FaceStarts {
    int s[7];
};

__global__ void k_win_keep(int T, FaceStarts f, const int32_t* __restrict__ raw_c, int32_t* __restrict__ keep) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) keep[t] = keep_entry(t, f.s, raw_c);
}

__global__ void k_win_compact(int T, const int32_t* __restrict__ keep, const int32_t* __restrict__ pos, const int32_t* __restrict__ raw_c,
                              int32_t* __restrict__ out) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x)
        if (keep[t]) out[pos[t]] = raw_c[t];
}

__global__ void k_win_runs(int nc, int npc, const int32_t* __restrict__ first, const int32_t* __restrict__ prun, int32_t* __restrict__ cs,
                           int32_t* __restrict__ cl, int32_t* __restrict__ inside_flag, int* __restrict__ err) {
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < nc + npc; u += gridDim.x * blockDim.x)
        if (final_run(u, nc, first, prun, cs, cl, inside_flag)) atomicCAS(err, 0, (int)WIN_ONE_POINT);
}

__global__ void k_win_inside(int U, const int32_t* __restrict__ flag, const int32_t* __restrict__ pos, const int32_t* __restrict__ cl,
                             int32_t* __restrict__ inside, int32_t* __restrict__ len_of_inside) {
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < U; u += gridDim.x * blockDim.x)
        if (flag[u]) {
            inside[pos[u]] = u;
            len_of_inside[pos[u]] = cl[u];
        }
}

__global__ void k_copy_f64(int n, const double* __restrict__ in, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = in[i];
}

// ---------------------------------------------------------------------------
// Generator: the host generator's Philox-4x32-10 streams (stream = CNT index,
// draw 0: length, 1-2: start, 3: initial direction, 3 + k: the k-th turn).
struct PhiloxDev {
    uint32_t k0, k1;
    __device__ void uniform2(uint32_t s, uint32_t d, double& u0, double& u1) const {
        uint32_t c0 = s, c1 = d, c2 = 0x43494359u, c3 = 0x42323030u;
        uint32_t key0 = k0, key1 = k1;
#pragma unroll
        for (int r = 0; r < 10; r++) {
            const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
            const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
            const uint32_t n0 = hi1 ^ c1 ^ key0, n2 = hi0 ^ c3 ^ key1;
            c0 = n0;
            c1 = lo1;
            c2 = n2;
            c3 = lo0;
            key0 += 0x9E3779B9u;
            key1 += 0xBB67AE85u;
        }
        const uint64_t a = ((uint64_t)c0 << 32) | c1, b = ((uint64_t)c2 << 32) | c3;
        u0 = (double)(a >> 11) * (1.0 / 9007199254740992.0);
        u1 = (double)(b >> 11) * (1.0 / 9007199254740992.0);
    }
};

__global__ void k_gen_counts(int nc, PhiloxDev rng, cicy_gen_params g, int32_t* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        double u0, u1;
        rng.uniform2((uint32_t)i, 0, u0, u1);
        const double L = g.len_min + u0 * (g.len_max - g.len_min);
        cnt[i] = 1 + (int)floor(L / g.step);
    }
}

__global__ void k_gen_fill(int nc, PhiloxDev rng, cicy_gen_params g, const int32_t* __restrict__ start, const int32_t* __restrict__ len,
                           double* __restrict__ x, double* __restrict__ y, double* __restrict__ z, int32_t* __restrict__ flag,
                           double* __restrict__ radii) {
    const double two_pi = 6.283185307179586476925286766559;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        double u0, u1, u2, u3, v0, v1;
        rng.uniform2((uint32_t)i, 1, u0, u1);
        rng.uniform2((uint32_t)i, 2, u2, u3);
        double px = g.sample.min_x + u0 * g.sample.len_x;
        double py = g.sample.min_y + u1 * g.sample.len_y;
        double pz = g.sample.min_z + u2 * g.sample.len_z;
        rng.uniform2((uint32_t)i, 3, v0, v1);
        const double ct = 2.0 * v0 - 1.0;
        const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
        const double ph = two_pi * v1;
        double dx = st * cos(ph), dy = st * sin(ph), dz = ct;
        const int b = start[i], np = len[i];
        radii[i] = g.radius;
        x[b] = px; y[b] = py; z[b] = pz; flag[b] = i;
        for (int k = 1; k < np; k++) {
            double w0, w1;
            rng.uniform2((uint32_t)i, 3u + (uint32_t)k, w0, w1);
            const double th = w0 * g.max_turn_rad;
            const double az = two_pi * w1;
            double ax, ay, az_;
            if (fabs(dx) < 0.9) { ax = 1; ay = 0; az_ = 0; } else { ax = 0; ay = 1; az_ = 0; }
            double e1x = ay * dz - az_ * dy, e1y = az_ * dx - ax * dz, e1z = ax * dy - ay * dx;
            const double n1 = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
            e1x /= n1; e1y /= n1; e1z /= n1;
            const double e2x = dy * e1z - dz * e1y, e2y = dz * e1x - dx * e1z, e2z = dx * e1y - dy * e1x;
            const double c = cos(th), s = sin(th), ca = cos(az), sa = sin(az);
            const double nx = c * dx + s * (ca * e1x + sa * e2x);
            const double ny = c * dy + s * (ca * e1y + sa * e2y);
            const double nz = c * dz + s * (ca * e1z + sa * e2z);
            const double nn = sqrt(nx * nx + ny * ny + nz * nz);
            dx = nx / nn; dy = ny / nn; dz = nz / nn;
            px = px + g.step * dx;
            py = py + g.step * dy;
            pz = pz + g.step * dz;
            x[b + k] = px; y[b + k] = py; z[b + k] = pz; flag[b + k] = i;
        }
    }
}

int grid_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)b;
}

void win_check(Ctx& c, const char* where) {
    const int e = read_i32(c, c.win_cnt.get() + 0);
    if (e == WIN_OK) return;
    if (e == WIN_NOT_AT_BOUNDARY)
        throw Fail{CICY_E_INPUT, "Error: point should be at boundary but it is not (Cutoff_Wins::Add_cnt_point_to_boundary_vectors)"};
    if (e == WIN_CAPACITY)
        throw Fail{CICY_E_CAPACITY, std::string(where) + ": a CNT is cut into more than " + std::to_string(kMaxSeg) + " segments"};
    if (e == WIN_ONE_POINT) throw Fail{CICY_E_INPUT, "Error in Extract_observation_window. A CNT has only one point."};
    if (e == WIN_LAYOUT)
        throw Fail{CICY_E_INPUT, std::string(where) +
                                     ": the network is not in generator / Read_Network layout (CNT i must be the i-th run of "
                                     "consecutive point ids, every point flagged with its CNT)"};
    throw Fail{CICY_E_INTERNAL, std::string(where) + ": window trim status " + std::to_string(e)};
}

}  // namespace

// Window 0 of a single-window run, trimmed in place on the context's network.
void extract_window_device(Ctx& c, const cicy_window_params& w) {
    const char* where = "cicy_ctx_extract_window";
    if (c.stage < 1) throw Fail{CICY_E_STATE, std::string(where) + ": no network on the device"};
    if (w.min_points < 2) throw Fail{CICY_E_INPUT, std::string(where) + ": min_points below 2 is not supported on the device"};
    cudaStream_t s = c.stream;
    CICY_TRACE("extract_window", s);
    WinGeom g{};
    cicy_cuboid win{};
    if (!window_geom(w, g, win))
        throw Fail{CICY_E_INPUT, std::string(where) + ": only single-window runs (win_max == win_min, cut_num = 0) are supported"};

    const int nc = c.n_cnts;
    Pts p{c.x.get(), c.y.get(), c.z.get(), c.flag.get()};
    // word 0 of win_cnt: error; the per-CNT arrays follow
    c.win_cnt.ensure(8 + 2 * (size_t)std::max(nc, 1) + 2);
    int32_t* err = c.win_cnt.get();
    int32_t* npieces = err + 8;
    int32_t* pbase = npieces + std::max(nc, 1) + 1;
    c.win_first.ensure(2 * (size_t)std::max(nc, 1));
    c.win_slot.ensure((size_t)std::max(nc, 1) * kSlot);
    c.win_ev.ensure((size_t)std::max(nc, 1) * kMaxEv);
    c.win_nev.ensure(std::max(nc, 1));
    CICY_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t) * 8, s));
    if (nc > 0) {
        // layout check: the runs follow one another in CNT order, flags are the CNT indices
        exclusive_scan_i32(c.clen.get(), pbase, nc, npieces, c.scan_tmp32, s, c.launches);
        k_win_layout<<<grid_for(nc), 256, 0, s>>>(nc, c.cstart.get(), c.clen.get(), pbase, c.flag.get(), err);
        k_win_trim<<<grid_for(nc, 128), 128, 0, s>>>(nc, g, p, c.cstart.get(), c.clen.get(), npieces, c.win_first.get(), c.win_slot.get(),
                                                     c.win_ev.get(), c.win_nev.get(), err);
        c.launches += 2;
        CICY_LAUNCH_CHECK();
    }
    win_check(c, where);
    exclusive_scan_i32(npieces, pbase, std::max(nc, 1), pbase + std::max(nc, 1), c.scan_tmp32, s, c.launches);
    const int npc = nc > 0 ? read_i32(c, pbase + std::max(nc, 1)) : 0;
    const int U = nc + npc;
    c.win_prun.ensure(2 * (size_t)std::max(npc, 1));
    c.win_pparent.ensure(std::max(npc, 1));
    c.win_pev.ensure(2 * (size_t)std::max(npc, 1));
    c.win_pnev.ensure(std::max(npc, 1));
    c.win_rad.ensure(std::max(U, 1));
    if (nc > 0) {
        k_copy_f64<<<grid_for(nc), 256, 0, s>>>(nc, c.radii.get(), c.win_rad.get());
        k_win_pieces<<<grid_for(nc, 128), 128, 0, s>>>(nc, g, p, npieces, pbase, c.win_slot.get(), c.radii.get(), c.win_prun.get(),
                                                       c.win_pparent.get(), c.win_pev.get(), c.win_pnev.get(), c.win_rad.get(), err);
        k_win_flags<<<grid_for(nc), 256, 0, s>>>(nc, c.cstart.get(), c.clen.get(), npieces, pbase, c.flag.get());
        c.launches += 3;
        CICY_LAUNCH_CHECK();
    }
    // boundary lists: counts per (face, unit), scan, scatter
    const size_t F = 6 * (size_t)std::max(U, 1);
    c.win_face.ensure(F + 1);
    c.win_off.ensure(F + 1);
    k_win_face_counts<<<grid_for(U), 256, 0, s>>>(nc, npc, c.win_ev.get(), c.win_nev.get(), c.win_pev.get(), c.win_pnev.get(),
                                                  c.win_face.get());
    exclusive_scan_i32(c.win_face.get(), c.win_off.get(), 6 * U, c.win_off.get() + 6 * U, c.scan_tmp32, s, c.launches);
    std::vector<int32_t> off7(7, 0);
    for (int b = 0; b <= 6; b++)
        CICY_CUDA(cudaMemcpyAsync(&off7[b], c.win_off.get() + (size_t)b * U, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    win_check(c, where);  // synchronizes (the face offsets are read) and reports a failed piece trim
    const int T = off7[6];
    c.win_raw_p.ensure(std::max(T, 1));
    c.win_raw_c.ensure(std::max(T, 1));
    // sized for both uses (the face lists' keep flags, then the inside flags of the U CNTs)
    c.win_keep.ensure(std::max({T, U, 1}) + 1);
    c.win_pos.ensure(std::max({T, U, 1}) + 1);
    k_win_scatter<<<grid_for(U), 256, 0, s>>>(nc, npc, c.win_ev.get(), c.win_nev.get(), c.win_pev.get(), c.win_pnev.get(), pbase,
                                              c.win_off.get(), c.win_raw_p.get(), c.win_raw_c.get());
    FaceStarts fs{};
    for (int b = 0; b < 7; b++) fs.s[b] = off7[b];
    k_win_keep<<<grid_for(T), 256, 0, s>>>(T, fs, c.win_raw_c.get(), c.win_keep.get());
    exclusive_scan_i32(c.win_keep.get(), c.win_pos.get(), T, c.win_pos.get() + T, c.scan_tmp32, s, c.launches);
    c.launches += 3;
    CICY_LAUNCH_CHECK();
    std::vector<int32_t> pos7(7, 0);
    for (int b = 0; b <= 6; b++) CICY_CUDA(cudaMemcpyAsync(&pos7[b], c.win_pos.get() + off7[b], sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    // final runs, Fill_cnts_inside
    c.win_cs.ensure(std::max(U, 1));
    c.win_cl.ensure(std::max(U, 1));
    c.bcnt_idx.ensure(std::max(T, 1));
    k_win_compact<<<grid_for(T), 256, 0, s>>>(T, c.win_keep.get(), c.win_pos.get(), c.win_raw_c.get(), c.bcnt_idx.get());
    CICY_CUDA(cudaStreamSynchronize(s));  // pos7 read before the keep flags and positions are reused below
    k_win_runs<<<grid_for(U), 256, 0, s>>>(nc, npc, c.win_first.get(), c.win_prun.get(), c.win_cs.get(), c.win_cl.get(), c.win_keep.get(),
                                           err);
    exclusive_scan_i32(c.win_keep.get(), c.win_pos.get(), U, c.win_pos.get() + U, c.scan_tmp32, s, c.launches);
    c.launches += 2;
    CICY_LAUNCH_CHECK();
    const int n_inside = read_i32(c, c.win_pos.get() + U);
    win_check(c, where);
    // the trimmed network replaces the uploaded one
    c.n_cnts = U;
    c.n_inside = n_inside;
    c.window = win;
    c.cstart.ensure(std::max(U, 1));
    c.clen.ensure(std::max(U, 1));
    c.radii.ensure(std::max(U, 1));
    c.inside.ensure(std::max(n_inside, 1));
    c.trav_off.ensure(n_inside + 1);
    CICY_CUDA(cudaMemcpyAsync(c.cstart.get(), c.win_cs.get(), sizeof(int32_t) * U, cudaMemcpyDeviceToDevice, s));
    CICY_CUDA(cudaMemcpyAsync(c.clen.get(), c.win_cl.get(), sizeof(int32_t) * U, cudaMemcpyDeviceToDevice, s));
    CICY_CUDA(cudaMemcpyAsync(c.radii.get(), c.win_rad.get(), sizeof(double) * U, cudaMemcpyDeviceToDevice, s));
    k_win_inside<<<grid_for(U), 256, 0, s>>>(U, c.win_keep.get(), c.win_pos.get(), c.win_cl.get(), c.inside.get(), c.trav_off.get());
    exclusive_scan_i32(c.trav_off.get(), c.trav_off.get(), n_inside, c.trav_off.get() + n_inside, c.scan_tmp32, s, c.launches);
    c.launches += 1;
    CICY_LAUNCH_CHECK();
    c.bpts_idx.ensure(std::max(T, 1));
    CICY_CUDA(cudaMemcpyAsync(c.bpts_idx.get(), c.win_raw_p.get(), sizeof(int32_t) * T, cudaMemcpyDeviceToDevice, s));
    c.h_bcnt_ptr.assign(pos7.begin(), pos7.end());
    c.h_bpts_ptr.assign(off7.begin(), off7.end());
    c.bcnt_ptr.ensure(7);
    c.bpts_ptr.ensure(7);
    CICY_CUDA(cudaMemcpyAsync(c.bcnt_ptr.get(), c.h_bcnt_ptr.data(), sizeof(int32_t) * 7, cudaMemcpyHostToDevice, s));
    CICY_CUDA(cudaMemcpyAsync(c.bpts_ptr.get(), c.h_bpts_ptr.data(), sizeof(int32_t) * 7, cudaMemcpyHostToDevice, s));
    c.h_cstart.resize(U);
    c.h_clen.resize(U);
    if (U) {
        CICY_CUDA(cudaMemcpyAsync(c.h_cstart.data(), c.win_cs.get(), sizeof(int32_t) * U, cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaMemcpyAsync(c.h_clen.data(), c.win_cl.get(), sizeof(int32_t) * U, cudaMemcpyDeviceToHost, s));
    }
    int32_t ntrav = 0;
    CICY_CUDA(cudaMemcpyAsync(&ntrav, c.trav_off.get() + n_inside, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CICY_CUDA(cudaStreamSynchronize(s));
    c.n_trav = ntrav;
    c.stage = 1;
    c.have_backbone = false;
    c.have_volumes = false;
    c.have_hybrid = false;
}

// Seeded CNT network generated on the device into the context (the layout the
// generator and Read_Network emit: CNT i is the i-th run of points, window = sample).
void generate_network_device(Ctx& c, const cicy_gen_params& g) {
    const char* where = "cicy_ctx_generate_cnt_network";
    if (g.n_cnts < 0 || !(g.step > 0) || !(g.len_max >= g.len_min) || !(g.len_min >= 0))
        throw Fail{CICY_E_INPUT, std::string(where) + ": invalid generator parameters"};
    if ((double)g.len_max / g.step >= (double)(1 << 30))
        throw Fail{CICY_E_CAPACITY, std::string(where) + ": 2^30 or more points per CNT"};
    cudaStream_t s = c.stream;
    CICY_TRACE("generate_network", s);
    const int nc = g.n_cnts;
    const PhiloxDev rng{(uint32_t)(g.seed & 0xffffffffu), (uint32_t)(g.seed >> 32)};
    c.clen.ensure(std::max(nc, 1));
    c.cstart.ensure(std::max(nc, 1) + 1);
    c.i64_scalar.ensure(8);
    c.i32_scalar.ensure(8);
    c.status.ensure(1);
    c.radii.ensure(std::max(nc, 1));
    int64_t np = 0;
    if (nc > 0) {
        k_gen_counts<<<grid_for(nc), 256, 0, s>>>(nc, rng, g, c.clen.get());
        CICY_LAUNCH_CHECK();
        // the total in 64 bits first: an int32 scan must not wrap
        std::vector<int32_t> h(nc);
        CICY_CUDA(cudaMemcpyAsync(h.data(), c.clen.get(), sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaStreamSynchronize(s));
        for (int i = 0; i < nc; i++) np += h[i];
        if (np >= (1LL << 31) - 1) throw Fail{CICY_E_CAPACITY, std::string(where) + ": 2^31 or more points"};
        exclusive_scan_i32(c.clen.get(), c.cstart.get(), nc, c.cstart.get() + nc, c.scan_tmp32, s, c.launches);
    }
    const size_t npts = std::max<int64_t>(np, 1);
    c.x.ensure(npts); c.y.ensure(npts); c.z.ensure(npts); c.flag.ensure(npts);
    if (nc > 0) {
        k_gen_fill<<<grid_for(nc, 128), 128, 0, s>>>(nc, rng, g, c.cstart.get(), c.clen.get(), c.x.get(), c.y.get(), c.z.get(),
                                                     c.flag.get(), c.radii.get());
        c.launches += 2;
        CICY_LAUNCH_CHECK();
    }
    c.n_points = (int)np;
    c.n_cnts = nc;
    c.n_inside = 0;
    c.n_trav = 0;
    c.window = g.sample;
    c.h_bcnt_ptr.assign(7, 0);
    c.h_bpts_ptr.assign(7, 0);
    c.bcnt_ptr.ensure(7); c.bpts_ptr.ensure(7);
    c.bcnt_idx.ensure(1); c.bpts_idx.ensure(1);
    c.inside.ensure(1);
    c.trav_off.ensure(1);
    CICY_CUDA(cudaMemsetAsync(c.bcnt_ptr.get(), 0, sizeof(int32_t) * 7, s));
    CICY_CUDA(cudaMemsetAsync(c.bpts_ptr.get(), 0, sizeof(int32_t) * 7, s));
    CICY_CUDA(cudaMemsetAsync(c.trav_off.get(), 0, sizeof(int32_t), s));
    CICY_CUDA(cudaMemsetAsync(c.status.get(), 0, sizeof(int), s));
    c.h_cstart.resize(nc);
    c.h_clen.resize(nc);
    if (nc) {
        CICY_CUDA(cudaMemcpyAsync(c.h_cstart.data(), c.cstart.get(), sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaMemcpyAsync(c.h_clen.data(), c.clen.get(), sizeof(int32_t) * nc, cudaMemcpyDeviceToHost, s));
    }
    CICY_CUDA(cudaStreamSynchronize(s));
    c.stage = 1;
    c.have_backbone = false;
    c.have_volumes = false;
    c.have_hybrid = false;
}

}  // namespace cicy
