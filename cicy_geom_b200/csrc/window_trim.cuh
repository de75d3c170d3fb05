// Window-0 trimming of a single-window run as host/device code (one call per
// CNT or per list entry; stage_window.cu launches them as kernels).  Restates
// Shells::Find_shell / Find_minimum_shell (Shells.cpp:120-149) and
// Cutoff_Wins::Trim_boundary_cnts (Cutoff_Wins.cpp:82-276),
// Add_cnt_segment_to_structure (:298-467), Substitute_boundary_point (:468-548),
// Where_is (:554-566), Where_is_with_boundary (:683-743),
// Add_cnt_point_to_boundary_vectors (:745-769) and Fill_cnts_inside (:803-831),
// CNT_wires branch, for a network whose CNT i is the i-th run of consecutive
// points.  Built without FMA contraction (nvcc --fmad=false, g++
// -ffp-contract=off), so device and host builds round alike.
#pragma once

#include <cmath>
#include <cstdint>

#include "../../include/cicy_b200.h"

namespace cicy {
namespace win {

constexpr double kZero = 1.0e-10;  // MathMatrix.h:18
constexpr int kMaxSeg = 16;        // segments one CNT may be cut into by the window
constexpr int kMaxEv = 2 * kMaxSeg;
constexpr int kSlot = 3 * (kMaxSeg - 1);  // (start, end, in shell 0) of each new piece of one CNT

// error codes (device word)
enum WinErr : int { WIN_OK = 0, WIN_NOT_AT_BOUNDARY = 1, WIN_CAPACITY = 2, WIN_INTERNAL = 3, WIN_ONE_POINT = 4, WIN_LAYOUT = 5 };

enum Loc : int { L_INSIDE = 0, L_OUTSIDE = 1, L_BOUNDARY = 2 };

struct WinGeom {
    double mn[3], mx[3];                        // window (Geom_sample::ex_win_*)
    double mid[3], layer[3], core[3], half[3];  // Shells::Generate_shells
    int n_shells;
    double step_cutoff;
    int min_points;
};

struct Pts {
    double* x;
    double* y;
    double* z;
    int32_t* flag;
    __host__ __device__ void copy(int to, int from) const {
        x[to] = x[from];
        y[to] = y[from];
        z[to] = z[from];
        flag[to] = flag[from];
    }
};

// Point_3D::is_at_cuboid_boundary / is_outside_cuboid (Geometry_3D.cpp:227-246) and Where_is
__host__ __device__ inline int where_is(const WinGeom& g, const Pts& p, int i) {
    const double px = p.x[i], py = p.y[i], pz = p.z[i];
    if (fabs(px - g.mn[0]) < kZero || fabs(px - g.mx[0]) < kZero || fabs(py - g.mn[1]) < kZero || fabs(py - g.mx[1]) < kZero ||
        fabs(pz - g.mn[2]) < kZero || fabs(pz - g.mx[2]) < kZero)
        return L_BOUNDARY;
    if ((px - g.mn[0] < kZero) || (px - g.mx[0] > kZero) || (py - g.mn[1] < kZero) || (py - g.mx[1] > kZero) ||
        (pz - g.mn[2] < kZero) || (pz - g.mx[2] > kZero))
        return L_OUTSIDE;
    return L_INSIDE;
}

// Shells::Find_shell along axis a
__host__ __device__ inline int find_shell(const WinGeom& g, double x_in, int a) {
    const double x = (x_in > g.mid[a]) ? 2 * g.mid[a] - x_in : x_in;
    if (x < g.layer[a] || fabs(x - g.layer[a]) < kZero) return 0;
    if (x > g.core[a]) return g.n_shells - 1;
    return (int)((x - g.layer[a] + kZero) / g.half[a]) + 1;
}

__host__ __device__ inline int imin(int a, int b) { return a < b ? a : b; }

// Shells::Find_minimum_shell == 0 for point i
__host__ __device__ inline bool in_shell0(const WinGeom& g, const Pts& p, int i) {
    int s = imin(find_shell(g, p.x[i], 0), find_shell(g, p.y[i], 1));
    s = imin(s, find_shell(g, p.z[i], 2));
    return s == 0;
}

__host__ __device__ inline double max_std(double a, double b) { return (a < b) ? b : a; }  // std::max(a, b)

// Substitute_boundary_point: moves point `out` along (in - out) onto the window face it crossed
__host__ __device__ inline void substitute(const WinGeom& g, const Pts& p, int in, int out) {
    const double Tx = p.x[in] - p.x[out], Ty = p.y[in] - p.y[out], Tz = p.z[in] - p.z[out];
    const double ox = p.x[out], oy = p.y[out], oz = p.z[out];
    double lx = -1.0, ly = -1.0, lz = -1.0;
    if ((ox - g.mn[0]) < kZero) lx = (g.mn[0] - ox) / Tx;
    else if ((g.mx[0] - ox) < kZero) lx = (g.mx[0] - ox) / Tx;
    if ((oy - g.mn[1]) < kZero) ly = (g.mn[1] - oy) / Ty;
    else if ((g.mx[1] - oy) < kZero) ly = (g.mx[1] - oy) / Ty;
    if ((oz - g.mn[2]) < kZero) lz = (g.mn[2] - oz) / Tz;
    else if ((g.mx[2] - oz) < kZero) lz = (g.mx[2] - oz) / Tz;
    const double l = max_std(lx, max_std(ly, lz));
    const double tx = Tx * l, ty = Ty * l, tz = Tz * l;
    p.x[out] = ox + tx;
    p.y[out] = oy + ty;
    p.z[out] = oz + tz;
    p.flag[out] = p.flag[in];
}

// Where_is_with_boundary: face of a boundary point (0 z_max, 1 z_min, 2 x_max, 3 y_max, 4 x_min, 5 y_min), -1 otherwise
__host__ __device__ inline int boundary_of(const WinGeom& g, const Pts& p, int i) {
    const double c[3] = {p.x[i], p.y[i], p.z[i]};
    for (int a = 0; a < 3; a++)
        if (!(g.mn[a] - c[a] <= kZero && c[a] - g.mx[a] <= kZero)) return -1;
    if (fabs(c[0] - g.mn[0]) < kZero) return 4;
    if (fabs(c[0] - g.mx[0]) < kZero) return 2;
    if (fabs(c[1] - g.mn[1]) < kZero) return 5;
    if (fabs(c[1] - g.mx[1]) < kZero) return 3;
    if (fabs(c[2] - g.mn[2]) < kZero) return 1;
    if (fabs(c[2] - g.mx[2]) < kZero) return 0;
    return -1;
}

// Point_3D::distance_to
__host__ __device__ inline double dist(const Pts& p, int a, int b) {
    const double dx = p.x[a] - p.x[b], dy = p.y[a] - p.y[b], dz = p.z[a] - p.z[b];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// Boundary event: point, face, segment number (0: the CNT being trimmed, m >= 1: its m-th new piece)
__host__ __device__ inline int64_t pack_event(int P, int face, int seg) { return ((int64_t)P << 16) | ((int64_t)face << 8) | seg; }
__host__ __device__ inline int ev_point(int64_t e) { return (int)(e >> 16); }
__host__ __device__ inline int ev_face(int64_t e) { return (int)((e >> 8) & 0xff); }
__host__ __device__ inline int ev_seg(int64_t e) { return (int)(e & 0xff); }

// Result of one CNT's trim: the kept index range and the boundary events.
struct TrimOut {
    int segments = 0;
    int first = 0, last = 0;  // kept index range of the trimmed CNT (segments > 0)
    int nev = 0;
};

// Trim_boundary_cnts for one CNT whose points are the run base .. base + n - 1.
// Pieces (segment m >= 1) get flag -m on their points and a slot (start, end,
// in shell 0); `allow_pieces` false (the pieces' own pass) makes a piece an error.
__host__ __device__ inline int trim_run(const WinGeom& g, const Pts& p, int base, int n, bool allow_pieces, TrimOut& o, int32_t* slots,
                                        int64_t* ev) {
    int start = 0, end = 0, last_inside = 0;
    int point_location = L_INSIDE;
    const int first_loc = where_is(g, p, base);
    // Add_cnt_segment_to_structure
    auto add_segment = [&](int s0, int e0, int end_loc) -> int {
        int new_start = s0, new_end = e0;
        int p_out_start = base + new_start;
        const int sl = where_is(g, p, p_out_start);
        if (sl != L_INSIDE) {
            if (sl == L_OUTSIDE) substitute(g, p, base + new_start + 1, p_out_start);
            if (dist(p, p_out_start, p_out_start + 1) - g.step_cutoff < kZero) {
                p.copy(p_out_start + 1, p_out_start);
                new_start++;
                p_out_start++;
            }
            const int b = boundary_of(g, p, p_out_start);
            if (b < 0) return WIN_NOT_AT_BOUNDARY;
            if (o.nev >= kMaxEv) return WIN_CAPACITY;
            ev[o.nev++] = pack_event(p_out_start, b, o.segments);
        }
        int p_out_end = base + new_end;
        if (end_loc != L_INSIDE) {
            if (end_loc == L_OUTSIDE) substitute(g, p, base + new_end - 1, p_out_end);
            if (dist(p, p_out_end - 1, p_out_end) - g.step_cutoff < kZero) {
                p.copy(p_out_end - 1, p_out_end);
                new_end--;
                p_out_end--;
            }
            const int b = boundary_of(g, p, p_out_end);
            if (b < 0) return WIN_NOT_AT_BOUNDARY;
            if (o.nev >= kMaxEv) return WIN_CAPACITY;
            ev[o.nev++] = pack_event(p_out_end, b, o.segments);
        }
        if (o.segments == 0) {
            o.first = new_start;
            o.last = new_end;
        } else {
            if (!allow_pieces) return WIN_INTERNAL;
            if (o.segments >= kMaxSeg) return WIN_CAPACITY;
            int sh0 = 0;
            for (int j = new_start; j <= new_end; j++) {
                p.flag[base + j] = -o.segments;
                sh0 |= in_shell0(g, p, base + j) ? 1 : 0;
            }
            int32_t* sl3 = slots + 3 * (o.segments - 1);
            sl3[0] = base + new_start;
            sl3[1] = base + new_end;
            sl3[2] = sh0;
        }
        o.segments++;
        return WIN_OK;
    };
    for (int j = 1; j < n; j++) {
        point_location = where_is(g, p, base + j);
        if (point_location != L_OUTSIDE) {
            last_inside = j;
        } else {
            end = j;
            const int n_points = (start == 0 && first_loc != L_OUTSIDE) ? end - start : end - start - 1;
            if (n_points >= g.min_points) {
                const int e = add_segment(start, end, point_location);
                if (e) return e;
            }
            start = j;
        }
    }
    if (last_inside == n - 1 && (last_inside - start + 1) >= g.min_points) {
        end = n - 1;
        const int e = add_segment(start, end, point_location);
        if (e) return e;
    }
    return WIN_OK;
}

// Window 0 and the shell geometry: Geom_sample::update_observation_window_geometry(0, ...)
// (Input_Reader.h:110-135) and Shells::Generate_shells (Shells.cpp:21-40).  False for a
// multi-window run (win_max != win_min), which is not supported.
inline bool window_geom(const cicy_window_params& w, WinGeom& g, cicy_cuboid& win) {
    win.len_x = w.win_max[0];
    win.len_y = w.win_max[1];
    win.len_z = w.win_max[2];
    win.min_x = w.sample.min_x + (w.sample.len_x - win.len_x) / 2.0;
    win.min_y = w.sample.min_y + (w.sample.len_y - win.len_y) / 2.0;
    win.min_z = w.sample.min_z + (w.sample.len_z - win.len_z) / 2.0;
    win.max_x = win.min_x + win.len_x;
    win.max_y = win.min_y + win.len_y;
    win.max_z = win.min_z + win.len_z;
    g.mn[0] = win.min_x; g.mn[1] = win.min_y; g.mn[2] = win.min_z;
    g.mx[0] = win.max_x; g.mx[1] = win.max_y; g.mx[2] = win.max_z;
    const double smin[3] = {w.sample.min_x, w.sample.min_y, w.sample.min_z};
    const double slen[3] = {w.sample.len_x, w.sample.len_y, w.sample.len_z};
    for (int a = 0; a < 3; a++) {
        g.mid[a] = smin[a] + slen[a] / 2.0;
        g.layer[a] = smin[a] + (slen[a] - w.win_max[a]) / 2.0;
        g.core[a] = smin[a] + (slen[a] - w.win_min[a]) / 2.0;
        g.half[a] = w.win_delt[a] / 2.0;
    }
    g.n_shells = 2;
    g.step_cutoff = w.step_length * 0.5;
    g.min_points = w.min_points;
    return (int)((w.win_max[0] - w.win_min[0] + kZero) / w.win_delt[0]) == 0;
}

// ---- per-item bodies of the passes (i: CNT, u: unit = CNT then piece, t: list entry) ----

// CNT i is the i-th run (expect = exclusive scan of the run lengths) and its points carry flag i.
__host__ __device__ inline bool layout_ok(int i, const int32_t* cstart, const int32_t* clen, const int32_t* expect, const int32_t* flag) {
    const int n = clen[i];
    if (n == 0) return true;
    bool ok = cstart[i] == expect[i];
    for (int k = 0; k < n && ok; k++) ok = flag[cstart[i] + k] == i;
    return ok;
}

// First pass: the trim of an original CNT of shell 0 (Trim_boundary_cnts over shells_cnt[0]).
__host__ __device__ inline int trim_cnt(int i, const WinGeom& g, const Pts& p, const int32_t* cstart, const int32_t* clen, int32_t* npieces,
                                        int32_t* first, int32_t* slots, int64_t* ev, int32_t* nev) {
    const int base = cstart[i], n = clen[i];
    npieces[i] = 0;
    nev[i] = 0;
    first[2 * i] = n ? base : 0;
    first[2 * i + 1] = n;
    bool sh0 = false;
    for (int k = 0; k < n && !sh0; k++) sh0 = in_shell0(g, p, base + k);
    if (!sh0) return WIN_OK;
    TrimOut o;
    const int e = trim_run(g, p, base, n, true, o, slots + (size_t)i * kSlot, ev + (size_t)i * kMaxEv);
    if (e) return e;
    nev[i] = o.nev;
    npieces[i] = o.segments > 0 ? o.segments - 1 : 0;
    first[2 * i] = o.segments > 0 ? base + o.first : 0;
    first[2 * i + 1] = o.segments > 0 ? o.last - o.first + 1 : 0;
    return WIN_OK;
}

// Second pass: the pieces of CNT i in creation order (upstream's loop reaches them after
// every original CNT of shell 0), their runs, parent and radius; pbase = exclusive scan of
// the pieces per CNT.
__host__ __device__ inline int trim_pieces(int i, int nc, const WinGeom& g, const Pts& p, const int32_t* npieces, const int32_t* pbase,
                                           const int32_t* slots, const double* radii, int32_t* prun, int32_t* pparent, int64_t* pev,
                                           int32_t* pnev, double* rad_out) {
    // every piece's fields are written, also after a failed trim: the passes after this one
    // read them before the host sees the error
    const int np = npieces[i];
    int err = WIN_OK;
    for (int k = 0; k < np; k++) {
        const int q = pbase[i] + k;
        const int32_t* sl3 = slots + (size_t)i * kSlot + 3 * k;
        const int s = sl3[0], e = sl3[1];
        pparent[q] = i;
        rad_out[nc + q] = radii[i];
        pnev[q] = 0;
        prun[2 * q] = s;
        prun[2 * q + 1] = e - s + 1;
        if (!sl3[2] || err) continue;
        TrimOut o;
        int64_t evq[kMaxEv];
        int r = trim_run(g, p, s, e - s + 1, false, o, nullptr, evq);
        if (!r && o.nev > 2) r = WIN_INTERNAL;
        if (r) {
            err = r;
            continue;
        }
        for (int t = 0; t < o.nev; t++) pev[2 * q + t] = evq[t];
        pnev[q] = o.nev;
        prun[2 * q] = o.segments > 0 ? s + o.first : 0;
        prun[2 * q + 1] = o.segments > 0 ? o.last - o.first + 1 : 0;
    }
    return err;
}

// Placeholder flags -m of CNT i's pieces -> the pieces' indices.
__host__ __device__ inline void fix_flags(int i, int nc, const int32_t* cstart, const int32_t* clen, const int32_t* npieces, const int32_t* pbase,
                                          int32_t* flag) {
    if (!npieces[i]) return;
    const int b = cstart[i], n = clen[i];
    for (int k = 0; k < n; k++) {
        const int f = flag[b + k];
        if (f < 0) flag[b + k] = nc + pbase[i] + (-f) - 1;
    }
}

// Boundary events of unit u per face, face-major (cnt[b * U + u]).
__host__ __device__ inline void face_counts(int u, int nc, int npc, const int64_t* ev, const int32_t* nev, const int64_t* pev,
                                            const int32_t* pnev, int32_t* cnt) {
    const int U = nc + npc;
    int c6[6] = {0, 0, 0, 0, 0, 0};
    const int64_t* e = u < nc ? ev + (size_t)u * kMaxEv : pev + 2 * (size_t)(u - nc);
    const int ne = u < nc ? nev[u] : pnev[u - nc];
    for (int t = 0; t < ne; t++) c6[ev_face(e[t])]++;
    for (int b = 0; b < 6; b++) cnt[(size_t)b * U + u] = c6[b];
}

// Unit u's events into the face lists at their scanned offsets: the point, and the CNT
// the event names (the unit itself, or in the first pass its m-th new piece).
__host__ __device__ inline void scatter_events(int u, int nc, int npc, const int64_t* ev, const int32_t* nev, const int64_t* pev,
                                               const int32_t* pnev, const int32_t* pbase, const int32_t* off, int32_t* raw_p, int32_t* raw_c) {
    const int U = nc + npc;
    int r6[6] = {0, 0, 0, 0, 0, 0};
    const int64_t* e = u < nc ? ev + (size_t)u * kMaxEv : pev + 2 * (size_t)(u - nc);
    const int ne = u < nc ? nev[u] : pnev[u - nc];
    for (int t = 0; t < ne; t++) {
        const int b = ev_face(e[t]), m = ev_seg(e[t]);
        const int pos = off[(size_t)b * U + u] + r6[b]++;
        raw_p[pos] = ev_point(e[t]);
        raw_c[pos] = (u < nc && m > 0) ? nc + pbase[u] + m - 1 : u;
    }
}

// Add_cnt_point_to_boundary_vectors adds a CNT to a face's list unless it is that list's
// last entry: keep entry t unless it starts no face list and repeats the entry before it.
__host__ __device__ inline int keep_entry(int t, const int* face_start, const int32_t* raw_c) {
    bool start = false;
    for (int b = 0; b < 6; b++) start |= (t == face_start[b]);
    return (start || raw_c[t] != raw_c[t - 1]) ? 1 : 0;
}

// Final run of unit u (original CNT, then piece) and its Fill_cnts_inside flag.
__host__ __device__ inline int final_run(int u, int nc, const int32_t* first, const int32_t* prun, int32_t* cs, int32_t* cl,
                                         int32_t* inside_flag) {
    const int32_t* r = u < nc ? first + 2 * (size_t)u : prun + 2 * (size_t)(u - nc);
    cs[u] = r[0];
    cl[u] = r[1];
    inside_flag[u] = r[1] > 2 ? 1 : 0;
    return r[1] == 1 ? WIN_ONE_POINT : WIN_OK;
}

}  // namespace win
}  // namespace cicy
