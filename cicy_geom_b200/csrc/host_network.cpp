// Host-side network sources upstream of the device hot path:
//  * a seeded, counter-based synthetic CNT network generator, and
//  * the single-window extraction (Shells + Cutoff_Wins, CNT_wires branch)
//    that turns a read/generated network into the window-trimmed network the
//    hot path consumes.
// Both are plain CPU code by design: they run once per network, are O(N_p),
// and sit before the drop-in boundary (App_Network_3D.cpp:85-136).
#include "cicy_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace cicy {

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): counter-based RNG.
struct Philox {
    uint32_t k0, k1;
    static inline void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
        uint64_t p = (uint64_t)a * (uint64_t)b;
        hi = (uint32_t)(p >> 32);
        lo = (uint32_t)p;
    }
    void block(const uint32_t ctr_in[4], uint32_t out[4]) const {
        uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
        uint32_t key0 = k0, key1 = k1;
        for (int r = 0; r < 10; r++) {
            uint32_t hi0, lo0, hi1, lo1;
            mulhilo(0xD2511F53u, c0, hi0, lo0);
            mulhilo(0xCD9E8D57u, c2, hi1, lo1);
            uint32_t n0 = hi1 ^ c1 ^ key0;
            uint32_t n1 = lo1;
            uint32_t n2 = hi0 ^ c3 ^ key1;
            uint32_t n3 = lo0;
            c0 = n0; c1 = n1; c2 = n2; c3 = n3;
            key0 += 0x9E3779B9u;
            key1 += 0xBB67AE85u;
        }
        out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
    }
    // Two uniform doubles in [0,1) from draw `d` of stream `s`.
    void uniform2(uint32_t s, uint32_t d, double& u0, double& u1) const {
        uint32_t c[4] = {s, d, 0x43494359u, 0x42323030u}, o[4];
        block(c, o);
        uint64_t a = ((uint64_t)o[0] << 32) | o[1];
        uint64_t b = ((uint64_t)o[2] << 32) | o[3];
        u0 = (double)(a >> 11) * (1.0 / 9007199254740992.0);
        u1 = (double)(b >> 11) * (1.0 / 9007199254740992.0);
    }
};

static int cnt_point_count(const Philox& rng, int32_t i, const cicy_gen_params& g) {
    double u0, u1;
    rng.uniform2((uint32_t)i, 0, u0, u1);
    double L = g.len_min + u0 * (g.len_max - g.len_min);
    return 1 + (int)std::floor(L / g.step);
}

static void cnt_fill(const Philox& rng, int32_t i, const cicy_gen_params& g, int np, double* x, double* y, double* z) {
    const double two_pi = 6.283185307179586476925286766559;
    double u0, u1, u2, u3;
    rng.uniform2((uint32_t)i, 1, u0, u1);
    rng.uniform2((uint32_t)i, 2, u2, u3);
    double px = g.sample.min_x + u0 * g.sample.len_x;
    double py = g.sample.min_y + u1 * g.sample.len_y;
    double pz = g.sample.min_z + u2 * g.sample.len_z;
    double v0, v1;
    rng.uniform2((uint32_t)i, 3, v0, v1);
    // isotropic initial direction: cos(theta) ~ U[-1,1], phi ~ U[0,2pi)
    double ct = 2.0 * v0 - 1.0;
    double st = std::sqrt(std::max(0.0, 1.0 - ct * ct));
    double ph = two_pi * v1;
    double dx = st * std::cos(ph), dy = st * std::sin(ph), dz = ct;
    (void)u3;
    x[0] = px; y[0] = py; z[0] = pz;
    for (int k = 1; k < np; k++) {
        double w0, w1;
        rng.uniform2((uint32_t)i, 3u + (uint32_t)k, w0, w1);
        double th = w0 * g.max_turn_rad;
        double az = two_pi * w1;
        // orthonormal frame (e1, e2) perpendicular to d
        double ax, ay, az_;
        if (std::fabs(dx) < 0.9) { ax = 1; ay = 0; az_ = 0; } else { ax = 0; ay = 1; az_ = 0; }
        double e1x = ay * dz - az_ * dy, e1y = az_ * dx - ax * dz, e1z = ax * dy - ay * dx;
        double n1 = std::sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
        e1x /= n1; e1y /= n1; e1z /= n1;
        double e2x = dy * e1z - dz * e1y, e2y = dz * e1x - dx * e1z, e2z = dx * e1y - dy * e1x;
        double c = std::cos(th), s = std::sin(th), ca = std::cos(az), sa = std::sin(az);
        double nx = c * dx + s * (ca * e1x + sa * e2x);
        double ny = c * dy + s * (ca * e1y + sa * e2y);
        double nz = c * dz + s * (ca * e1z + sa * e2z);
        double nn = std::sqrt(nx * nx + ny * ny + nz * nz);
        dx = nx / nn; dy = ny / nn; dz = nz / nn;
        px = px + g.step * dx;
        py = py + g.step * dy;
        pz = pz + g.step * dz;
        x[k] = px; y[k] = py; z[k] = pz;
    }
}

HostNetwork* generate_cnt_network(const cicy_gen_params& g) {
    HostNetwork* h = new HostNetwork;
    Philox rng{(uint32_t)(g.seed & 0xffffffffu), (uint32_t)(g.seed >> 32)};
    int32_t nc = g.n_cnts;
    h->radii.assign(nc, g.radius);
    h->structure_ptr.assign(nc + 1, 0);
    for (int32_t i = 0; i < nc; i++) h->structure_ptr[i + 1] = h->structure_ptr[i] + cnt_point_count(rng, i, g);
    int64_t np = h->structure_ptr[nc];
    h->x.resize(np); h->y.resize(np); h->z.resize(np); h->flag.resize(np);
    h->structure_idx.resize(np);
    unsigned nt = g.n_threads > 0 ? (unsigned)g.n_threads : std::max(1u, std::thread::hardware_concurrency());
    nt = std::min<unsigned>(nt, 64);
    auto work = [&](unsigned t) {
        for (int32_t i = (int32_t)t; i < nc; i += (int32_t)nt) {
            int64_t s = h->structure_ptr[i], e = h->structure_ptr[i + 1];
            cnt_fill(rng, i, g, (int)(e - s), &h->x[s], &h->y[s], &h->z[s]);
            for (int64_t p = s; p < e; p++) { h->flag[p] = i; h->structure_idx[p] = p; }
        }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; t++) th.emplace_back(work, t);
    work(0);
    for (auto& t : th) t.join();
    h->boundary_cnt_ptr.assign(7, 0);
    h->boundary_pts_ptr.assign(7, 0);
    h->window = g.sample;
    return h;
}

// ---------------------------------------------------------------------------
// Window extraction (window 0, CNT_wires).  Restates, with the same operation
// order, Shells::Generate_shells / Find_shell (Shells.cpp:21-149) and
// Cutoff_Wins::Trim_boundary_cnts (Cutoff_Wins.cpp:82-276),
// Add_cnt_segment_to_structure (:298-467), Substitute_boundary_point (:468-548),
// Where_is (:554-566), Where_is_with_boundary (:683-743),
// Add_cnt_point_to_boundary_vectors (:745-769), Fill_cnts_inside (:803-831).
namespace {

const double kZero = 1.0e-10;  // MathMatrix.h:18

struct P3 {
    double x, y, z;
    int flag;
};

enum Loc { INSIDE = 0, OUTSIDE = 1, BOUNDARY = 2 };

struct WinCtx {
    cicy_cuboid win;
    double mid[3], layer[3], core[3], half[3];
    int n_shells;
    std::vector<P3> pts;
    std::vector<std::vector<int64_t> > structure;
    std::vector<double> radii;
    std::vector<std::vector<int> > shells;
    std::vector<std::vector<int> > bcnt;
    std::vector<std::vector<int64_t> > bpts;
    double step_cutoff;
    int min_points;

    bool at_boundary(const P3& p) const {  // Point_3D::is_at_cuboid_boundary (Geometry_3D.cpp:238-246)
        return std::fabs(p.x - win.min_x) < kZero || std::fabs(p.x - win.max_x) < kZero ||
               std::fabs(p.y - win.min_y) < kZero || std::fabs(p.y - win.max_y) < kZero ||
               std::fabs(p.z - win.min_z) < kZero || std::fabs(p.z - win.max_z) < kZero;
    }
    bool outside(const P3& p) const {  // Point_3D::is_outside_cuboid (Geometry_3D.cpp:227-235)
        return (p.x - win.min_x < kZero) || (p.x - win.max_x > kZero) || (p.y - win.min_y < kZero) ||
               (p.y - win.max_y > kZero) || (p.z - win.min_z < kZero) || (p.z - win.max_z > kZero);
    }
    Loc where_is(const P3& p) const {
        if (at_boundary(p)) return BOUNDARY;
        if (outside(p)) return OUTSIDE;
        return INSIDE;
    }
    int find_shell(double x_in, int a) const {  // Shells::Find_shell
        double x = (x_in > mid[a]) ? 2 * mid[a] - x_in : x_in;
        if (x < layer[a] || std::fabs(x - layer[a]) < kZero) return 0;
        if (x > core[a]) return n_shells - 1;
        return (int)((x - layer[a] + kZero) / half[a]) + 1;
    }
    void add_to_shells(const P3& p) {  // Shells::Add_to_cnt_shells + Find_minimum_shell (CNT_wires)
        int s = std::min(find_shell(p.x, 0), find_shell(p.y, 1));
        s = std::min(s, find_shell(p.z, 2));
        if (shells[s].empty() || shells[s].back() != p.flag) shells[s].push_back(p.flag);
    }
    void substitute(const P3& pin, P3& pout) const {
        double Tx = pin.x - pout.x, Ty = pin.y - pout.y, Tz = pin.z - pout.z;
        auto lam = [](double plane, double xo, double xt) { return (plane - xo) / xt; };
        double lx = -1.0, ly = -1.0, lz = -1.0;
        if ((pout.x - win.min_x) < kZero) lx = lam(win.min_x, pout.x, Tx);
        else if ((win.max_x - pout.x) < kZero) lx = lam(win.max_x, pout.x, Tx);
        if ((pout.y - win.min_y) < kZero) ly = lam(win.min_y, pout.y, Ty);
        else if ((win.max_y - pout.y) < kZero) ly = lam(win.max_y, pout.y, Ty);
        if ((pout.z - win.min_z) < kZero) lz = lam(win.min_z, pout.z, Tz);
        else if ((win.max_z - pout.z) < kZero) lz = lam(win.max_z, pout.z, Tz);
        double l = std::max(lx, std::max(ly, lz));
        double tx = Tx * l, ty = Ty * l, tz = Tz * l;
        pout.x = pout.x + tx;
        pout.y = pout.y + ty;
        pout.z = pout.z + tz;
        pout.flag = pin.flag;
    }
    int boundary_of(const P3& p) const {  // Where_is_with_boundary; -1 when not at a boundary
        auto bounded = [](double c, double lo, double hi) { return (lo - c <= kZero && c - hi <= kZero); };
        if (!bounded(p.x, win.min_x, win.max_x)) return -1;
        if (!bounded(p.y, win.min_y, win.max_y)) return -1;
        if (!bounded(p.z, win.min_z, win.max_z)) return -1;
        if (std::fabs(p.x - win.min_x) < kZero) return 4;
        if (std::fabs(p.x - win.max_x) < kZero) return 2;
        if (std::fabs(p.y - win.min_y) < kZero) return 5;
        if (std::fabs(p.y - win.max_y) < kZero) return 3;
        if (std::fabs(p.z - win.min_z) < kZero) return 1;
        if (std::fabs(p.z - win.max_z) < kZero) return 0;
        return -1;
    }
    bool add_boundary(int64_t P, int cnt_num) {
        int b = boundary_of(pts[P]);
        if (b < 0) return false;
        if (bcnt[b].empty() || bcnt[b].back() != cnt_num) bcnt[b].push_back(cnt_num);
        bpts[b].push_back(P);
        return true;
    }
    bool add_segment(int start, int end, int CNT, Loc end_loc, int& segments, int& first_idx, int& last_idx) {
        int new_start = start, new_end = end;
        int64_t p_out_start = structure[CNT][new_start];
        int64_t p_ins_start = structure[CNT][new_start + 1];
        Loc sl = where_is(pts[p_out_start]);
        if (sl != INSIDE) {
            if (sl == OUTSIDE) substitute(pts[p_ins_start], pts[p_out_start]);
            int cnt_num = segments ? (int)structure.size() : CNT;
            if (dist(pts[p_out_start], pts[p_out_start + 1]) - step_cutoff < kZero) {
                pts[p_out_start + 1] = pts[p_out_start];
                new_start++;
                p_out_start++;
            }
            if (!add_boundary(p_out_start, cnt_num)) return false;
        }
        int64_t p_out_end = structure[CNT][new_end];
        int64_t p_ins_end = structure[CNT][new_end - 1];
        if (end_loc != INSIDE) {
            if (end_loc == OUTSIDE) substitute(pts[p_ins_end], pts[p_out_end]);
            int cnt_num = segments ? (int)structure.size() : CNT;
            if (dist(pts[p_out_end - 1], pts[p_out_end]) - step_cutoff < kZero) {
                pts[p_out_end - 1] = pts[p_out_end];
                new_end--;
                p_out_end--;
            }
            if (!add_boundary(p_out_end, cnt_num)) return false;
        }
        if (segments == 0) {
            first_idx = new_start;
            last_idx = new_end;
        } else {
            int new_cnt = (int)structure.size();
            std::vector<int64_t> tmp;
            for (int j = new_start; j <= new_end; j++) {
                int64_t P = structure[CNT][j];
                pts[P].flag = new_cnt;
                tmp.push_back(P);
                add_to_shells(pts[P]);
            }
            radii.push_back(radii[CNT]);
            structure.push_back(tmp);
        }
        segments++;
        return true;
    }
    static double dist(const P3& a, const P3& b) {  // Point_3D::distance_to (Geometry_3D.cpp:64-70)
        double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
        return std::sqrt(dx * dx + dy * dy + dz * dz);
    }
    bool trim() {
        bcnt.assign(6, std::vector<int>());
        bpts.assign(6, std::vector<int64_t>());
        Loc point_location = INSIDE;
        for (size_t i = 0; i < shells[0].size(); i++) {
            int CNT = shells[0][i];
            int start = 0, end = 0, first_idx = 0, last_idx = 0, segments = 0, last_inside = 0;
            int cnt_points = (int)structure[CNT].size();
            if (!cnt_points) continue;
            int64_t P1 = structure[CNT][0];
            Loc first_loc = where_is(pts[P1]);
            for (int j = 1; j < cnt_points; j++) {
                P1 = structure[CNT][j];
                point_location = where_is(pts[P1]);
                if (point_location != OUTSIDE) {
                    last_inside = j;
                } else {
                    end = j;
                    int n_points = (start == 0 && first_loc != OUTSIDE) ? end - start : end - start - 1;
                    if (n_points >= min_points)
                        if (!add_segment(start, end, CNT, point_location, segments, first_idx, last_idx)) return false;
                    start = j;
                }
            }
            if (last_inside == cnt_points - 1 && (last_inside - start + 1) >= min_points) {
                end = cnt_points - 1;
                if (!add_segment(start, end, CNT, point_location, segments, first_idx, last_idx)) return false;
            }
            if (segments > 0) {
                if (first_idx != 0) {
                    for (int k = first_idx; k <= last_idx; k++) structure[CNT][k - first_idx] = structure[CNT][k];
                    last_idx = last_idx - first_idx;
                }
                for (int k = last_idx + 1; k < cnt_points; k++) structure[CNT].pop_back();
            } else {
                structure[CNT].clear();
            }
        }
        return true;
    }
};

}  // namespace

// Window 0 and the shell geometry: Geom_sample::update_observation_window_geometry(0, ...)
// (Input_Reader.h:110-135) and the midpoints / boundary layer / core / half steps of
// Shells::Generate_shells (Shells.cpp:21-40); single-window runs only.
bool window_geometry(const cicy_window_params& w, WinCtx& c, std::string& err) {
    c.win.len_x = w.win_max[0];
    c.win.len_y = w.win_max[1];
    c.win.len_z = w.win_max[2];
    c.win.min_x = w.sample.min_x + (w.sample.len_x - c.win.len_x) / 2.0;
    c.win.min_y = w.sample.min_y + (w.sample.len_y - c.win.len_y) / 2.0;
    c.win.min_z = w.sample.min_z + (w.sample.len_z - c.win.len_z) / 2.0;
    c.win.max_x = c.win.min_x + c.win.len_x;
    c.win.max_y = c.win.min_y + c.win.len_y;
    c.win.max_z = c.win.min_z + c.win.len_z;
    const double* smin[3] = {&w.sample.min_x, &w.sample.min_y, &w.sample.min_z};
    const double* slen[3] = {&w.sample.len_x, &w.sample.len_y, &w.sample.len_z};
    for (int a = 0; a < 3; a++) {
        c.mid[a] = *smin[a] + *slen[a] / 2.0;
        c.layer[a] = *smin[a] + (*slen[a] - w.win_max[a]) / 2.0;
        c.core[a] = *smin[a] + (*slen[a] - w.win_min[a]) / 2.0;
        c.half[a] = w.win_delt[a] / 2.0;
    }
    int num = (int)((w.win_max[0] - w.win_min[0] + kZero) / w.win_delt[0]);
    if (num != 0) {
        err = "extract_window: only single-window runs (win_max == win_min, cut_num = 0) are supported";
        return false;
    }
    c.n_shells = num + 2;
    return true;
}

cicy_status extract_window(const HostNetwork& in, const cicy_window_params& w, HostNetwork** out, std::string& err) {
    WinCtx c;
    if (!window_geometry(w, c, err)) return CICY_E_INPUT;
    c.step_cutoff = w.step_length * 0.5;
    c.min_points = w.min_points;
    int64_t np = (int64_t)in.x.size();
    c.pts.resize(np);
    for (int64_t i = 0; i < np; i++) c.pts[i] = P3{in.x[i], in.y[i], in.z[i], in.flag[i]};
    int32_t nc = (int32_t)in.radii.size();
    c.structure.resize(nc);
    for (int32_t i = 0; i < nc; i++)
        c.structure[i].assign(in.structure_idx.begin() + in.structure_ptr[i], in.structure_idx.begin() + in.structure_ptr[i + 1]);
    c.radii = in.radii;
    c.shells.assign(c.n_shells, std::vector<int>());
    for (int64_t i = 0; i < np; i++) c.add_to_shells(c.pts[i]);
    if (!c.trim()) {
        err = "Error: point should be at boundary but it is not (Cutoff_Wins::Add_cnt_point_to_boundary_vectors)";
        return CICY_E_INPUT;
    }
    HostNetwork* h = new HostNetwork;
    h->x.resize(np); h->y.resize(np); h->z.resize(np); h->flag.resize(np);
    for (int64_t i = 0; i < np; i++) { h->x[i] = c.pts[i].x; h->y[i] = c.pts[i].y; h->z[i] = c.pts[i].z; h->flag[i] = c.pts[i].flag; }
    h->radii = c.radii;
    h->structure_ptr.assign(1, 0);
    for (auto& s : c.structure) {
        for (auto p : s) h->structure_idx.push_back(p);
        h->structure_ptr.push_back((int64_t)h->structure_idx.size());
    }
    // Cutoff_Wins::Fill_cnts_inside
    for (size_t i = 0; i < c.structure.size(); i++) {
        if (c.structure[i].size() > 2) h->cnts_inside.push_back((int32_t)i);
        else if (c.structure[i].size() == 1) {
            delete h;
            err = "Error in Extract_observation_window. CNT " + std::to_string(i) + " has only one point.";
            return CICY_E_INPUT;
        }
    }
    h->boundary_cnt_ptr.assign(1, 0);
    h->boundary_pts_ptr.assign(1, 0);
    for (int b = 0; b < 6; b++) {
        for (auto v : c.bcnt[b]) h->boundary_cnt_idx.push_back(v);
        h->boundary_cnt_ptr.push_back((int64_t)h->boundary_cnt_idx.size());
        for (auto v : c.bpts[b]) h->boundary_pts_idx.push_back(v);
        h->boundary_pts_ptr.push_back((int64_t)h->boundary_pts_idx.size());
    }
    h->window = c.win;
    *out = h;
    return CICY_OK;
}

// ---------------------------------------------------------------------------
// Read_Network::Read_sample_geometry + Read_cnt_data_from_dat / _from_csv
// (Read_Network.cpp:154-467), CNT branch: the files of `dir` into the layout
// the generator emits (points in CNT order, flag = CNT index, structure = the
// consecutive point ids, window = the sample).  Both formats are read whole and
// parsed in memory (strtod, the conversion the upstream stream extraction
// performs, so the doubles are the same); the upstream error cases (a file
// ending before every CNT or point was read, n_cnts mismatch on the CSV's first
// line, missing files) fail with CICY_E_INPUT and the upstream message.
namespace {

bool slurp(const std::string& path, std::string& out) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(n > 0 ? (size_t)n : 0);
    const size_t got = n > 0 ? std::fread(&out[0], 1, (size_t)n, f) : 0;
    std::fclose(f);
    return got == out.size();
}

// `count` numbers separated by one character each (the stream's ignore()), then the rest of the line.
bool parse_line(const char*& p, const char* end, int count, double* v) {
    if (p >= end) return false;
    for (int i = 0; i < count; i++) {
        char* q = nullptr;
        v[i] = std::strtod(p, &q);
        if (q == p) return false;
        p = q;
        if (i + 1 < count && p < end) p++;  // the separator
    }
    while (p < end && *p != '\n') p++;
    if (p < end) p++;
    return true;
}

}  // namespace

cicy_status read_network_files(const std::string& dir, int file_type, HostNetwork** out, std::string& err) {
    HostNetwork* h = new HostNetwork;
    auto fail = [&](const std::string& m) {
        delete h;
        err = m;
        return CICY_E_INPUT;
    };
    std::string text;
    if (!slurp(dir + "/sample_geom.csv", text))
        return fail("Error in Read_sample_geometry: Failed to open file with sample geometry data sample_geom.csv.");
    {
        const char* p = text.data();
        const char* e = p + text.size();
        double a[3], l[3];
        if (!parse_line(p, e, 3, a) || !parse_line(p, e, 3, l)) return fail("Error in Read_sample_geometry: sample_geom.csv needs two lines");
        cicy_cuboid& w = h->window;
        w.min_x = a[0]; w.min_y = a[1]; w.min_z = a[2];
        w.len_x = l[0]; w.len_y = l[1]; w.len_z = l[2];
        w.max_x = w.min_x + w.len_x;
        w.max_y = w.min_y + w.len_y;
        w.max_z = w.min_z + w.len_z;
    }
    std::vector<int32_t> np;
    if (file_type == 0) {
        std::string st;
        if (!slurp(dir + "/cnt_struct.dat", st)) return fail("Failed to open CNT structure file cnt_struct.dat.");
        if (st.size() < 4) return fail("Error in Read_cnt_data_from_dat. The end-of-file of cnt_struct.dat has been reached before reading all CNT data.");
        int32_t n = 0;
        std::memcpy(&n, st.data(), 4);
        if (n < 0 || st.size() < 4 + 12 * (size_t)n)
            return fail("Error in Read_cnt_data_from_dat. The end-of-file of cnt_struct.dat has been reached before reading all CNT data.");
        np.resize(n);
        h->radii.resize(n);
        for (int32_t i = 0; i < n; i++) {
            std::memcpy(&np[i], st.data() + 4 + 12 * (size_t)i, 4);
            std::memcpy(&h->radii[i], st.data() + 8 + 12 * (size_t)i, 8);
        }
    } else if (file_type == 1) {
        std::string st;
        if (!slurp(dir + "/cnt_struct.csv", st))
            return fail("Error in Read_cnt_data_from_csv: Failed to open CNT structure file cnt_struct.csv.");
        const char* p = st.data();
        const char* e = p + st.size();
        double v[2];
        if (!parse_line(p, e, 2, v)) return fail("Error in Read_cnt_data_from_csv. cnt_struct.csv is empty.");
        if ((int64_t)v[0] != (int64_t)v[1])
            return fail("Error in Read_cnt_data_from_csv. The first line of file cnt_struct.csv indicates different number of CNTs: " +
                        std::to_string((int64_t)v[0]) + " and " + std::to_string((int64_t)v[1]));
        const int32_t n = (int32_t)v[0];
        np.resize(std::max(n, 0));
        h->radii.resize(np.size());
        for (int32_t i = 0; i < n; i++) {
            if (!parse_line(p, e, 2, v))
                return fail("Error in Read_cnt_data_from_csv. The end-of-file of cnt_struct.csv has been reached before reading all CNT data.");
            np[i] = (int32_t)v[0];
            h->radii[i] = v[1];
        }
    } else {
        return fail("Error in Generate_nanoparticle_network_from_file. Invalid file type to read CNT network from. Valid options are 'csv' or 'dat' only.");
    }
    const int32_t n = (int32_t)np.size();
    h->structure_ptr.assign(n + 1, 0);
    for (int32_t i = 0; i < n; i++) {
        if (np[i] < 0) return fail("Error in Read_cnt_data: CNT " + std::to_string(i) + " has a negative number of points");
        h->structure_ptr[i + 1] = h->structure_ptr[i] + np[i];
    }
    const int64_t N = h->structure_ptr[n];
    h->x.resize(N); h->y.resize(N); h->z.resize(N); h->flag.resize(N); h->structure_idx.resize(N);
    for (int32_t i = 0; i < n; i++)
        for (int64_t q = h->structure_ptr[i]; q < h->structure_ptr[i + 1]; q++) {
            h->flag[q] = i;
            h->structure_idx[q] = q;
        }
    if (file_type == 0) {
        std::string co;
        if (!slurp(dir + "/cnt_coordinates.dat", co)) return fail("Failed to open point cordinates file cnt_coordinates.dat.");
        if (co.size() < 24 * (size_t)N)
            return fail("Error in Read_cnt_data_from_dat. The end-of-file of cnt_coordinates.dat has been reached before reading all CNT data.");
        for (int64_t q = 0; q < N; q++) {
            std::memcpy(&h->x[q], co.data() + 24 * q, 8);
            std::memcpy(&h->y[q], co.data() + 24 * q + 8, 8);
            std::memcpy(&h->z[q], co.data() + 24 * q + 16, 8);
        }
    } else {
        std::string co;
        if (!slurp(dir + "/cnt_coordinates.csv", co)) return fail("Failed to open point cordinates file cnt_coordinates.csv.");
        // lines are independent: split the text at line ends, count the lines of each
        // piece, and parse the pieces on host threads into their point ranges
        const char* text0 = co.data();
        const size_t len = co.size();
        const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<size_t> cut(nt + 1, len);
        cut[0] = 0;
        for (unsigned t = 1; t < nt; t++) {
            size_t c = std::max(cut[t - 1], len * t / nt);
            while (c > 0 && c < len && text0[c - 1] != '\n') c++;
            cut[t] = c;
        }
        std::vector<int64_t> lines(nt + 1, 0);
        for (unsigned t = 0; t < nt; t++) {
            int64_t k = 0;
            for (size_t c = cut[t]; c < cut[t + 1]; c++) k += text0[c] == '\n';
            if (cut[t + 1] > cut[t] && text0[cut[t + 1] - 1] != '\n') k++;  // a last line without its newline
            lines[t + 1] = lines[t] + k;
        }
        if (lines[nt] < N)
            return fail("Error in Read_cnt_data_from_csv. The end-of-file of cnt_coordinates.csv has been reached before reading all CNT data.");
        std::vector<int> bad(nt, 0);
        auto work = [&](unsigned t) {
            const char* p = text0 + cut[t];
            const char* e = text0 + cut[t + 1];
            for (int64_t q = lines[t]; q < std::min(lines[t + 1], N); q++) {
                double v[3];
                if (!parse_line(p, e, 3, v)) {
                    bad[t] = 1;
                    return;
                }
                h->x[q] = v[0];
                h->y[q] = v[1];
                h->z[q] = v[2];
            }
        };
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; t++) th.emplace_back(work, t);
        work(0);
        for (auto& t : th) t.join();
        for (unsigned t = 0; t < nt; t++)
            if (bad[t]) return fail("Error in Read_cnt_data_from_csv: a line of cnt_coordinates.csv is not x,y,z");
    }
    h->boundary_cnt_ptr.assign(7, 0);
    h->boundary_pts_ptr.assign(7, 0);
    *out = h;
    return CICY_OK;
}

// ---------------------------------------------------------------------------
// GNPs as Read_Network::Read_gnp_data_from_dat builds them (Read_Network.cpp:576-679):
// rotation matrix Generate_Network::Get_transformation_matrix (Generate_Network.cpp:3466-3480),
// vertices Obtain_gnp_vertex_coordinates (:3848-3867) through Point_3D::rotation
// (Geometry_3D.cpp:147-165), face planes Update_gnp_plane_equations (:3869-3889) through
// Plane_3D(P1, P2, P3) (Geometry_3D.cpp: normal (P2-P1) x (P3-P1), made unit, offset
// -N.P1).  Same operation order as upstream, so the doubles are identical (host code,
// no FMA contraction).
namespace {

struct V3 {
    double x, y, z;
};

V3 rotate(const double* M, const V3& p, const V3& d) {
    return V3{M[0] * p.x + M[1] * p.y + M[2] * p.z + d.x, M[3] * p.x + M[4] * p.y + M[5] * p.z + d.y,
              M[6] * p.x + M[7] * p.y + M[8] * p.z + d.z};
}

void plane(const V3& P1, const V3& P2, const V3& P3, double* out) {
    const V3 u{P2.x - P1.x, P2.y - P1.y, P2.z - P1.z}, w{P3.x - P1.x, P3.y - P1.y, P3.z - P1.z};
    double a = u.y * w.z - w.y * u.z;
    double b = -(u.x * w.z - w.x * u.z);
    double c = u.x * w.y - w.x * u.y;
    const double len = std::sqrt(a * a + b * b + c * c);
    a = a / len;
    b = b / len;
    c = c / len;
    out[0] = a;
    out[1] = b;
    out[2] = c;
    out[3] = (a * P1.x + b * P1.y + c * P1.z) * (-1);
}

}  // namespace

cicy_status read_gnp_file(const std::string& dir, GnpSet** out, std::string& err) {
    std::string st;
    if (!slurp(dir + "/gnp_data.dat", st)) {
        err = "Failed to open file with GNP geometric data gnp_data.dat.";
        return CICY_E_INPUT;
    }
    int32_t n = 0;
    if (st.size() >= 4) std::memcpy(&n, st.data(), 4);
    if (st.size() < 4 || n < 0 || st.size() < 4 + 56 * (size_t)n) {
        err = "Error in Read_gnp_data_from_dat. The end-of-file of gnp_data.dat has been reached before reading all GNP data.";
        return CICY_E_INPUT;
    }
    GnpSet* g = new GnpSet;
    g->n = n;
    g->l.resize(n); g->t.resize(n); g->center.resize(3 * (size_t)n); g->rotation.resize(9 * (size_t)n);
    g->vertices.resize(24 * (size_t)n); g->planes.resize(24 * (size_t)n);
    for (int32_t i = 0; i < n; i++) {
        double r[7];
        std::memcpy(r, st.data() + 4 + 56 * (size_t)i, 56);
        const double l = r[0], t = r[1], theta = r[2], phi = r[3];
        g->l[i] = l;
        g->t[i] = t;
        double* M = &g->rotation[9 * (size_t)i];
        M[0] = std::cos(phi) * std::cos(theta);
        M[1] = -std::sin(phi);
        M[2] = std::cos(phi) * std::sin(theta);
        M[3] = std::sin(phi) * std::cos(theta);
        M[4] = std::cos(phi);
        M[5] = std::sin(phi) * std::sin(theta);
        M[6] = -std::sin(theta);
        M[7] = 0.0;
        M[8] = std::cos(theta);
        const V3 c{r[4], r[5], r[6]};
        g->center[3 * (size_t)i] = c.x;
        g->center[3 * (size_t)i + 1] = c.y;
        g->center[3 * (size_t)i + 2] = c.z;
        const V3 loc[8] = {{l / 2, l / 2, t / 2},   {-l / 2, l / 2, t / 2},   {-l / 2, -l / 2, t / 2},   {l / 2, -l / 2, t / 2},
                           {l / 2, l / 2, -t / 2},  {-l / 2, l / 2, -t / 2},  {-l / 2, -l / 2, -t / 2},  {l / 2, -l / 2, -t / 2}};
        V3 v[8];
        for (int k = 0; k < 8; k++) {
            v[k] = rotate(M, loc[k], c);
            g->vertices[24 * (size_t)i + 3 * k] = v[k].x;
            g->vertices[24 * (size_t)i + 3 * k + 1] = v[k].y;
            g->vertices[24 * (size_t)i + 3 * k + 2] = v[k].z;
        }
        static const int F[6][3] = {{0, 1, 3}, {4, 7, 5}, {0, 3, 4}, {0, 4, 1}, {1, 5, 2}, {2, 6, 3}};
        for (int f = 0; f < 6; f++) plane(v[F[f][0]], v[F[f][1]], v[F[f][2]], &g->planes[24 * (size_t)i + 4 * f]);
    }
    *out = g;
    return CICY_OK;
}

HostNetwork* host_network_from_view(const cicy_network& n) {
    HostNetwork* h = new HostNetwork;
    h->x.assign(n.x, n.x + n.n_points);
    h->y.assign(n.y, n.y + n.n_points);
    h->z.assign(n.z, n.z + n.n_points);
    h->flag.assign(n.flag, n.flag + n.n_points);
    h->radii.assign(n.radii, n.radii + n.n_cnts);
    h->structure_ptr.assign(n.structure_ptr, n.structure_ptr + n.n_cnts + 1);
    h->structure_idx.assign(n.structure_idx, n.structure_idx + n.structure_ptr[n.n_cnts]);
    if (n.n_inside > 0) h->cnts_inside.assign(n.cnts_inside, n.cnts_inside + n.n_inside);
    if (n.boundary_cnt_ptr) {
        h->boundary_cnt_ptr.assign(n.boundary_cnt_ptr, n.boundary_cnt_ptr + 7);
        h->boundary_cnt_idx.assign(n.boundary_cnt_idx, n.boundary_cnt_idx + n.boundary_cnt_ptr[6]);
    } else {
        h->boundary_cnt_ptr.assign(7, 0);
    }
    if (n.boundary_pts_ptr) {
        h->boundary_pts_ptr.assign(n.boundary_pts_ptr, n.boundary_pts_ptr + 7);
        h->boundary_pts_idx.assign(n.boundary_pts_idx, n.boundary_pts_idx + n.boundary_pts_ptr[6]);
    } else {
        h->boundary_pts_ptr.assign(7, 0);
    }
    h->window = n.window;
    return h;
}

void host_network_view(const HostNetwork& h, cicy_network& v) {
    std::memset(&v, 0, sizeof(v));
    v.n_points = (int64_t)h.x.size();
    v.x = h.x.data(); v.y = h.y.data(); v.z = h.z.data(); v.flag = h.flag.data();
    v.n_cnts = (int32_t)h.radii.size();
    v.structure_ptr = h.structure_ptr.data();
    v.structure_idx = h.structure_idx.data();
    v.radii = h.radii.data();
    v.n_inside = (int32_t)h.cnts_inside.size();
    v.cnts_inside = h.cnts_inside.data();
    v.boundary_cnt_ptr = h.boundary_cnt_ptr.data();
    v.boundary_cnt_idx = h.boundary_cnt_idx.data();
    v.boundary_pts_ptr = h.boundary_pts_ptr.data();
    v.boundary_pts_idx = h.boundary_pts_idx.data();
    v.window = h.window;
}

// ---------------------------------------------------------------------------
// GNP part of the window extraction (window 0): Shells::Add_to_gnp_shells
// (Shells.cpp:150-178) and Cutoff_Wins::Fill_gnps_inside (Cutoff_Wins.cpp:833-869)
// with Find_gnp_boundary_points (:871-987),
// Find_intersections_of_gnp_edges_with_window_boundaries (:1016-1091),
// Find_two_intersections_of_gnp_edges_with_window (:1093-1135),
// Find_intersections_of_window_edges_with_gnp_faces (:1137-1191),
// Does_edge_intersect_gnp (:1193-1271), Find_window_vertex_inside_gnp
// (:1273-1318) and GNP::Is_point_inside_gnp (Geometry_3D.h:352-379), in
// upstream's operation order.  GNPs whose shells reach window 0 get one
// boundary point per window face they cross: the average of the points
// accumulated on that face (GNP vertices on it, GNP edges cut by it, window
// edges through the GNP, a window corner inside it), and a volume inside the
// window: l^2 t times the share of a 20 x 20 grid on its mid-plane that lies in
// the window (Generate_Network::Approximate_gnp_volume_inside_sample,
// Generate_Network.cpp:4750-4810).
namespace {

struct V3w {
    double x, y, z;
};
V3w operator+(const V3w& a, const V3w& b) { return V3w{a.x + b.x, a.y + b.y, a.z + b.z}; }
V3w operator-(const V3w& a, const V3w& b) { return V3w{a.x - b.x, a.y - b.y, a.z - b.z}; }
V3w operator*(const V3w& a, double s) { return V3w{a.x * s, a.y * s, a.z * s}; }
double dotw(const V3w& a, const V3w& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

struct GnpWin {
    const WinCtx& c;
    // Where_is_with_boundary: 0 inside, 1 outside, 2 boundary (face in `b`)
    int where(const V3w& p, int& b) const {
        auto bounded = [](double v, double lo, double hi) { return (lo - v <= kZero && v - hi <= kZero); };
        if (!bounded(p.x, c.win.min_x, c.win.max_x) || !bounded(p.y, c.win.min_y, c.win.max_y) || !bounded(p.z, c.win.min_z, c.win.max_z))
            return 1;
        if (std::fabs(p.x - c.win.min_x) < kZero) b = 4;
        else if (std::fabs(p.x - c.win.max_x) < kZero) b = 2;
        else if (std::fabs(p.y - c.win.min_y) < kZero) b = 5;
        else if (std::fabs(p.y - c.win.max_y) < kZero) b = 3;
        else if (std::fabs(p.z - c.win.min_z) < kZero) b = 1;
        else if (std::fabs(p.z - c.win.max_z) < kZero) b = 0;
        else return 0;
        return 2;
    }
    void window_vertices(V3w W[8]) const {
        const V3w m{c.win.min_x, c.win.min_y, c.win.min_z};
        W[0] = V3w{c.win.max_x, c.win.max_y, c.win.max_z};
        W[1] = m + V3w{0, c.win.len_y, c.win.len_z};
        W[2] = m + V3w{0, 0, c.win.len_z};
        W[3] = m + V3w{c.win.len_x, 0, c.win.len_z};
        W[4] = m + V3w{c.win.len_x, c.win.len_y, 0};
        W[5] = m + V3w{0, c.win.len_y, 0};
        W[6] = m;
        W[7] = m + V3w{c.win.len_x, 0, 0};
    }
};

}  // namespace

cicy_status gnp_window(const GnpSet& g, const cicy_window_params& w, GnpWindow& out, std::string& err) {
    WinCtx c;
    if (!window_geometry(w, c, err)) return CICY_E_INPUT;
    out = GnpWindow{};
    out.boundary_gnp.assign(6, std::vector<int32_t>());
    out.boundary_pts.assign(6, std::vector<int32_t>());
    out.structure.assign(g.n, std::vector<int32_t>());
    out.volume.assign(g.n, std::nan(""));
    const GnpWin gw{c};
    V3w W[8];
    gw.window_vertices(W);
    static const int ged[12][2] = {{0, 1}, {0, 3}, {0, 4}, {2, 1}, {2, 3}, {2, 6}, {5, 1}, {5, 4}, {5, 6}, {7, 3}, {7, 4}, {7, 6}};
    static const int wb[12][2] = {{0, 3}, {0, 2}, {2, 3}, {0, 4}, {0, 5}, {4, 5}, {3, 4}, {1, 3}, {1, 4}, {2, 5}, {1, 2}, {1, 5}};
    static const int corner_b[8][3] = {{0, 2, 3}, {0, 3, 4}, {0, 4, 5}, {0, 2, 5}, {1, 2, 3}, {1, 3, 4}, {1, 4, 5}, {1, 2, 5}};
    static const int adj[6][4] = {{2, 3, 4, 5}, {2, 3, 4, 5}, {0, 1, 3, 5}, {0, 1, 2, 4}, {0, 1, 3, 5}, {0, 1, 2, 4}};
    static const int vref[6] = {0, 4, 0, 0, 1, 2};
    for (int i = 0; i < g.n; i++) {
        const double* Vd = &g.vertices[24 * (size_t)i];
        const double* Fd = &g.planes[24 * (size_t)i];
        V3w V[8], N[6];
        for (int k = 0; k < 8; k++) V[k] = V3w{Vd[3 * k], Vd[3 * k + 1], Vd[3 * k + 2]};
        for (int f = 0; f < 6; f++) N[f] = V3w{Fd[4 * f], Fd[4 * f + 1], Fd[4 * f + 2]};
        // Add_to_gnp_shells: the least and greatest shell of the vertices
        int smin = 0, smax = 0;
        for (int k = 0; k < 8; k++) {
            int s = std::min(c.find_shell(V[k].x, 0), c.find_shell(V[k].y, 1));
            s = std::min(s, c.find_shell(V[k].z, 2));
            if (k == 0 || s < smin) smin = s;
            if (k == 0 || s > smax) smax = s;
        }
        if (0 < smin) {
            out.inside.push_back(i);
            continue;
        }
        if (!(0 >= smin && 0 <= smax)) continue;
        // Find_gnp_boundary_points
        std::vector<V3w> acc[6];
        int loc[8], n_inside = 0;
        for (int k = 0; k < 8; k++) {
            int b = -1;
            loc[k] = gw.where(V[k], b);
            if (loc[k] == 0) n_inside++;
            else if (loc[k] == 2) acc[b].push_back(V[k]);
        }
        if (n_inside == 0) continue;
        out.inside.push_back(i);
        if (n_inside == 8) continue;
        for (int e = 0; e < 12; e++) {  // GNP edges cut by the window's faces
            const int v1 = ged[e][0], v2 = ged[e][1];
            if ((loc[v1] == 0 && loc[v2] == 1) || (loc[v2] == 0 && loc[v1] == 1)) {
                const V3w& pin = loc[v1] == 0 ? V[v1] : V[v2];
                const V3w& po = loc[v1] == 0 ? V[v2] : V[v1];
                P3 a{pin.x, pin.y, pin.z, i}, b{po.x, po.y, po.z, i};
                c.substitute(a, b);
                int bb = -1;
                if (gw.where(V3w{b.x, b.y, b.z}, bb) != 2) {
                    err = "Error in Find_intersections_of_gnp_edges_with_window_boundaries: point is not at a boundary (GNP " + std::to_string(i) + ")";
                    return CICY_E_INPUT;
                }
                acc[bb].push_back(V3w{b.x, b.y, b.z});
            } else if (loc[v1] == 1 && loc[v2] == 1) {
                const V3w A = V[v1], B = V[v2];
                auto cut = [&](double a1, double a2, double wc) {
                    if ((a1 - wc < kZero && a2 - wc > kZero) || (a2 - wc < kZero && a1 - wc > kZero)) {
                        const double lambda = (wc - a1) / (a2 - a1);
                        const V3w P = A + (B - A) * lambda;
                        int pb = -1;
                        if (gw.where(P, pb) == 2) acc[pb].push_back(P);
                    }
                };
                cut(A.x, B.x, c.win.min_x);
                cut(A.x, B.x, c.win.max_x);
                cut(A.y, B.y, c.win.min_y);
                cut(A.y, B.y, c.win.max_y);
                cut(A.z, B.z, c.win.min_z);
                cut(A.z, B.z, c.win.max_z);
            }
        }
        for (int e = 0; e < 12; e++) {  // window edges through the GNP's faces
            const V3w& P1 = W[ged[e][0]];
            const V3w V1V2 = W[ged[e][1]] - P1;
            for (int f = 0; f < 6; f++) {
                const int l1 = dotw(N[f], P1 - V[vref[f]]) > kZero;
                const int l2 = dotw(N[f], W[ged[e][1]] - V[vref[f]]) > kZero;
                if (l1 == l2) continue;
                const double lambda = (-dotw(N[f], P1) - Fd[4 * f + 3]) / dotw(N[f], V1V2);
                const V3w P = P1 + V1V2 * lambda;
                bool ignore = false;
                for (int j = 0; j < 4 && !ignore; j++) ignore = dotw(N[adj[f][j]], P - V[vref[adj[f][j]]]) > kZero;
                if (!ignore) {
                    acc[wb[e][0]].push_back(P);
                    acc[wb[e][1]].push_back(P);
                    break;
                }
            }
        }
        for (int k = 0; k < 8; k++) {  // a window corner inside the GNP
            const V3w& P = W[k];
            const V3w V4P = P - V[4];
            if (dotw(N[0], P - V[0]) < kZero && dotw(N[1], V4P) < kZero && dotw(N[2], V4P) < kZero && dotw(N[4], P - V[1]) < kZero &&
                dotw(N[3], V4P) < kZero && dotw(N[5], P - V[2]) < kZero) {
                for (int j = 0; j < 3; j++) acc[corner_b[k][j]].push_back(P);
                break;
            }
        }
        {  // Approximate_gnp_volume_inside_sample on the window
            const V3w c3{(V[3].x + V[7].x) / 2.0, (V[3].y + V[7].y) / 2.0, (V[3].z + V[7].z) / 2.0};
            const V3w c0{(V[0].x + V[4].x) / 2.0, (V[0].y + V[4].y) / 2.0, (V[0].z + V[4].z) / 2.0};
            const V3w c2{(V[2].x + V[6].x) / 2.0, (V[2].y + V[6].y) / 2.0, (V[2].z + V[6].z) / 2.0};
            const V3w c1{(V[1].x + V[5].x) / 2.0, (V[1].y + V[5].y) / 2.0, (V[1].z + V[5].z) / 2.0};
            const V3w dir_right = c0 - c3, dir_right_up = c1 - c2;
            const int np = 20;
            int in = 0;
            for (int a = 0; a < np; a++) {
                const double lr = (double)a / (np - 1);
                const V3w start = c3 + dir_right * lr, end = c2 + dir_right_up * lr, dir_up = end - start;
                for (int b = 0; b < np; b++) {
                    const double lu = (double)b / (np - 1);
                    const V3w q = start + dir_up * lu;
                    if (!(q.x < c.win.min_x || q.x > c.win.max_x || q.y < c.win.min_y || q.y > c.win.max_y || q.z < c.win.min_z || q.z > c.win.max_z))
                        in++;
                }
            }
            double vol = g.l[i] * g.l[i] * g.t[i];
            if (in != 0) vol = vol * ((double)in / (np * np));
            out.volume[i] = vol;
        }
        for (int b = 0; b < 6; b++) {
            if (acc[b].empty()) continue;
            V3w avg{0.0, 0.0, 0.0};
            for (const V3w& q : acc[b]) avg = avg + q;
            const double n = (double)acc[b].size();
            const int32_t P = (int32_t)(out.points.size() / 3);
            out.boundary_gnp[b].push_back(i);
            out.boundary_pts[b].push_back(P);
            out.structure[i].push_back(P);
            out.points.insert(out.points.end(), {avg.x / n, avg.y / n, avg.z / n});
            out.point_gnp.push_back(i);
            out.point_boundary.push_back(b);
        }
    }
    return CICY_OK;
}

}  // namespace cicy
