// Host build of the device window trim (test helper): window_trim.cuh, the
// source the extraction kernels of stage_window.cu compile, driven by g++
// without FMA contraction through the same sequence of passes the device runs
// (layout check, first trim pass, scan of the pieces, the pieces' pass, flag
// fix-up, face counts, scan, scatter, run-length compaction, runs,
// Fill_cnts_inside), each pass as a loop over its items.  The CPU tests compare
// its output with the host restatement (cicy_extract_window).
//
//   host_window <in.bin> <out.bin>
//
// in.bin:  int32 n_points, n_cnts, min_points; double sample[9], win_max[3],
//          win_min[3], win_delt[3], step_length; double x, y, z [n_points];
//          int32 flag [n_points]; int32 cstart, clen [n_cnts]; double radii [n_cnts]
// out.bin: int32 status, n_points, n_cnts, n_inside, n_bcnt, n_bpts;
//          double x, y, z; int32 flag; int32 cstart, clen; double radii;
//          int32 inside, bcnt_ptr[7], bcnt_idx, bpts_ptr[7], bpts_idx; double window[9]
#include <cstdio>
#include <vector>

#define __host__
#define __device__
#include "window_trim.cuh"

using namespace cicy::win;

template <class T>
static bool get(FILE* f, std::vector<T>& v, size_t n) {
    v.resize(n);
    return n == 0 || fread(v.data(), sizeof(T), n, f) == n;
}
template <class T>
static void put(FILE* f, const std::vector<T>& v, size_t n) {
    if (n) fwrite(v.data(), sizeof(T), n, f);
}
static std::vector<int32_t> exclusive_scan(const std::vector<int32_t>& in, size_t n) {
    std::vector<int32_t> out(n + 1, 0);
    for (size_t i = 0; i < n; i++) out[i + 1] = out[i] + in[i];
    return out;
}

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    FILE* f = fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t hdr[3];
    if (fread(hdr, 4, 3, f) != 3) return 3;
    const int np = hdr[0], nc = hdr[1];
    cicy_window_params w{};
    double wd[22];
    if (fread(wd, 8, 22, f) != 22) return 3;
    w.sample = cicy_cuboid{wd[0], wd[1], wd[2], wd[3], wd[4], wd[5], wd[6], wd[7], wd[8]};
    for (int a = 0; a < 3; a++) {
        w.win_max[a] = wd[9 + a];
        w.win_min[a] = wd[12 + a];
        w.win_delt[a] = wd[15 + a];
    }
    w.step_length = wd[18];
    w.min_points = hdr[2];
    std::vector<double> x, y, z, radii;
    std::vector<int32_t> flag, cstart, clen;
    if (!get(f, x, np) || !get(f, y, np) || !get(f, z, np) || !get(f, flag, np) || !get(f, cstart, nc) || !get(f, clen, nc) ||
        !get(f, radii, nc))
        return 3;
    fclose(f);

    int status = WIN_OK;
    auto note = [&](int e) {
        if (e && !status) status = e;
    };
    WinGeom g{};
    cicy_cuboid win{};
    if (!window_geom(w, g, win)) note(WIN_INTERNAL);
    Pts p{x.data(), y.data(), z.data(), flag.data()};
    const size_t NC = nc > 0 ? nc : 1;
    std::vector<int32_t> npieces(NC, 0), first(2 * NC, 0), slots(NC * kSlot, 0), nev(NC, 0);
    std::vector<int64_t> ev(NC * kMaxEv, 0);
    std::vector<int32_t> expect = exclusive_scan(clen, nc);
    for (int i = 0; i < nc; i++)
        if (!layout_ok(i, cstart.data(), clen.data(), expect.data(), flag.data())) note(WIN_LAYOUT);
    for (int i = 0; i < nc && !status; i++)
        note(trim_cnt(i, g, p, cstart.data(), clen.data(), npieces.data(), first.data(), slots.data(), ev.data(), nev.data()));
    std::vector<int32_t> pbase = exclusive_scan(npieces, nc);
    const int npc = pbase[nc], U = nc + npc;
    const size_t NP = npc > 0 ? npc : 1;
    std::vector<int32_t> prun(2 * NP, 0), pparent(NP, 0), pnev(NP, 0);
    std::vector<int64_t> pev(2 * NP, 0);
    std::vector<double> rad(U > 0 ? U : 1, 0.0);
    for (int i = 0; i < nc; i++) rad[i] = radii[i];
    for (int i = 0; i < nc && !status; i++)
        note(trim_pieces(i, nc, g, p, npieces.data(), pbase.data(), slots.data(), radii.data(), prun.data(), pparent.data(), pev.data(),
                         pnev.data(), rad.data()));
    for (int i = 0; i < nc && !status; i++) fix_flags(i, nc, cstart.data(), clen.data(), npieces.data(), pbase.data(), flag.data());
    std::vector<int32_t> cnt(6 * (size_t)U + 1, 0);
    for (int u = 0; u < U; u++) face_counts(u, nc, npc, ev.data(), nev.data(), pev.data(), pnev.data(), cnt.data());
    std::vector<int32_t> off = exclusive_scan(cnt, 6 * (size_t)U);
    int fs[7];
    for (int b = 0; b <= 6; b++) fs[b] = off[(size_t)b * U];
    const int T = fs[6];
    std::vector<int32_t> raw_p(T > 0 ? T : 1), raw_c(T > 0 ? T : 1), keep(T > 0 ? T : 1);
    for (int u = 0; u < U && !status; u++)
        scatter_events(u, nc, npc, ev.data(), nev.data(), pev.data(), pnev.data(), pbase.data(), off.data(), raw_p.data(), raw_c.data());
    for (int t = 0; t < T; t++) keep[t] = keep_entry(t, fs, raw_c.data());
    std::vector<int32_t> pos = exclusive_scan(keep, T);
    std::vector<int32_t> bcnt(pos[T] > 0 ? pos[T] : 1);
    for (int t = 0; t < T; t++)
        if (keep[t]) bcnt[pos[t]] = raw_c[t];
    std::vector<int32_t> bcnt_ptr(7), bpts_ptr(7);
    for (int b = 0; b <= 6; b++) {
        bcnt_ptr[b] = pos[fs[b]];
        bpts_ptr[b] = fs[b];
    }
    std::vector<int32_t> cs(U > 0 ? U : 1), cl(U > 0 ? U : 1), inflag(U > 0 ? U : 1);
    for (int u = 0; u < U && !status; u++) note(final_run(u, nc, first.data(), prun.data(), cs.data(), cl.data(), inflag.data()));
    std::vector<int32_t> ipos = exclusive_scan(inflag, U);
    const int n_inside = ipos[U];
    std::vector<int32_t> inside(n_inside > 0 ? n_inside : 1);
    for (int u = 0; u < U; u++)
        if (inflag[u]) inside[ipos[u]] = u;

    FILE* o = fopen(argv[2], "wb");
    if (!o) return 2;
    const int32_t head[6] = {status, np, U, n_inside, pos[T], T};
    fwrite(head, 4, 6, o);
    put(o, x, np);
    put(o, y, np);
    put(o, z, np);
    put(o, flag, np);
    put(o, cs, U);
    put(o, cl, U);
    put(o, rad, U);
    put(o, inside, n_inside);
    put(o, bcnt_ptr, 7);
    put(o, bcnt, pos[T]);
    put(o, bpts_ptr, 7);
    put(o, raw_p, T);
    const double wo[9] = {win.min_x, win.min_y, win.min_z, win.len_x, win.len_y, win.len_z, win.max_x, win.max_y, win.max_z};
    fwrite(wo, 8, 9, o);
    fclose(o);
    return 0;
}
