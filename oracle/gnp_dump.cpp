/*
 * gnp_dump — TEST ORACLE DRIVER (never shipped, never on the product path).
 *
 * Links the upstream CICY_geom objects compiled in place by oracle/Makefile
 * and dumps, for the GNPs of a directory's gnp_data.dat + sample_geom.csv:
 *   - every GNP as upstream builds it when reading the file
 *     (Read_Network::Read_gnp_data_from_dat, Read_Network.cpp:576-679):
 *     side, thickness, centre, rotation matrix, the 8 vertices and the 6 face
 *     planes (normal and offset);
 *   - for every candidate pair (a < b whose bounding spheres come within the
 *     tunnelling cutoff), the upstream GNP-GNP distance step of
 *     Label_gnps_in_window (Hoshen_Kopelman::Get_distance_between_GNPs,
 *     Hoshen_Kopelman.cpp:770-823: GJK distance, EPA when the GNPs
 *     interpenetrate, then the move of GNP b): distance, direction, the
 *     interpenetration flag and the displacement of b.
 *
 *   gnp_dump <dir> <out.bin> <van_der_Waals_dist> <tunneling_dist> [<gs_min> <overlap_cnt> <overlap_gnp>]
 *
 * With the last three arguments it also dumps upstream's GNP part of the
 * contact grid over the whole sample with every GNP inside
 * (Contact_grid::Fill_sectioned_domain_gnps, Contact_grid.cpp:297-512, on the
 * region grid of Generate_contact_grid + Adjust_regions_if_needed, :18-102):
 * the region counts and sizes and each region's GNP list.
 *
 * If the directory holds gnp_queries.dat (int n, then n x {x, y, z, GNP index}
 * as doubles), it also dumps upstream's closest GNP point to each query point
 * (Generate_Network::Get_gnp_point_closest_to_point, Generate_Network.cpp:5577-
 * 5856, the CNT-GNP distance of Find_adjacent_labels): distance, closest point
 * and flag (-1: the point is inside the GNP).
 *
 * If the directory also holds cnt_struct.dat / cnt_coordinates.dat and the grid
 * arguments are given, it runs upstream's mixed contact pass on the whole
 * sample (Contact_grid::Generate_contact_grid for GNP_CNT_mix, then
 * Hoshen_Kopelman::Find_adjacent_labels, Hoshen_Kopelman.cpp:1989-2142, with a
 * CNT point inside a GNP counted as no contact, ignore_eror_cnt_inside_gnp = 1)
 * and dumps the CNT sectioned domain and the CNT-GNP contacts: point, GNP,
 * contact-point number, junction distance, and the contact points in order,
 * then the labels of the hybrid sample: Make_cnt_clusters, Make_gnp_clusters
 * (GNP-GNP contacts with junction points) and Make_mixed_clusters, in
 * Determine_clusters_and_percolation's order, the GNP point lists and
 * junctions, and the triangulation of every GNP's points
 * (Triangulation::Generate_3d_trangulation).
 *
 * For every candidate pair within the tunnelling cutoff it also runs the
 * junction step of Label_gnps_in_window (Find_junction_points_for_gnps with
 * the moved second GNP, allow_simplex3 = false as App_Network_3D sets it, then
 * the point on the second GNP moved back) and dumps its success flag, both
 * points and whether each lies outside the sample.
 *
 * With "flow <step length>" after the window side (-1: the sample), it also
 * runs upstream's stages for GNP_CNT_mix on window 0 (Shells,
 * Extract_observation_window, Generate_contact_grid,
 * Determine_clusters_and_percolation) and dumps the clusters, families and
 * junction groups (flow_* records); with "electrical" after the step length,
 * also Electrical_analysis::Perform_analysis_on_clusters along x and the
 * resistances it writes, then a stage-by-stage replay of it (e_* records);
 * "electrical_time" skips the replay.  flow_seconds: steady_clock time of the
 * window extraction, contact grid, clusters and percolation, electrical stage.
 * A unit-pass tolerance after the mode (> 0) solves the unit-resistor systems to that
 * tolerance and the real-resistor ones to 1e-10: the electrical stage is then the
 * replay alone (upstream's own calls in Perform_analysis_on_clusters' order, since that
 * method takes one tolerance for both passes), timed as the electrical stage, with the
 * resistances from its parallel resistors (Calculate_resistances_and_resistivities).
 *
 * With a gnp_resistor_cases.dat in the directory it evaluates upstream's
 * Direct_Electrifying::Calculate_resistance_gnp on each case (gnp_resistances).
 *
 * It also runs the GNP part of the window extraction for window 0
 * (Shells::Generate_shells, Cutoff_Wins::Fill_gnps_inside) with the sample as
 * the window, or a centred window of side argv[8] when given, and dumps
 * gnps_inside, boundary_gnp, boundary_gnp_pts and the boundary points.
 *
 * Output records: u32 name length, name, u8 type ('i' int32, 'd' float64),
 * u64 count, payload (the layout oracle/dumpio.py reads).
 */
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <set>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <unistd.h>
#include <vector>

#include "Contact_grid.h"
#include "Generate_Network.h"
#include "Hns.h"
#include "Hoshen_Kopelman.h"
#include "Input_Reader.h"
#include "Cutoff_Wins.h"
#include "Direct_Electrifying.h"
#include "Electrical_analysis.h"
#include "Read_Network.h"
#include "Shells.h"
#include "Triangulation.h"

namespace {

struct Out {
    FILE* f = nullptr;
    void rec(const std::string& name, char type, const void* data, unsigned long long count, size_t elem) {
        unsigned n = (unsigned)name.size();
        fwrite(&n, 4, 1, f);
        fwrite(name.data(), 1, n, f);
        fwrite(&type, 1, 1, f);
        fwrite(&count, 8, 1, f);
        if (count) fwrite(data, elem, count, f);
    }
    void f64(const std::string& name, const std::vector<double>& v) { rec(name, 'd', v.data(), v.size(), 8); }
    void i32(const std::string& name, const std::vector<int>& v) { rec(name, 'i', v.data(), v.size(), 4); }
};

// Lists of indices as CSR records <name>_ptr, <name>_idx.
template <class List>
void dump_csr(Out& o, const std::string& name, const std::vector<List>& lists) {
    std::vector<int> p(1, 0), x;
    for (size_t r = 0; r < lists.size(); r++) {
        for (size_t k = 0; k < lists[r].size(); k++) x.push_back((int)lists[r][k]);
        p.push_back((int)x.size());
    }
    o.i32(name + "_ptr", p);
    o.i32(name + "_idx", x);
}

// A number argument, parsed whole (a stray text such as "np.float64(...)" would read as 0).
double number(const char* s) {
    char* end = nullptr;
    const double v = strtod(s, &end);
    if (end == s || *end != '\0') {
        fprintf(stderr, "gnp_dump: not a number: %s\n", s);
        exit(1);
    }
    return v;
}

// One DEA system of the staged electrical replay and what its assembly left behind.
struct StagedSystem {
    long int nodes = 0, reserved = 0;
    std::vector<long int> row_ptr, col_ind;
    std::vector<double> values, diagonal, b, x0, voltages;
    std::map<long int, long int> lmm_cnts, lmm_gnps;
    std::map<long int, double> cnt_rad;
    std::vector<std::vector<long int> > tri;  // triangulation edges (v1, v2 pairs) of each GNP of the cluster
};

// Direct_Electrifying::Compute_voltage_field (Direct_Electrifying.cpp:11-113) replayed through its
// public members, CNTs and GNPs, keeping the assembled system.
// Tolerance of the unit-resistor (R_flag = 0) solves of the replay; <= 0: the flow's tolerance.
double g_tol_unit = 0.0;

int staged_field(Direct_Electrifying* D, int j, int R_flag, const cuboid& win, const Simu_para& sp, const Electric_para& ep,
                 const Cutoff_dist& cf, Hoshen_Kopelman* HoKo, Cutoff_Wins* CW, const std::vector<Point_3D>& pts,
                 const std::vector<double>& radii, const std::vector<std::vector<long int> >& sg, const std::vector<Point_3D>& pg,
                 std::vector<GNP>& gnps, StagedSystem& S) {
    const int reserved = D->Get_global_nodes(HoKo->family[j]);
    if (reserved == -1) return 0;
    long int global_nodes = reserved;
    if (HoKo->clusters_cnt.size() && HoKo->clusters_cnt[j].size())
        if (!D->LM_matrix_for_cnts(j, HoKo, CW, global_nodes)) return 0;
    if (HoKo->clusters_gnp.size() && HoKo->clusters_gnp[j].size())
        if (!D->LM_matrix_for_gnps(j, HoKo, CW, sg, global_nodes)) return 0;
    std::vector<long int> col_ind, row_ptr;
    std::vector<double> values, diagonal(global_nodes, 0), R(global_nodes - reserved, 0), VEF(reserved, 0.0);
    if (!D->Fill_sparse_stiffness_matrix(R_flag, global_nodes, reserved, cf.van_der_Waals_dist, j, ep, HoKo, pts, radii, sg, pg, gnps,
                                         col_ind, row_ptr, values, diagonal, R, VEF))
        return 0;
    S.b = R;
    std::vector<double> V_guess(global_nodes - reserved, 0.0);
    if (R_flag && reserved == 2) {
        if (!D->Initial_guess_for_CG(j, reserved, HoKo->family[j], win, ep.applied_voltage, HoKo->clusters_cnt, HoKo->elements_cnt, pts,
                                     HoKo->clusters_gnp, pg, R, V_guess))
            return 0;
        if (!D->Update_residual_vector(col_ind, row_ptr, values, diagonal, V_guess, R)) return 0;
    }
    S.x0 = V_guess;
    const double tol = (!R_flag && g_tol_unit > 0) ? g_tol_unit : sp.tolerance;
    if (!D->Solve_DEA_equations_CG_SSS(global_nodes, reserved, tol, col_ind, row_ptr, values, diagonal, R, VEF, V_guess)) return 0;
    S.nodes = global_nodes;
    S.reserved = reserved;
    S.row_ptr = row_ptr;
    S.col_ind = col_ind;
    S.values = values;
    S.diagonal = diagonal;
    S.voltages = D->voltages;
    S.lmm_cnts = D->LMM_cnts;
    S.lmm_gnps = D->LMM_gnps;
    S.cnt_rad = D->points_cnt_rad;
    S.tri.clear();
    if (HoKo->clusters_gnp.size())
        for (int g : HoKo->clusters_gnp[j]) {
            std::vector<long int> e;
            for (const auto& t : gnps[g].triangulation) { e.push_back(t.v1); e.push_back(t.v2); }
            S.tri.push_back(e);
        }
    return 1;
}

void dump_staged(Out& o, const std::string& p, const StagedSystem& S) {
    auto l2i = [](const std::vector<long int>& v) { return std::vector<int>(v.begin(), v.end()); };
    o.i32(p + "nodes", {(int)S.nodes, (int)S.reserved});
    o.i32(p + "row_ptr", l2i(S.row_ptr));
    o.i32(p + "col_ind", l2i(S.col_ind));
    o.f64(p + "values", S.values);
    o.f64(p + "diag", S.diagonal);
    o.f64(p + "b", S.b);
    o.f64(p + "x0", S.x0);
    o.f64(p + "voltages", S.voltages);
    std::vector<int> a, b;
    for (const auto& kv : S.lmm_cnts) { a.push_back((int)kv.first); b.push_back((int)kv.second); }
    o.i32(p + "lmm_cnt_pts", a);
    o.i32(p + "lmm_cnt_nodes", b);
    a.clear(); b.clear();
    for (const auto& kv : S.lmm_gnps) { a.push_back((int)kv.first); b.push_back((int)kv.second); }
    o.i32(p + "lmm_gnp_pts", a);
    o.i32(p + "lmm_gnp_nodes", b);
    a.clear();
    std::vector<double> r;
    for (const auto& kv : S.cnt_rad) { a.push_back((int)kv.first); r.push_back(kv.second); }
    o.i32(p + "cnt_rad_pts", a);
    o.f64(p + "cnt_rad", r);
    dump_csr(o, p + "tri", S.tri);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        fprintf(stderr, "usage: gnp_dump <dir> <out.bin> <van_der_Waals_dist> <tunneling_dist> [<gs_min> <overlap_cnt> <overlap_gnp> [<window side>]]\n");
        return 1;
    }
    const std::string out_path = argv[2];
    const double vdw = number(argv[3]), dt = number(argv[4]);
    if (chdir(argv[1]) != 0) { fprintf(stderr, "cannot chdir to %s\n", argv[1]); return 2; }
    open_deffo_stream((char*)"gnp_log.txt");
    Read_Network RN;
    Geom_sample geom;
    if (!RN.Read_sample_geometry(geom)) return 3;
    std::vector<GNP> gnps;
    if (!RN.Read_gnp_data_from_dat(geom.sample, gnps)) return 4;

    Out o;
    o.f = fopen(out_path.c_str(), "wb");
    if (!o.f) return 5;
    if (FILE* rf = fopen("gnp_resistor_cases.dat", "rb")) {
        // Direct_Electrifying::Calculate_resistance_gnp on the cases of the file:
        // int n, then per case P1 (3), P2 (3), rad1, rad2, rho_surf, rho_t
        int nc = 0;
        if (fread(&nc, 4, 1, rf) != 1) return 18;
        std::vector<double> rr;
        Direct_Electrifying D;
        for (int k = 0; k < nc; k++) {
            double v[10];
            if (fread(v, 8, 10, rf) != 10) return 18;
            Electric_para ep;
            ep.resistivity_GNP_surf = v[8];
            ep.resistivity_GNP_t = v[9];
            double Re = -1.0;
            const int ok = D.Calculate_resistance_gnp(Point_3D(v[0], v[1], v[2]), Point_3D(v[3], v[4], v[5]), v[6], v[7], ep, Re);
            rr.push_back(ok ? Re : -1.0);
        }
        fclose(rf);
        o.f64("gnp_resistances", rr);
    }
    {
        // GNP part of the window extraction for window 0 (Shells::Generate_shells,
        // Cutoff_Wins::Fill_gnps_inside); the window's side is argv[8] when given, else the sample's
        Geom_sample gw = geom;
        const double side = argc >= 9 ? number(argv[8]) : -1.0;
        gw.win_max_x = gw.win_min_x = side > 0 ? side : geom.sample.len_x;
        gw.win_max_y = gw.win_min_y = side > 0 ? side : geom.sample.wid_y;
        gw.win_max_z = gw.win_min_z = side > 0 ? side : geom.sample.hei_z;
        gw.win_delt_x = gw.win_delt_y = gw.win_delt_z = 0.25;
        gw.cut_num = 0;
        std::vector<std::vector<int> > shells_cnt;
        std::vector<Shell> shells_gnp(gnps.size());
        std::vector<Point_3D> no_points;
        Shells SH;
        if (!SH.Generate_shells("GNP_cuboids", gw, no_points, gnps, shells_cnt, shells_gnp)) return 16;
        const cuboid win = gw.update_observation_window_geometry(0, "GNP_cuboids");
        std::vector<GNP> gcopy = gnps;
        for (GNP& gg : gcopy) gg.volume = std::nan("");  // upstream leaves the volume of GNPs it does not process unset
        std::vector<std::vector<long int> > st(gnps.size());
        std::vector<Point_3D> pg;
        Cutoff_Wins CW;
        if (!CW.Fill_gnps_inside(0, win, shells_gnp, gcopy, st, pg)) return 17;
        o.i32("win_inside", CW.gnps_inside);
        dump_csr(o, "win_bgnp", CW.boundary_gnp);
        dump_csr(o, "win_bpts", CW.boundary_gnp_pts);
        dump_csr(o, "win_structure", st);
        std::vector<double> xyz;
        for (const Point_3D& q : pg) xyz.insert(xyz.end(), {q.x, q.y, q.z});
        o.f64("win_points", xyz);
        o.f64("win_box", {win.poi_min.x, win.poi_min.y, win.poi_min.z, win.len_x, win.wid_y, win.hei_z, win.max_x, win.max_y, win.max_z});
        std::vector<double> vol;
        for (const GNP& gg : gcopy) vol.push_back(gg.volume);
        o.f64("win_volume", vol);
    }
    std::vector<double> lt, center, rot, vert, planes;
    for (const GNP& g : gnps) {
        lt.push_back(g.l);
        lt.push_back(g.t);
        center.insert(center.end(), {g.center.x, g.center.y, g.center.z});
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) rot.push_back(g.rotation.element[r][c]);
        for (int v = 0; v < 8; v++) vert.insert(vert.end(), {g.vertices[v].x, g.vertices[v].y, g.vertices[v].z});
        for (int f = 0; f < 6; f++) planes.insert(planes.end(), {g.faces[f].coef[0], g.faces[f].coef[1], g.faces[f].coef[2], g.faces[f].coef[3]});
    }
    o.f64("gnp_lt", lt);
    o.f64("gnp_center", center);
    o.f64("gnp_rotation", rot);
    o.f64("gnp_vertices", vert);
    o.f64("gnp_planes", planes);

    Cutoff_dist cut;
    cut.van_der_Waals_dist = vdw;
    cut.tunneling_dist = dt;
    Hoshen_Kopelman HK;
    std::vector<int> pa, pb, pflag;
    std::vector<double> dist, dir, disp;
    std::vector<int> jn_pair, jn_ok, jn_out;
    std::vector<double> jn_pts;
    const int n = (int)gnps.size();
    for (int a = 0; a < n; a++)
        for (int b = a + 1; b < n; b++) {
            // bounding spheres (half diagonal of the l x l x t cuboid) within the cutoff
            const double ra = 0.5 * std::sqrt(2 * gnps[a].l * gnps[a].l + gnps[a].t * gnps[a].t);
            const double rb = 0.5 * std::sqrt(2 * gnps[b].l * gnps[b].l + gnps[b].t * gnps[b].t);
            const double dc = std::sqrt((gnps[a].center.x - gnps[b].center.x) * (gnps[a].center.x - gnps[b].center.x) +
                                        (gnps[a].center.y - gnps[b].center.y) * (gnps[a].center.y - gnps[b].center.y) +
                                        (gnps[a].center.z - gnps[b].center.z) * (gnps[a].center.z - gnps[b].center.z));
            if (dc > ra + rb + dt) continue;
            GNP gnp_B = gnps[b];
            Point_3D disp_tot(0, 0, 0), N(0, 0, 0);
            bool p_flag = false;
            double d = 0;
            if (!HK.Get_distance_between_GNPs(cut, gnps, a, b, p_flag, disp_tot, N, d, gnp_B)) return 6;
            if (d <= dt) {
                // the junction step of Label_gnps_in_window for a pair within the cutoff
                Point_3D PA, PB;
                std::vector<Point_3D> scratch;
                const int ok = HK.Find_junction_points_for_gnps(false, geom.sample, gnps[a], gnp_B, N, d, scratch, PA, PB);
                if (ok && p_flag) PB = PB - disp_tot;
                jn_pair.push_back((int)pa.size());
                jn_ok.push_back(ok);
                jn_out.push_back(ok ? (PA.is_outside_cuboid(geom.sample) ? 1 : 0) + (PB.is_outside_cuboid(geom.sample) ? 2 : 0) : -1);
                jn_pts.insert(jn_pts.end(), {PA.x, PA.y, PA.z, PB.x, PB.y, PB.z});
            }
            pa.push_back(a);
            pb.push_back(b);
            pflag.push_back(p_flag ? 1 : 0);
            dist.push_back(d);
            dir.insert(dir.end(), {N.x, N.y, N.z});
            disp.insert(disp.end(), {disp_tot.x, disp_tot.y, disp_tot.z});
        }
    if (argc >= 8) {
        const double gs = number(argv[5]), ov_cnt = number(argv[6]), ov_gnp = number(argv[7]);
        geom.gs_minx = geom.gs_miny = geom.gs_minz = gs;
        geom.gs_overlap_cnt = ov_cnt;
        geom.gs_overlap_gnp = ov_gnp;
        const cuboid& w = geom.sample;
        int nreg[3] = {std::max(1, (int)(w.len_x / gs)), std::max(1, (int)(w.wid_y / gs)), std::max(1, (int)(w.hei_z / gs))};
        double lreg[3] = {gs, gs, gs};
        Contact_grid CG;
        if (!CG.Adjust_regions_if_needed(std::max(ov_cnt, ov_gnp), geom, w, nreg, lreg)) return 7;
        const int tot = nreg[0] * nreg[1] * nreg[2];
        std::vector<int> inside(n);
        for (int i = 0; i < n; i++) inside[i] = i;
        CG.sectioned_domain_gnps.assign(tot, std::vector<int>());
        if (!CG.Fill_sectioned_domain_gnps(w, gnps, inside, ov_gnp, nreg, lreg, tot)) return 8;
        std::vector<int> sptr(1, 0), sidx;
        for (const auto& r : CG.sectioned_domain_gnps) {
            sidx.insert(sidx.end(), r.begin(), r.end());
            sptr.push_back((int)sidx.size());
        }
        std::vector<Point_3D> pts;
        std::vector<double> radii;
        std::vector<std::vector<long int> > structure;
        if (FILE* cf = fopen("cnt_struct.dat", "rb")) {
            fclose(cf);
            if (!RN.Read_cnt_data_from_dat(pts, radii, structure)) return 9;
            std::vector<int> cin(structure.size());
            for (size_t i = 0; i < cin.size(); i++) cin[i] = (int)i;
            using clk = std::chrono::steady_clock;
            auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
            std::vector<double> ref_seconds;  // contact grid, CNT clusters, GNP clusters, mixed clusters (the upstream calls only)
            const auto t0 = clk::now();
            Contact_grid CG2;
            if (!CG2.Generate_contact_grid(0, "GNP_CNT_mix", geom, w, cin, pts, structure, inside, gnps)) return 10;
            ref_seconds.push_back(secs(t0, clk::now()));
            Hoshen_Kopelman HK2;
            HK2.ignore_eror_cnt_inside_gnp = 1;
            std::vector<int> labels_cnt(structure.size(), -1), labels_gnp(gnps.size(), -1);
            std::vector<int> labels_mixed(structure.size() + gnps.size(), -1), labels_labels_mixed;
            std::vector<Point_3D> contact_points_gnp;
            std::map<long int, std::map<int, long int> > point_contacts;
            std::map<long int, std::map<int, double> > point_contacts_dist;
            std::vector<std::map<int, std::set<long int> > > gnp_cnt_point_contacts(gnps.size());
            if (!HK2.Find_adjacent_labels(0, labels_cnt, labels_gnp, cut, pts, radii, CG2.sectioned_domain_cnts, gnps, CG2.sectioned_domain_gnps,
                                          contact_points_gnp, point_contacts, point_contacts_dist, gnp_cnt_point_contacts, labels_mixed,
                                          labels_labels_mixed))
                return 11;
            std::vector<int> sdc_ptr(1, 0), sdc_idx, mp, mg, mi;
            std::vector<double> md, mpts;
            for (const auto& r : CG2.sectioned_domain_cnts) {
                for (long int v : r) sdc_idx.push_back((int)v);
                sdc_ptr.push_back((int)sdc_idx.size());
            }
            for (const auto& pc : point_contacts)
                for (const auto& gc : pc.second) {
                    mp.push_back((int)pc.first);
                    mg.push_back(gc.first);
                    mi.push_back((int)gc.second);
                    md.push_back(point_contacts_dist[pc.first][gc.first]);
                }
            for (const auto& c : contact_points_gnp) mpts.insert(mpts.end(), {c.x, c.y, c.z});
            // labels of the hybrid sample: Make_cnt_clusters, Make_gnp_clusters, Make_mixed_clusters
            // (Hoshen_Kopelman.cpp:40-80 order), tol_gnp = 1.5 t_max as Input_Reader.cpp:1161 sets it
            Hoshen_Kopelman HK3;
            HK3.ignore_eror_cnt_inside_gnp = 1;
            Cutoff_dist cut3 = cut;
            cut3.min_points = 5;
            double t_max = 0.0;
            for (const GNP& g : gnps) t_max = std::max(t_max, g.t);
            cut3.tol_gnp = 1.5 * t_max;
            cut3.tol_gnp2 = cut3.tol_gnp * cut3.tol_gnp;
            std::vector<int> lab_cnt(structure.size(), -1), lab_gnp(gnps.size(), -1);
            int n_labels_cnt = 0;
            auto t1 = clk::now();
            if (!HK3.Make_cnt_clusters("GNP_CNT_mix", pts, radii, cut3, CG2.sectioned_domain_cnts, structure, lab_cnt, n_labels_cnt)) return 12;
            ref_seconds.push_back(secs(t1, clk::now()));
            int n_total = n_labels_cnt;
            std::vector<std::vector<long int> > structure_gnp(gnps.size());
            std::vector<Point_3D> points_gnp;
            std::vector<bool> bp_flags;
            t1 = clk::now();
            if (!HK3.Make_gnp_clusters(false, geom.sample, inside, CG2.sectioned_domain_gnps, gnps, cut3, 0, n_labels_cnt, n_total, structure_gnp,
                                       points_gnp, lab_gnp, bp_flags))
                return 13;
            ref_seconds.push_back(secs(t1, clk::now()));
            o.i32("lab_cnt", lab_cnt);
            o.i32("lab_gnp", lab_gnp);
            o.i32("lab_counts", {n_labels_cnt, n_total});
            auto dump_points = [&](const std::string& pre) {
                std::vector<double> xyz;
                std::vector<int> sp(1, 0), si;
                for (const Point_3D& q : points_gnp) xyz.insert(xyz.end(), {q.x, q.y, q.z});
                for (const auto& st : structure_gnp) {
                    for (long int v : st) si.push_back((int)v);
                    sp.push_back((int)si.size());
                }
                o.f64(pre + "points", xyz);
                o.i32(pre + "structure_ptr", sp);
                o.i32(pre + "structure_idx", si);
            };
            auto dump_junctions = [&](const std::string& name, const std::vector<Junction>& js) {
                std::vector<int> v;
                std::vector<double> dd;
                for (const Junction& j : js) {
                    v.insert(v.end(), {(int)j.P1, j.N1, (int)j.P2, j.N2});
                    dd.push_back(j.junction_dist);
                }
                o.i32(name, v);
                o.f64(name + "_dist", dd);
            };
            dump_points("gnpjn_");
            dump_junctions("junctions_gnp", HK3.junctions_gnp);
            int n_clusters = n_total;
            t1 = clk::now();
            if (!HK3.Make_mixed_clusters(n_total, cut3, pts, radii, CG2.sectioned_domain_cnts, gnps, CG2.sectioned_domain_gnps, lab_cnt, lab_gnp,
                                         structure_gnp, points_gnp, n_clusters))
                return 14;
            ref_seconds.push_back(secs(t1, clk::now()));
            o.f64("ref_seconds", ref_seconds);
            dump_points("mixjn_");
            dump_junctions("junctions_mixed", HK3.junctions_mixed);
            {
                // Triangulation::Generate_3d_trangulation of every GNP's points (Triangulation.cpp:12-56)
                std::vector<int> tp(1, 0), ti;
                for (size_t g = 0; g < gnps.size(); g++) {
                    GNP gc = gnps[g];
                    gc.triangulation.clear();
                    Triangulation TR;
                    if (!TR.Generate_3d_trangulation(points_gnp, structure_gnp[g], gc)) return 15;
                    for (const EdgeL& e : gc.triangulation) ti.insert(ti.end(), {(int)e.v1, (int)e.v2});
                    tp.push_back((int)ti.size() / 2);
                }
                o.i32("tri_ptr", tp);
                o.i32("tri_edges", ti);
            }
            {
                std::vector<int> ep(1, 0), ei;
                for (const auto& e : HK3.elements_cnt) {
                    for (long int v : e) ei.push_back((int)v);
                    ep.push_back((int)ei.size());
                }
                o.i32("mix_elements_ptr", ep);
                o.i32("mix_elements_idx", ei);
            }
            o.i32("mixlab_cnt", lab_cnt);
            o.i32("mixlab_gnp", lab_gnp);
            o.i32("mixlab_count", {n_clusters});
            o.i32("mix_sd_cnt_ptr", sdc_ptr);
            o.i32("mix_sd_cnt_idx", sdc_idx);
            o.i32("mix_point", mp);
            o.i32("mix_gnp", mg);
            o.i32("mix_index", mi);
            o.f64("mix_dist", md);
            o.f64("mix_contact_points", mpts);
        }
        o.i32("sd_n_regions", {nreg[0], nreg[1], nreg[2]});
        o.f64("sd_l_regions", {lreg[0], lreg[1], lreg[2]});
        o.i32("sd_ptr", sptr);
        o.i32("sd_idx", sidx);
    }
    if (FILE* qf = fopen("gnp_queries.dat", "rb")) {
        int nq = 0;
        if (fread(&nq, 4, 1, qf) != 1) nq = 0;
        std::vector<double> q(4 * (size_t)std::max(nq, 0));
        if (nq > 0 && fread(q.data(), 8, q.size(), qf) != q.size()) nq = 0;
        fclose(qf);
        Generate_Network GN;
        std::vector<double> qd, qp;
        std::vector<int> qflag;
        for (int i = 0; i < nq; i++) {
            Point_3D P(q[4 * i], q[4 * i + 1], q[4 * i + 2]);
            double dist = 0;
            Point_3D C = GN.Get_gnp_point_closest_to_point(gnps[(int)q[4 * i + 3]], P, dist);
            qd.push_back(dist);
            qp.insert(qp.end(), {C.x, C.y, C.z});
            qflag.push_back(C.flag);
        }
        o.f64("query_dist", qd);
        o.f64("query_point", qp);
        o.i32("query_flag", qflag);
    }
    if (argc >= 11 && std::string(argv[9]) == "flow") {
        // Upstream's stages for GNP_CNT_mix on window 0 = the sample, in App_Network_3D's order
        // (App_Network_3D.cpp:120-180): Shells, Cutoff_Wins::Extract_observation_window,
        // Contact_grid::Generate_contact_grid, Hoshen_Kopelman::Determine_clusters_and_percolation
        // (CNT points inside a GNP ignored), with min_points 5 and tol_gnp = 1.5 t_max.
        using fclk = std::chrono::steady_clock;
        auto fsecs = [](fclk::time_point a, fclk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
        std::vector<double> flow_seconds;  // window extraction, contact grid, clusters and percolation, electrical analysis
        auto ft0 = fclk::now();
        Geom_sample gw = geom;
        gw.win_max_x = gw.win_min_x = geom.sample.len_x;
        gw.win_max_y = gw.win_min_y = geom.sample.wid_y;
        gw.win_max_z = gw.win_min_z = geom.sample.hei_z;
        gw.win_delt_x = gw.win_delt_y = gw.win_delt_z = 0.25;
        gw.cut_num = 0;
        gw.gs_minx = gw.gs_miny = gw.gs_minz = number(argv[5]);
        gw.gs_overlap_cnt = number(argv[6]);
        gw.gs_overlap_gnp = number(argv[7]);
        std::vector<Point_3D> pts;
        std::vector<double> radii;
        std::vector<std::vector<long int> > structure;
        if (!RN.Read_cnt_data_from_dat(pts, radii, structure)) return 20;
        std::vector<std::vector<int> > shells_cnt;
        std::vector<Shell> shells_gnp(gnps.size());
        Shells SH;
        if (!SH.Generate_shells("GNP_CNT_mix", gw, pts, gnps, shells_cnt, shells_gnp)) return 21;
        const cuboid win = gw.update_observation_window_geometry(0, "GNP_CNT_mix");
        Nanotube_Geo cg;
        cg.min_points = 5;
        cg.step_length = number(argv[10]);
        std::vector<GNP> gf = gnps;
        std::vector<std::vector<long int> > sg(gnps.size());
        std::vector<Point_3D> pg;
        Cutoff_Wins CW;
        if (!CW.Extract_observation_window(0, "GNP_CNT_mix", gw, win, cg, gf, structure, radii, pts, shells_cnt, shells_gnp, sg, pg)) return 22;
        auto ft1 = fclk::now();
        flow_seconds.push_back(fsecs(ft0, ft1));
        Contact_grid CGf;
        if (!CGf.Generate_contact_grid(0, "GNP_CNT_mix", gw, win, CW.cnts_inside, pts, structure, CW.gnps_inside, gf)) return 23;
        auto ft2 = fclk::now();
        flow_seconds.push_back(fsecs(ft1, ft2));
        Simu_para sp;
        sp.particle_type = "GNP_CNT_mix";
        sp.allow_simplex3 = false;
        Visualization_flags vf;
        vf.generated_nanoparticles = vf.clusters = vf.percolated_clusters = vf.backbone = vf.triangulations = 0;
        Cutoff_dist cf = cut;
        cf.min_points = 5;
        double t_max = 0.0;
        for (const GNP& g : gf) t_max = std::max(t_max, g.t);
        cf.tol_gnp = 1.5 * t_max;
        cf.tol_gnp2 = cf.tol_gnp * cf.tol_gnp;
        Hoshen_Kopelman HF;
        HF.ignore_eror_cnt_inside_gnp = 1;
        if (!HF.Determine_clusters_and_percolation(0, geom.sample, sp, cf, vf, CW.cnts_inside, CGf.sectioned_domain_cnts, structure, pts, radii,
                                                   CW.boundary_cnt, CW.gnps_inside, CGf.sectioned_domain_gnps, gf, CW.boundary_gnp, sg, pg))
            return 24;
        auto ft3 = fclk::now();
        flow_seconds.push_back(fsecs(ft2, ft3));
        o.i32("flow_cnts_inside", CW.cnts_inside);
        o.i32("flow_gnps_inside", CW.gnps_inside);
        dump_csr(o, "flow_boundary_cnt", CW.boundary_cnt);
        dump_csr(o, "flow_boundary_gnp", CW.boundary_gnp);
        dump_csr(o, "flow_clusters_cnt", HF.clusters_cnt);
        dump_csr(o, "flow_clusters_gnp", HF.clusters_gnp);
        dump_csr(o, "flow_isolated_cnt", HF.isolated_cnt);
        dump_csr(o, "flow_isolated_gnp", HF.isolated_gnp);
        o.i32("flow_family", HF.family);
        dump_csr(o, "flow_cluster_cnt_junctions", HF.cluster_cnt_junctions);
        dump_csr(o, "flow_cluster_gnp_junctions", HF.cluster_gnp_junctions);
        dump_csr(o, "flow_cluster_mix_junctions", HF.cluster_mix_junctions);
        dump_csr(o, "flow_structure_gnp", sg);
        std::vector<double> xyz;
        for (const Point_3D& q : pg) xyz.insert(xyz.end(), {q.x, q.y, q.z});
        o.f64("flow_points_gnp", xyz);
        if (argc >= 12 && (std::string(argv[11]) == "electrical" || std::string(argv[11]) == "electrical_time")) {
            const bool staged = std::string(argv[11]) == "electrical";  // "electrical_time": the timed calls only
            if (argc >= 13) g_tol_unit = number(argv[12]);
            const bool replay = staged || g_tol_unit > 0;  // replay-only when the unit pass has its own tolerance
            // Electrical_analysis::Perform_analysis_on_clusters along x (unit-resistor pass, backbone,
            // real pass), the parameters of the hybrid configuration: rho_CNT 1e-3, GNP in-plane 1e-4
            // and through-plane 1 Ohm um, exponential tunnelling junctions (Input_Reader.cpp:1445-1456),
            // CG tolerance 1e-10; resistances.txt is read back
            Electric_para ep;
            ep.applied_voltage = 1.0;
            ep.resistivity_CNT = 1e-3;
            ep.resistivity_GNP_surf = 1e-4;
            ep.resistivity_GNP_t = 1.0;
            ep.resistivity_matrix = 1.03e20;
            ep.junction_type = "exponential";
            ep.junction_resistance = 1e7;
            ep.h_plank = 6.62606957;
            ep.e_charge = 1.60217662;
            ep.e_mass = 9.10938291;
            ep.lambda_barrier = 0.5;
            const double sq = sqrt(2.0 * ep.e_mass * ep.lambda_barrier * ep.e_charge);
            ep.C1 = 10.0 * ep.h_plank * ep.h_plank / (ep.e_mass * ep.e_mass * sq);
            ep.C2 = 4000.0 * PI * sq / ep.h_plank;
            sp.simulation_scope = 0;
            sp.resistances[0] = 1;
            sp.resistances[1] = sp.resistances[2] = 0;
            sp.tolerance = 1e-10;
            Output_data_flags of;
            of.cnt_gnp_flag = of.gnp_data = of.prec_gnp = of.cnt_data = 0;
            remove("resistances.txt");
            // state after Determine_clusters_and_percolation, for the staged replay below
            Hoshen_Kopelman HS = HF;
            std::vector<GNP> gs = gf;
            std::vector<std::vector<long int> > ss = sg;
            Electrical_analysis EA;
            auto ft4 = fclk::now();
            if (g_tol_unit <= 0) {
                if (!EA.Perform_analysis_on_clusters(0, win, sp, ep, cf, vf, of, &HF, &CW, structure, pts, radii, pg, sg, gf)) return 25;
                flow_seconds.push_back(fsecs(ft4, fclk::now()));
            }
            std::vector<double> res;
            // ---- staged replay of Perform_analysis_on_clusters (Electrical_analysis.cpp:10-145) and
            // Electrical_resistance_along_each_percolated_direction (:229-289), dumping each stage (e_*)
            if (replay) {
                std::vector<std::vector<long int> > pb;  // GNP boundary points kept by Remove_gnp_points_in_non_relevant_boundaries
                for (const GNP& g : gs) {
                    std::vector<long int> v;
                    for (const auto& q : g.pts_boundary) { v.push_back(q.first); v.push_back(q.second); }
                    pb.push_back(v);
                }
                dump_csr(o, "e_pts_boundary", pb);
                dump_csr(o, "e_structure_gnp_start", ss);
                dump_csr(o, "e_boundary_gnp_pts", CW.boundary_gnp_pts);
                dump_csr(o, "e_boundary_cnt_pts", CW.boundary_cnt_pts);
                std::vector<double> gvol, gt;
                for (const GNP& g : gs) { gvol.push_back(g.volume); gt.push_back(g.t); }
                o.f64("e_gnp_volume", gvol);
                o.f64("e_gnp_t", gt);
                std::vector<int> jm;
                std::vector<double> jmd;
                for (const Junction& q : HS.junctions_mixed) { jm.insert(jm.end(), {(int)q.P1, q.N1, (int)q.P2, q.N2}); jmd.push_back(q.junction_dist); }
                o.i32("e_junctions_mixed", jm);
                o.f64("e_junctions_mixed_dist", jmd);
                std::vector<int> jgv;
                std::vector<double> jgd;
                for (const Junction& q : HS.junctions_gnp) { jgv.insert(jgv.end(), {(int)q.P1, q.N1, (int)q.P2, q.N2}); jgd.push_back(q.junction_dist); }
                o.i32("e_junctions_gnp", jgv);
                o.f64("e_junctions_gnp_dist", jgd);
                std::vector<int> jcv;
                std::vector<double> jcd;
                for (const Junction& q : HS.junctions_cnt) { jcv.insert(jcv.end(), {(int)q.P1, q.N1, (int)q.P2, q.N2}); jcd.push_back(q.junction_dist); }
                o.i32("e_junctions_cnt", jcv);
                o.f64("e_junctions_cnt_dist", jcd);
                std::vector<std::vector<long int> > el0;
                for (const auto& e : HS.elements_cnt) el0.push_back(std::vector<long int>(e.begin(), e.end()));
                dump_csr(o, "e_elements_start", el0);
                std::vector<std::vector<double> > par(3);
                const int nclu = EA.Get_number_of_clusters(HS.clusters_cnt, HS.clusters_gnp);
                EA.Clear_triangulations(HS.clusters_gnp, gs);
                Backbone_Network* BN = new Backbone_Network;
                for (int j = 0; j < nclu; j++) {
                    const std::string pj = "e_c" + std::to_string(j) + "_";
                    Direct_Electrifying* D = new Direct_Electrifying;
                    StagedSystem su;
                    if (!staged_field(D, j, 0, win, sp, ep, cf, &HS, &CW, pts, radii, ss, pg, gs, su)) return 26;
                    dump_staged(o, pj + "u_", su);
                    {
                        Backbone_Network bz;
                        std::vector<std::vector<double> > cur;
                        double zc = 0;
                        bz.Find_zero_current(j, 0, D->voltages, D->LMM_cnts, D->LMM_gnps, &HS, cf, pts, radii, pg, gs, cur, zc);
                        o.f64(pj + "zero_current", {zc});
                    }
                    if (!BN->Determine_backbone_network(j, 0, sp.simulation_scope, 0, D->voltages, D->LMM_cnts, D->LMM_gnps, ep, cf, structure,
                                                        pts, radii, pg, ss, gs, &HS)) return 27;
                    delete D;
                    std::vector<std::vector<long int> > el;
                    for (const auto& e : HS.elements_cnt) el.push_back(std::vector<long int>(e.begin(), e.end()));
                    dump_csr(o, pj + "bb_elements", el);
                    dump_csr(o, pj + "bb_structure_gnp", ss);
                    o.i32(pj + "bb_clusters_cnt", HS.clusters_cnt.size() ? HS.clusters_cnt[j] : std::vector<int>());
                    o.i32(pj + "bb_clusters_gnp", HS.clusters_gnp.size() ? HS.clusters_gnp[j] : std::vector<int>());
                    o.i32(pj + "bb_cnt_junctions", HS.cluster_cnt_junctions.size() ? HS.cluster_cnt_junctions[j] : std::vector<int>());
                    o.i32(pj + "bb_gnp_junctions", HS.cluster_gnp_junctions.size() ? HS.cluster_gnp_junctions[j] : std::vector<int>());
                    o.i32(pj + "bb_mix_junctions", HS.cluster_mix_junctions.size() ? HS.cluster_mix_junctions[j] : std::vector<int>());
                    if (sp.simulation_scope) continue;
                    if (HS.clusters_gnp.size() && j) EA.Clear_triangulations_of_cluster(HS.clusters_gnp[j - 1], gs);
                    std::vector<int> dirs;
                    if (!EA.Vector_of_directions(HS.family[j], sp, dirs)) return 28;
                    const int family = HS.family[j];
                    for (int d : dirs) {
                        Direct_Electrifying* DR = new Direct_Electrifying;
                        HS.family[j] = d;
                        StagedSystem sr;
                        if (!staged_field(DR, j, 1, win, sp, ep, cf, &HS, &CW, pts, radii, ss, pg, gs, sr)) return 29;
                        const size_t before = par[d].size();
                        if (!EA.Calculate_parallel_resistor(d, j, ep, DR, pts, radii, HS.elements_cnt, HS.clusters_cnt, CW.boundary_cnt, pg, gs,
                                                            HS.clusters_gnp, CW.boundary_gnp, par)) return 30;
                        const std::string pd = pj + "d" + std::to_string(d) + "_";
                        dump_staged(o, pd, sr);
                        o.f64(pd + "R", {par[d].size() > before ? par[d].back() : 0.0});
                        delete DR;
                    }
                    HS.family[j] = family;
                }
                std::vector<double> vols;
                for (double v : BN->volumes_cnt) vols.push_back(v);
                for (double v : BN->volumes_gnp) vols.push_back(v);
                for (double v : BN->dead_branches) vols.push_back(v);
                for (double v : BN->dead_gnps) vols.push_back(v);
                o.f64("e_bn_volumes", vols);
                delete BN;
                if (g_tol_unit > 0) {
                    // Calculate_resistances_and_resistivities (Electrical_analysis.cpp:873-987): parallel
                    // resistors of each direction, the matrix resistance where none percolates
                    const double len[3] = {win.len_x, win.wid_y, win.hei_z};
                    const double area[3] = {win.wid_y * win.hei_z, win.len_x * win.hei_z, win.len_x * win.wid_y};
                    for (int d = 0; d < 3; d++) {
                        if (par[d].empty()) {
                            res.push_back(ep.resistivity_matrix * len[d] / area[d]);
                            continue;
                        }
                        if (par[d].size() == 1) {
                            res.push_back(par[d].front());
                            continue;
                        }
                        double inv = 0;
                        for (double r : par[d]) inv = inv + 1 / r;
                        res.push_back(1 / inv);
                    }
                    flow_seconds.push_back(fsecs(ft4, fclk::now()));
                }
            }
            o.f64("flow_seconds", flow_seconds);
            if (g_tol_unit <= 0)
                if (FILE* rf = fopen("resistances.txt", "r")) {
                    double v;
                    while (fscanf(rf, "%lf", &v) == 1) res.push_back(v);
                    fclose(rf);
                }
            o.f64("flow_resistances", res);
        }
    }
    o.i32("junc_pair", jn_pair);
    o.i32("junc_ok", jn_ok);
    o.i32("junc_outside", jn_out);
    o.f64("junc_points", jn_pts);
    o.i32("pair_a", pa);
    o.i32("pair_b", pb);
    o.i32("pair_penetrating", pflag);
    o.f64("pair_dist", dist);
    o.f64("pair_direction", dir);
    o.f64("pair_displacement", disp);
    fclose(o.f);
    return 0;
}
