/*
 * ref_dump — TEST ORACLE DRIVER (never shipped, never on the product path).
 *
 * Links the unmodified upstream CICY_geom objects (compiled in place from the
 * upstream tree by oracle/Makefile, with oracle/ref_compat.h force-included)
 * and replays the single-window network-to-conductance path of
 * App_Network_3D::Generate_nanoparticle_resistor_network
 * (App_Network_3D.cpp:11-186) on a `Read_Network` input directory, either
 *
 *   ref_dump dump <dir> <out.bin> [tol_unit]
 *                                   dumping every intermediate the hot path
 *                                   produces (window-trimmed network,
 *                                   sectioned domain, raw point contacts,
 *                                   labels, junctions, elements, percolated
 *                                   clusters, each DEA system and solution,
 *                                   the backbone, resistances), or
 *   ref_dump time <dir> [tol_unit [reps]]
 *                                   running the hot path `reps` times on the
 *                                   window (fresh objects each time) and
 *                                   printing per-stage steady_clock times, with
 *                                   the hot path's start and end on the
 *                                   system-wide monotonic clock, as one JSON
 *                                   line per repetition (the CPU baseline), or
 *   ref_dump app <dir>              calling the upstream top-level
 *                                   App_Network_3D unchanged (it appends
 *                                   resistances.txt in <dir>).
 *
 * The electrical stage is replayed call-by-call from
 * Electrical_analysis::Perform_analysis_on_clusters (Electrical_analysis.cpp:10-145)
 * and Direct_Electrifying::Compute_voltage_field (Direct_Electrifying.cpp:11-113)
 * using only their public member functions, so the DEA matrices and voltages
 * can be captured; `app` mode exists to check that this replay and the
 * upstream top level give identical resistances.
 *
 * Upstream solves every DEA system to the one Simulation_Parameters tolerance
 * of input.dat.  The optional `tol_unit` gives the unit-resistor systems (the
 * ones whose currents classify the backbone, Backbone_Network.cpp:64-242) their
 * own tolerance, as the device path's cicy_params.tolerance_unit does; the
 * real-resistor systems keep the input.dat tolerance.  Without it the replay
 * is upstream's exactly.
 */
#include "Hns.h"
using namespace hns;
#include "Input_Reader.h"
#include "Read_Network.h"
#include "Shells.h"
#include "Cutoff_Wins.h"
#include "Contact_grid.h"
#include "Hoshen_Kopelman.h"
#include "Direct_Electrifying.h"
#include "Backbone_Network.h"
#include "Electrical_analysis.h"
#include "App_Network_3D.h"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <unistd.h>

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Minimal named-array container: [u32 name_len][name][u8 type][u64 count][payload]
// type: 'i' int32, 'l' int64, 'd' float64.
struct Dump {
    FILE* f = nullptr;
    void open(const char* path) { f = fopen(path, "wb"); }
    void close() { if (f) fclose(f); f = nullptr; }
    void raw(const std::string& name, char type, const void* data, uint64_t count, size_t elsz) {
        if (!f) return;
        uint32_t nl = (uint32_t)name.size();
        fwrite(&nl, 4, 1, f);
        fwrite(name.data(), 1, nl, f);
        fwrite(&type, 1, 1, f);
        fwrite(&count, 8, 1, f);
        if (count) fwrite(data, elsz, count, f);
    }
    void i32(const std::string& n, const std::vector<int>& v) { raw(n, 'i', v.data(), v.size(), 4); }
    void i64(const std::string& n, const std::vector<long int>& v) { raw(n, 'l', v.data(), v.size(), 8); }
    void f64(const std::string& n, const std::vector<double>& v) { raw(n, 'd', v.data(), v.size(), 8); }
    template <class T>
    void csr_i32(const std::string& n, const std::vector<std::vector<T> >& vv) {
        std::vector<long int> ptr(1, 0);
        std::vector<int> idx;
        for (auto& v : vv) { for (auto x : v) idx.push_back((int)x); ptr.push_back((long int)idx.size()); }
        i64(n + "_ptr", ptr); i32(n + "_idx", idx);
    }
    template <class T>
    void csr_i64(const std::string& n, const std::vector<std::vector<T> >& vv) {
        std::vector<long int> ptr(1, 0);
        std::vector<long int> idx;
        for (auto& v : vv) { for (auto x : v) idx.push_back((long int)x); ptr.push_back((long int)idx.size()); }
        i64(n + "_ptr", ptr); i64(n + "_idx", idx);
    }
    void sets(const std::string& n, const std::vector<std::set<long int> >& vv) {
        std::vector<long int> ptr(1, 0), idx;
        for (auto& s : vv) { for (auto x : s) idx.push_back(x); ptr.push_back((long int)idx.size()); }
        i64(n + "_ptr", ptr); i64(n + "_idx", idx);
    }
};

struct Captured {
    long int nodes = 0, reserved = 0;
    std::vector<long int> row_ptr, col_ind;
    std::vector<double> values, diagonal, b, x0, vef, voltages;
    std::vector<long int> lmm_pts, lmm_nodes;
    double t_assembly = 0, t_solve = 0;
};

// Direct_Electrifying::Compute_voltage_field (Direct_Electrifying.cpp:11-113), CNT-only
// branches, with the intermediate system captured.
// Tolerance of the unit-resistor (R_flag = 0) solves; <= 0: the input.dat tolerance.
double g_tol_unit = 0.0;

int compute_voltage_field(Direct_Electrifying* D, int n_cluster, int R_flag, const cuboid& window, Input* I,
                          Hoshen_Kopelman* HoKo, Cutoff_Wins* CW, std::vector<Point_3D>& points,
                          std::vector<double>& radii, std::vector<std::vector<long int> >& sg,
                          std::vector<Point_3D>& pg, std::vector<GNP>& gnps, Captured* cap) {
    double t0 = now_s();
    int reserved = D->Get_global_nodes(HoKo->family[n_cluster]);
    if (reserved == -1) return 0;
    long int global_nodes = reserved;
    if (HoKo->clusters_cnt.size() && HoKo->clusters_cnt[n_cluster].size())
        if (!D->LM_matrix_for_cnts(n_cluster, HoKo, CW, global_nodes)) return 0;
    std::vector<long int> col_ind, row_ptr;
    std::vector<double> values, diagonal(global_nodes, 0), R(global_nodes - reserved, 0), VEF(reserved, 0.0);
    if (!D->Fill_sparse_stiffness_matrix(R_flag, global_nodes, reserved, I->cutoff_dist.van_der_Waals_dist, n_cluster,
                                         I->electric_para, HoKo, points, radii, sg, pg, gnps, col_ind, row_ptr, values,
                                         diagonal, R, VEF))
        return 0;
    std::vector<double> V_guess(global_nodes - reserved, 0.0);
    if (cap) cap->b = R;
    if (R_flag && reserved == 2) {
        if (!D->Initial_guess_for_CG(n_cluster, reserved, HoKo->family[n_cluster], window, I->electric_para.applied_voltage,
                                     HoKo->clusters_cnt, HoKo->elements_cnt, points, HoKo->clusters_gnp, pg, R, V_guess))
            return 0;
        if (!D->Update_residual_vector(col_ind, row_ptr, values, diagonal, V_guess, R)) return 0;
    }
    if (cap) cap->x0 = V_guess;
    double t1 = now_s();
    const double tol = (!R_flag && g_tol_unit > 0) ? g_tol_unit : I->simu_para.tolerance;
    if (!D->Solve_DEA_equations_CG_SSS(global_nodes, reserved, tol, col_ind, row_ptr, values, diagonal, R, VEF, V_guess))
        return 0;
    double t2 = now_s();
    if (cap) {
        cap->nodes = global_nodes;
        cap->reserved = reserved;
        cap->row_ptr = row_ptr;
        cap->col_ind = col_ind;
        cap->values = values;
        cap->diagonal = diagonal;
        cap->vef = VEF;
        cap->voltages = D->voltages;
        cap->lmm_pts.clear();
        cap->lmm_nodes.clear();
        for (auto& kv : D->LMM_cnts) { cap->lmm_pts.push_back(kv.first); cap->lmm_nodes.push_back(kv.second); }
        cap->t_assembly = t1 - t0;
        cap->t_solve = t2 - t1;
    }
    return 1;
}

void dump_system(Dump& d, const std::string& p, const Captured& c) {
    d.i64(p + "nodes", std::vector<long int>{c.nodes, c.reserved});
    d.i64(p + "row_ptr", c.row_ptr);
    d.i64(p + "col_ind", c.col_ind);
    d.f64(p + "values", c.values);
    d.f64(p + "diag", c.diagonal);
    d.f64(p + "b", c.b);
    d.f64(p + "x0", c.x0);
    d.f64(p + "vef", c.vef);
    d.f64(p + "voltages", c.voltages);
    d.i64(p + "lmm_pts", c.lmm_pts);
    d.i64(p + "lmm_nodes", c.lmm_nodes);
    d.f64(p + "times", std::vector<double>{c.t_assembly, c.t_solve});
}

int run_staged(const char* dir, const char* dump_path, bool timing_json, int reps) {
    if (chdir(dir) != 0) { fprintf(stderr, "cannot chdir to %s\n", dir); return 2; }
    open_deffo_stream((char*)"ref_log.txt");
    Dump d;
    if (dump_path) d.open(dump_path);

    Input* I = new Input;
    if (!I->Data_Initialization()) return 3;
    std::ifstream infile("input.dat");
    if (!infile || !I->Read_input_file(infile)) { fprintf(stderr, "bad input.dat\n"); return 3; }
    infile.close();

    double T[16] = {0};
    std::vector<Point_3D> points;
    std::vector<double> radii;
    std::vector<std::vector<long int> > structure;
    std::vector<GNP> gnps;
    std::vector<std::vector<int> > shells_cnts;

    double t0 = now_s();
    Read_Network* RN = new Read_Network;
    if (!RN->Generate_nanoparticle_network_from_file(I->simu_para, I->vis_flags, I->geom_sample, points, radii, structure, gnps)) return 4;
    delete RN;
    double t1 = now_s();
    std::vector<Shell> shell_gnps(gnps.size());
    Shells* SH = new Shells;
    if (!SH->Generate_shells(I->simu_para.particle_type, I->geom_sample, points, gnps, shells_cnts, shell_gnps)) return 4;
    delete SH;
    double t2 = now_s();
    std::vector<Point_3D> points_gnp;
    std::vector<std::vector<long int> > structure_gnp;
    cuboid window = I->geom_sample.update_observation_window_geometry(0, I->simu_para.particle_type);
    Cutoff_Wins* CW = new Cutoff_Wins;
    if (!CW->Extract_observation_window(0, I->simu_para.particle_type, I->geom_sample, window, I->nanotube_geo, gnps, structure,
                                        radii, points, shells_cnts, shell_gnps, structure_gnp, points_gnp)) return 5;
    double t3 = now_s();

    if (dump_path) {
        d.f64("window", {window.poi_min.x, window.poi_min.y, window.poi_min.z, window.len_x, window.wid_y, window.hei_z,
                         window.max_x, window.max_y, window.max_z});
        const Geom_sample& g = I->geom_sample;
        d.f64("params", {g.gs_minx, g.gs_miny, g.gs_minz, g.gs_overlap_cnt, g.gs_overlap_gnp,
                         I->cutoff_dist.van_der_Waals_dist, I->cutoff_dist.tunneling_dist, (double)I->cutoff_dist.min_points,
                         I->electric_para.applied_voltage, I->electric_para.resistivity_CNT, I->electric_para.C1,
                         I->electric_para.C2, I->electric_para.resistivity_matrix, I->simu_para.tolerance,
                         I->nanotube_geo.step_length, (double)I->nanotube_geo.min_points});
        std::vector<double> xyz;
        std::vector<int> flag;
        xyz.reserve(points.size() * 3);
        for (auto& p : points) { xyz.push_back(p.x); xyz.push_back(p.y); xyz.push_back(p.z); flag.push_back(p.flag); }
        d.f64("points_xyz", xyz);
        d.i32("points_flag", flag);
        d.csr_i64("structure", structure);
        d.f64("radii", radii);
        d.i32("cnts_inside", CW->cnts_inside);
        d.csr_i32("boundary_cnt", CW->boundary_cnt);
        d.csr_i64("boundary_pts", CW->boundary_cnt_pts);
    }

    // The hot path (contact grid, clusters, electrical analysis) `reps` times on the
    // same window, each on fresh objects and a fresh copy of the window's network;
    // only the first repetition is dumped.
    const std::vector<Point_3D> points0 = points;
    const std::vector<std::vector<long int> > structure0 = structure;
    const std::vector<double> radii0 = radii;
    for (int rep = 0; rep < reps; rep++) {
        const bool dumping = dump_path && rep == 0;
        if (rep) { points = points0; structure = structure0; radii = radii0; }
        double t4 = now_s();
        Contact_grid* CG = new Contact_grid;
        if (!CG->Generate_contact_grid(0, I->simu_para.particle_type, I->geom_sample, window, CW->cnts_inside, points, structure,
                                       CW->gnps_inside, gnps)) return 6;
        double t5 = now_s();
        Hoshen_Kopelman* HoKo = new Hoshen_Kopelman;
        if (!HoKo->Determine_clusters_and_percolation(0, I->geom_sample.sample, I->simu_para, I->cutoff_dist, I->vis_flags,
                                                      CW->cnts_inside, CG->sectioned_domain_cnts, structure, points, radii,
                                                      CW->boundary_cnt, CW->gnps_inside, CG->sectioned_domain_gnps, gnps,
                                                      CW->boundary_gnp, structure_gnp, points_gnp)) return 7;
        double t6 = now_s();

        if (dumping) {
            d.csr_i64("sd", CG->sectioned_domain_cnts);
            // Raw point contacts and labels: a second, independent call of the public
            // Hoshen_Kopelman::Label_cnts_in_window (Hoshen_Kopelman.cpp:249-372) + Cleanup_labels.
            Hoshen_Kopelman hk2;
            std::vector<int> labels(structure.size(), -1), ll;
            std::vector<std::map<int, std::set<long int> > > ce(radii.size());
            std::map<long int, std::map<int, long int> > pc;
            std::map<long int, std::map<int, double> > pcd;
            hk2.Label_cnts_in_window(points, radii, I->cutoff_dist, CG->sectioned_domain_cnts, pc, pcd, ce, labels, ll);
            int n_labels = 0;
            std::vector<int> labels_raw = labels;
            hk2.Cleanup_labels(ll, labels, n_labels);
            std::vector<long int> pa, pb;
            std::vector<int> cb;
            std::vector<double> dist;
            for (auto& a : pc)
                for (auto& b : a.second) {
                    pa.push_back(a.first); cb.push_back(b.first); pb.push_back(b.second);
                    dist.push_back(pcd.at(a.first).at(b.first));
                }
            d.i64("pc_Pa", pa); d.i32("pc_CNTb", cb); d.i64("pc_Pb", pb); d.f64("pc_dist", dist);
            d.i32("labels_cnt", labels);
            d.i32("n_labels", {n_labels});
            std::vector<long int> jp1, jp2;
            std::vector<int> jn1, jn2;
            std::vector<double> jd;
            for (auto& j : HoKo->junctions_cnt) { jp1.push_back(j.P1); jn1.push_back(j.N1); jp2.push_back(j.P2); jn2.push_back(j.N2); jd.push_back(j.junction_dist); }
            d.i64("junc_P1", jp1); d.i32("junc_N1", jn1); d.i64("junc_P2", jp2); d.i32("junc_N2", jn2); d.f64("junc_dist", jd);
            d.sets("elements", HoKo->elements_cnt);
            d.csr_i32("clusters", HoKo->clusters_cnt);
            d.csr_i32("isolated", HoKo->isolated_cnt);
            d.i32("family", HoKo->family);
            d.csr_i32("cluster_junc", HoKo->cluster_cnt_junctions);
        }
        delete CG;

        // ---- Electrical_analysis::Perform_analysis_on_clusters (Electrical_analysis.cpp:10-145), replayed
        double t7 = now_s();
        Electrical_analysis EA;
        std::vector<std::vector<double> > parallel(3, std::vector<double>());
        int n_clusters = EA.Get_number_of_clusters(HoKo->clusters_cnt, HoKo->clusters_gnp);
        Backbone_Network* BN = new Backbone_Network;
        double t_unit = 0, t_bb = 0, t_real = 0;
        for (int j = 0; j < n_clusters; j++) {
            std::string pj = "c" + std::to_string(j) + "_";
            double a0 = now_s();
            Direct_Electrifying* DEA = new Direct_Electrifying;
            Captured cu;
            if (!compute_voltage_field(DEA, j, 0, window, I, HoKo, CW, points, radii, structure_gnp, points_gnp, gnps, dumping ? &cu : nullptr)) return 8;
            double a1 = now_s();
            if (dumping) {
                dump_system(d, pj + "u_", cu);
                Backbone_Network bz;
                std::vector<std::vector<double> > cur;
                double zc = 0;
                bz.Find_zero_current(j, 0, DEA->voltages, DEA->LMM_cnts, DEA->LMM_gnps, HoKo, I->cutoff_dist, points, radii, points_gnp, gnps, cur, zc);
                d.f64(pj + "zero_current", {zc});
                std::vector<double> flat;
                for (auto& v : cur) for (auto x : v) flat.push_back(x);
                d.f64(pj + "elem_currents", flat);
            }
            if (!BN->Determine_backbone_network(j, 0, I->simu_para.simulation_scope, 0, DEA->voltages, DEA->LMM_cnts, DEA->LMM_gnps,
                                                I->electric_para, I->cutoff_dist, structure, points, radii, points_gnp, structure_gnp, gnps, HoKo)) return 9;
            delete DEA;
            double a2 = now_s();
            if (dumping) {
                d.sets(pj + "bb_elements", HoKo->elements_cnt);
                d.i32(pj + "bb_cluster", HoKo->clusters_cnt[j]);
                d.i32(pj + "bb_junc", HoKo->cluster_cnt_junctions.size() ? HoKo->cluster_cnt_junctions[j] : std::vector<int>());
            }
            if (!I->simu_para.simulation_scope) {
                // Electrical_analysis::Electrical_resistance_along_each_percolated_direction (Electrical_analysis.cpp:229-289)
                std::vector<int> dirs;
                if (!EA.Vector_of_directions(HoKo->family[j], I->simu_para, dirs)) return 10;
                int family = HoKo->family[j];
                for (size_t k = 0; k < dirs.size(); k++) {
                    Direct_Electrifying* DR = new Direct_Electrifying;
                    HoKo->family[j] = dirs[k];
                    Captured cr;
                    if (!compute_voltage_field(DR, j, 1, window, I, HoKo, CW, points, radii, structure_gnp, points_gnp, gnps, dumping ? &cr : nullptr)) return 11;
                    size_t before = parallel[dirs[k]].size();
                    if (!EA.Calculate_parallel_resistor(dirs[k], j, I->electric_para, DR, points, radii, HoKo->elements_cnt, HoKo->clusters_cnt,
                                                        CW->boundary_cnt, points_gnp, gnps, HoKo->clusters_gnp, CW->boundary_gnp, parallel)) return 12;
                    if (dumping) {
                        std::string pd = pj + "d" + std::to_string(dirs[k]) + "_";
                        dump_system(d, pd, cr);
                        d.f64(pd + "R", {parallel[dirs[k]].size() > before ? parallel[dirs[k]].back() : 0.0});
                    }
                    delete DR;
                }
                HoKo->family[j] = family;
            }
            double a3 = now_s();
            t_unit += a1 - a0; t_bb += a2 - a1; t_real += a3 - a2;
        }
        // Electrical_analysis::Calculate_resistances_and_resistivities (Electrical_analysis.cpp:873-932)
        std::vector<double> resistors(3, 0);
        for (int i = 0; i < 3; i++) {
            if (parallel[i].empty()) EA.Calculate_matrix_resistance(i, window, I->electric_para.resistivity_matrix, resistors[i]);
            else if (parallel[i].size() == 1) resistors[i] = parallel[i].front();
            else { double R = 0; for (double r : parallel[i]) R = R + 1 / r; resistors[i] = 1 / R; }
        }
        // the backbone's volumes before the fractions step, then
        // Electrical_analysis::Calculate_percolated_families_fractions (Electrical_analysis.cpp:678-756),
        // the last call of Perform_analysis_on_clusters (:114-119): volumes_cnt[7] = dead + non-percolated
        const std::vector<double> bn_volumes = {BN->volumes_cnt[0], BN->volumes_cnt[1], BN->volumes_cnt[2],
                                                BN->dead_branches[0], BN->dead_branches[1], BN->dead_branches[2]};
        if (!EA.Calculate_percolated_families_fractions(I->out_flags.cnt_gnp_flag, structure, points, radii, gnps, HoKo, BN)) return 13;
        double t8 = now_s();
        if (dumping) {
            d.f64("resistances", resistors);
            d.f64("bn_volumes", bn_volumes);
            d.f64("bn_volumes_cnt", BN->volumes_cnt);
            d.f64("bn_volumes_gnp", BN->volumes_gnp);
            d.f64("bn_dead_branches", BN->dead_branches);
            d.f64("bn_dead_gnps", BN->dead_gnps);
            d.f64("stage_times", {t1 - t0, t2 - t1, t3 - t2, t5 - t4, t6 - t5, t8 - t7, t_unit, t_bb, t_real});
            d.close();
        }
        delete BN;
        if (timing_json) {
            printf("{\"read_s\": %.6f, \"shells_s\": %.6f, \"window_s\": %.6f, \"grid_s\": %.6f, \"hk_s\": %.6f, "
                   "\"ea_s\": %.6f, \"unit_dea_s\": %.6f, \"backbone_s\": %.6f, \"real_dea_s\": %.6f, \"hot_s\": %.6f, "
                   "\"n_points\": %ld, \"n_clusters\": %d, \"R\": [%.17g, %.17g, %.17g], \"rep\": %d, "
                   "\"t_start\": %.6f, \"t_end\": %.6f}\n",
                   t1 - t0, t2 - t1, t3 - t2, t5 - t4, t6 - t5, t8 - t7, t_unit, t_bb, t_real, (t6 - t4) + (t8 - t7),
                   (long)points.size(), n_clusters, resistors[0], resistors[1], resistors[2], rep, t4, t8);
            fflush(stdout);
        }
        delete HoKo;
    }
    delete CW;
    delete I;
    return 0;
}

int run_app(const char* dir) {
    if (chdir(dir) != 0) return 2;
    open_deffo_stream((char*)"ref_log.txt");
    Input* I = new Input;
    if (!I->Data_Initialization()) return 3;
    std::ifstream infile("input.dat");
    if (!infile || !I->Read_input_file(infile)) return 3;
    infile.close();
    App_Network_3D app;
    double t0 = now_s();
    int ok = app.Generate_nanoparticle_resistor_network(I);
    double t1 = now_s();
    printf("{\"ok\": %d, \"wall_s\": %.6f}\n", ok, t1 - t0);
    delete I;
    return ok ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc >= 4 && std::string(argv[1]) == "dump") {
        if (argc >= 5) g_tol_unit = atof(argv[4]);
        return run_staged(argv[2], argv[3], false, 1);
    }
    if (argc >= 3 && std::string(argv[1]) == "time") {
        if (argc >= 4) g_tol_unit = atof(argv[3]);
        const int reps = argc >= 5 ? atoi(argv[4]) : 1;
        return run_staged(argv[2], nullptr, true, reps < 1 ? 1 : reps);
    }
    if (argc >= 3 && std::string(argv[1]) == "app") return run_app(argv[2]);
    fprintf(stderr, "usage: ref_dump dump <dir> <out.bin> [tol_unit] | time <dir> [tol_unit [reps]] | app <dir>\n");
    return 1;
}
