// The device context behind `cicy_ctx`: one network's device buffers, the
// stream, and the host-side bookkeeping of the stage sequence.
#pragma once

#include <vector>

#include "dev_common.cuh"
#include "solver.cuh"

namespace cicy {

// Region grid of Contact_grid::Generate_contact_grid / Adjust_regions_if_needed.
struct GridGeom {
    int n[3];
    double l[3];
    double min[3];
    double overlap;  // Geom_sample::gs_overlap_cnt
    long long total;
};

// One assembled DEA system kept for copy-out and for the backbone/current steps.
struct DeaSystem {
    int cluster = -1, pass = -2;  // pass -1: unit resistors; 0,1,2: real, along x,y,z
    int64_t nodes = 0, reserved = 0, nnz_lower = 0, iterations = 0;
    int restarts = 0;
    bool cluster_solver = false;
    int mg_levels = 0;
    int fallback = 0;  // 1: the learned preconditioner failed and Jacobi-PCG solved the system
    std::vector<int32_t> h_chain_start, h_chain_len;
    // scalar fields back to their defaults (device buffers are kept)
    void reset() {
        cluster = -1;
        pass = -2;
        nodes = reserved = nnz_lower = iterations = 0;
        restarts = 0;
        cluster_solver = false;
        mg_levels = 0;
        fallback = 0;
        rel_residual = seconds = 0;
        h_chain_start.clear();
        h_chain_len.clear();
    }
    double rel_residual = 0, seconds = 0;
    // device: strict-lower CSR of the free block (SSS), diagonal, rhs, x0, voltages (all nodes)
    DBuf<int32_t> row_ptr, col;
    DBuf<double> val, diag, b, x0, volt;
};

// The GNP side of a mixed CNT/GNP network for its electrical stage (hybrid_dea.cuh):
// upstream's GNP members after Determine_clusters_and_percolation, on the device,
// and the working state of the DEA passes.
struct HybridDev {
    int n_gnps = 0, n_pts = 0, n_clusters = 0;
    double rs = 0, rt = 0;              // GNP in-plane and through-plane resistivity
    int n_tri_pass = 0;                 // triangulation edges of the system being assembled
    DBuf<double> pts;                   // GNP points, xyz
    DBuf<int32_t> sptr, sidx, scount;   // structure_gnp: capacity CSR, current length per GNP (kept points at the front)
    DBuf<int32_t> nb;                   // boundary points per GNP (GNP::pts_boundary.size())
    DBuf<double> t, vol, geom;          // thickness, volume, triangulation frame (l, centre[3], rotation[9], face-0 normal[3])
    DBuf<int32_t> bg_idx, bgp_idx;      // boundary_gnp, boundary_gnp_pts (six faces)
    std::vector<int32_t> h_bg_ptr, h_bgp_ptr;
    int n_jg = 0, n_jm = 0;             // junctions_gnp, junctions_mixed (P1, N1, P2, N2, distance)
    DBuf<int32_t> jg_p1, jg_n1, jg_p2, jg_n2, jm_p1, jm_n1, jm_p2, jm_n2;
    DBuf<double> jg_d, jm_d;
    // per cluster: GNP list and junction lists (the junction lists shrink in the backbone)
    std::vector<int32_t> h_cg_ptr, h_cgj_ptr, h_cmj_ptr, cgj_len, cmj_len;
    DBuf<int32_t> cg_idx, cgj_idx, cmj_idx;
    // per pass
    DBuf<int32_t> lmm_g, rad_from, tri_cnt, tri, gcnt, goff, pt_removed, alive, alive_scan, tmp_list, seg_start;
    DBuf<double> cnt_rad, bterm;
    DBuf<int32_t> bvalid, boff, elem_removed, removed_cnt, to_remove, mix_alive, gj_alive, live, elem_tmp;
    DBuf<uint64_t> key;
    DBuf<uint32_t> val;
    DBuf<unsigned char> tri_work;
    DBuf<double> vol_acc;               // volumes_cnt[8], volumes_gnp[8], dead_branches[7], dead_gnps[7]
};

// The GNP part of one DEA system of a mixed cluster (lists on the device).
struct GnpPass {
    HybridDev* hy;
    const int32_t* gnps;
    int n_gnps;
    const int32_t* mix;
    int n_mix;
    const int32_t* gj;
    int n_gj;
};

struct Ctx {
    Ctx() = default;
    Ctx(const Ctx&) = delete;
    Ctx& operator=(const Ctx&) = delete;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // second stream for the backbone and family volumes, which no later stage of the step reads:
    // they run beside the real-resistor pass (events order them after their inputs and before
    // the results are read)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_main = nullptr, ev_side = nullptr;
    std::string err;
    int64_t launches = 0;
    int stage = 0;  // 1 uploaded, 2 grid, 3 clusters, 4 electrical
    cicy_solver_opts solver{CICY_PRECISION_FP64, CICY_PRECOND_JACOBI, 300, 0};
    int num_sms = 148;

    // ---- network (device) ----
    int n_points = 0, n_cnts = 0, n_inside = 0, n_trav = 0;
    cicy_cuboid window{};
    DBuf<double> x, y, z, radii;
    DBuf<int32_t> flag, cstart, clen, inside, trav_off, trav_pt;
    std::vector<int32_t> h_bcnt_ptr, h_bcnt_idx, h_bpts_ptr;  // host copies of the face lists (sizes)
    DBuf<int32_t> bcnt_idx, bpts_idx, bcnt_ptr, bpts_ptr;
    std::vector<int32_t> h_cstart, h_clen;

    // ---- grid ----
    GridGeom grid{};
    int n_slots = 0;
    DBuf<int32_t> region_cnt, region_ptr, region_cur, slot_region, seg_large;
    DBuf<uint32_t> slot_q, slot_sorted;
    DBuf<int> status;      // device status word (DevErr)
    DBuf<int32_t> i32_scalar;  // small device scalars for totals
    DBuf<int64_t> i64_scalar;

    // ---- contacts / labels ----
    int n_raw = 0, n_uc = 0, n_labels = 0, n_junc = 0, n_perc = 0;
    DBuf<int32_t> raw_a, raw_b, raw_pa, raw_pb;
    DBuf<double> raw_d;
    DBuf<uint64_t> raw_key;
    DBuf<int32_t> raw_count;
    DBuf<uint64_t> sort_k;
    DBuf<uint32_t> sort_v;
    DBuf<int32_t> flags, flags_scan;
    DBuf<int32_t> uc_a, uc_b, uc_pa, uc_pb;
    DBuf<double> uc_d;
    DBuf<int32_t> parent, uf_root, labels, root_rank;
    DBuf<unsigned long long> minkey;
    DBuf<int32_t> grp_start, junc_cnt, junc_ofs;
    DBuf<int32_t> j_p1, j_n1, j_p2, j_n2;
    DBuf<double> j_d;
    DBuf<int32_t> mark, mark_scan, elem_idx, has_junc;
    DBuf<int32_t> face_bits, perc_bits, perc_index;
    std::vector<int32_t> h_family;  // family of each percolated cluster
    DBuf<int32_t> clu_ptr, clu_idx, cj_ptr, cj_idx;          // percolated clusters (after percolation)
    std::vector<int32_t> h_clu_ptr, h_cj_ptr;
    // backbone state: kept element range per CNT, alive flags, trimmed cluster lists
    DBuf<int32_t> bb_lo, bb_hi;                              // element-list index range kept per CNT (-1 dead)
    DBuf<int32_t> bbclu_ptr, bbclu_idx, bbcj_ptr, bbcj_idx;  // clusters/junctions after backbone
    std::vector<int32_t> h_bbclu_ptr, h_bbcj_ptr;
    bool have_backbone = false;

    // ---- DEA ----
    std::vector<DeaSystem*> systems;
    std::vector<DeaSystem*> sys_pool;  // systems of earlier runs, reused
    DBuf<int32_t> lmm;         // node of each point in the current solve (-1 none)
    DBuf<int32_t> cnt_nodes, cnt_node_base, cnt_fresh, claim;
    DBuf<int32_t> e_n1, e_n2, e_op;
    DBuf<double> e_g;
    DBuf<int32_t> work_i32a, work_i32b, work_i32c;
    DBuf<double> work_f64a;
    RadixScratch rs;
    RadixScratch rs_side;  // sorts issued on `side`
    DBuf<int32_t> scan_tmp32;
    DBuf<int64_t> scan_tmp64;
    // CG scratch
    DBuf<int32_t> cg_rp, cg_ci;
    DBuf<double> cg_val, cg_minv, cg_x, cg_r, cg_p, cg_q, cg_z, cg_w, cg_s, cg_part;
    DBuf<unsigned int> barrier;
    DBuf<double> cg_scal;
    DBuf<long long> cg_iters;
    // assembly / backbone scratch
    DBuf<uint64_t> dkey, stage_keys;
    DBuf<uint32_t> dval;
    DBuf<double> runval, vef, cur_out, bterm;
    DBuf<int32_t> bvalid;
    DBuf<int32_t> eb, ee, alive, alive_scan, tmp_list;
    DBuf<unsigned long long> imax;
    std::vector<int32_t> bb_clu_len, bb_cj_len;
    // backbone volumes: per-CNT parts of the cluster being classified, the isolated-list sort,
    // and the volume members (volumes_cnt[8], dead_branches[7], total_volumes[8], fractions[8])
    DBuf<double> vol3, vol_acc;
    DBuf<int32_t> vol_kind;
    DBuf<int32_t> bb_pts;  // per backbone member: CNT, end points and cut points of its current-carrying part
    DBuf<uint64_t> vol_key;
    DBuf<uint32_t> vol_cnt;
    DBuf<double> vol_iso;               // whole-CNT volumes of the isolated list
    bool have_volumes = false;
    HybridDev* hy = nullptr;  // mixed CNT/GNP electrical stage (cicy_hybrid_electrical)
    bool have_hybrid = false;
    DBuf<int32_t> chain_start, chain_len;
    SolverWork sw;
    GnnState gnn;
    DBuf<float> gnn_params;  // learned preconditioner parameters (cicy_ctx_set_learned_params)

    // ---- network construction on the device (stage_window.cu) ----
    DBuf<int32_t> win_cnt, win_first, win_slot, win_nev, win_face, win_off, win_keep, win_pos;
    DBuf<int32_t> win_prun, win_pparent, win_pnev, win_cs, win_cl, win_raw_p, win_raw_c;
    DBuf<int64_t> win_ev, win_pev;
    DBuf<double> win_rad;

    // ---- CNT-GNP contacts (cicy_gnp_cnt_contacts), indexed by contact-point number ----
    int n_mix = 0;
    DBuf<int32_t> mix_point, mix_gnp;
    DBuf<double> mix_dist, mix_closest;
    std::vector<int32_t> h_mixj;        // cicy_mixed_junctions results
    std::vector<double> h_mixj_dist, h_mixj_points;

    ~Ctx();
};

// Public members of Hoshen_Kopelman after Determine_clusters_and_percolation for a mixed
// network (host copies, CSR with int64 offsets), as cicy_mixed_percolation returns them.
struct MixedClusters {
    std::vector<int32_t> family;
    std::vector<int64_t> clu_cnt_ptr, clu_gnp_ptr, iso_cnt_ptr, iso_gnp_ptr, jc_ptr, jg_ptr, jm_ptr, st_ptr, pb_ptr;
    std::vector<int32_t> clu_cnt, clu_gnp, iso_cnt, iso_gnp, jc, jg, jm, pb_face;
    std::vector<int64_t> st_idx, pb_point;
};

// Stage entry points (throw Fail on error).
void upload_network(Ctx& c, const cicy_network& net);
// Network construction on the device (stage_window.cu).
void generate_network_device(Ctx& c, const cicy_gen_params& g);
void extract_window_device(Ctx& c, const cicy_window_params& w);
void run_contact_grid(Ctx& c, const cicy_params& p);
void run_clusters(Ctx& c, const cicy_params& p);
void run_electrical(Ctx& c, const cicy_params& p, cicy_result* out);
// Clusters and percolation of a mixed CNT/GNP network (mixed_percolation.cu).
void run_mixed_percolation(Ctx& c, const cicy_mixed_state& in, MixedClusters& out);
// Electrical_analysis::Perform_analysis_on_clusters for a mixed CNT/GNP network (hybrid_dea.cuh).
void run_hybrid_electrical(Ctx& c, const cicy_hybrid_state& h, const cicy_params& p, double rho_gnp_surf, double rho_gnp_t,
                           cicy_result* out);
struct GnpSet;
struct GnpGrid;
// CNT-GNP contacts of the hybrid grid (gnp_grid.cu); returns the number of contacts.
int run_gnp_cnt_contacts(Ctx& c, const GnpSet& g, const GnpGrid& grid, const cicy_params& p, int inside_is_error);
// Make_mixed_clusters' labels (gnp_labels.cu); returns the number of clusters.
int run_mixed_labels(Ctx& c, const int32_t* labels_gnp, int n_gnps, int n_total_labels, int32_t* labels_cnt_out, int32_t* labels_gnp_out);
// Compress_mixed_contacts on the context's CNT-GNP contacts (gnp_labels.cu):
// junctions (P_cnt, CNT, P_gnp, GNP) x4, distances and the new GNP points.
int run_mixed_junctions(Ctx& c, int n_points_before, int min_points, std::vector<int32_t>& junctions, std::vector<double>& dist,
                        std::vector<double>& points);

// Learned preconditioner: edge weights for the system being solved (learned.cu).
const float* learned_edge_weights(Ctx& c, const SolverSystem& ss, int n_chains, cudaStream_t s);

// Helpers shared across translation units.
int32_t read_i32(Ctx& c, const int32_t* dptr);
void check_status(Ctx& c, const char* where);

}  // namespace cicy
