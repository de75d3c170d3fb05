/*
 * cicy_b200.h — C ABI of the B200 (sm_100a) network-to-conductance hot path of
 * CICY_geom: tunnelling-contact search, Hoshen-Kopelman cluster labelling,
 * junction compression, percolation, DEA resistor-network assembly, Jacobi
 * conjugate-gradient voltage solves, backbone extraction and the effective
 * resistance, exactly as the upstream classes compute them.
 *
 * Plain C: pointers and sizes only, no C++ or CUDA types.  Every function
 * returns a cicy_status (0 = success).  A failing call leaves a message
 * readable through cicy_last_error(ctx); that mirrors the upstream convention
 * of returning 0 and printing "Error in <function> ..." to hout.
 *
 * Upstream interfaces each entry point replaces are cited as file:line of the
 * CICY_geom sources.
 *
 * Threading: a context owns one CUDA device, one CUDA stream and the device
 * buffers of one network.  Calls on one context must not overlap; distinct
 * contexts are independent.  All compute calls are synchronous from the
 * host's point of view: they return once their results are complete.
 *
 * Index widths: point ids are int64 at the boundary (upstream `long int`),
 * CNT ids int32 (upstream `int`).  Inside the device path point ids are
 * 32-bit; networks with 2^31 or more points are rejected with CICY_E_CAPACITY.
 */
#ifndef CICY_B200_H
#define CICY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    CICY_OK = 0,
    CICY_E_INPUT = 1,         /* malformed or inconsistent input */
    CICY_E_CAPACITY = 2,      /* a documented size limit was exceeded */
    CICY_E_DEVICE = 3,        /* a CUDA runtime error */
    CICY_E_TIMEOUT = 4,       /* a bounded device-side wait gave up */
    CICY_E_ZERO_DIAGONAL = 5, /* Direct_Electrifying.cpp:458-484 zero-diagonal check */
    CICY_E_STATE = 6,         /* stages called out of order */
    CICY_E_INTERNAL = 7
} cicy_status;

typedef struct cicy_ctx cicy_ctx;
typedef struct cicy_host_network cicy_host_network;

/* struct cuboid (Geometry_3D.h:133-152). */
typedef struct {
    double min_x, min_y, min_z;
    double len_x, len_y, len_z;
    double max_x, max_y, max_z;
} cicy_cuboid;

/* The fields of Geom_sample, Cutoff_dist, Simu_para and Electric_para
 * (Input_Reader.h:33-297) that the hot path reads. */
typedef struct {
    double gs_min[3];           /* Geom_sample::gs_minx, gs_miny, gs_minz */
    double gs_overlap_cnt;      /* Geom_sample::gs_overlap_cnt (= 2 r_max + d_tunnel, Input_Reader.cpp:1035) */
    double gs_overlap_gnp;      /* Geom_sample::gs_overlap_gnp (only enters region sizing) */
    double van_der_waals_dist;  /* Cutoff_dist::van_der_Waals_dist */
    double tunneling_dist;      /* Cutoff_dist::tunneling_dist */
    int32_t min_points;         /* Cutoff_dist::min_points (junction compression) */
    int32_t simulation_scope;   /* Simu_para::simulation_scope: 0 resistances, 1 backbone only, 2 clusters only */
    int32_t resistances[3];     /* Simu_para::resistances (x, y, z) */
    int32_t junction_type;      /* Electric_para::junction_type: 0 "constant", 1 "exponential" */
    double tolerance;           /* Simu_para::tolerance (CG stop: |r_k| <= tol |r_0|) */
    double applied_voltage;     /* Electric_para::applied_voltage */
    double resistivity_cnt;     /* Electric_para::resistivity_CNT */
    double resistivity_matrix;  /* Electric_para::resistivity_matrix */
    double junction_resistance; /* Electric_para::junction_resistance ("constant") */
    double C1, C2;              /* Electric_para::C1, C2 ("exponential", Input_Reader.cpp:1450-1456) */
    double tolerance_unit;      /* CG tolerance of the unit-resistor (backbone) pass; 0: `tolerance`.
                                   No upstream counterpart: upstream uses one tolerance for both passes,
                                   but the backbone's 1e-9 I_max current threshold (Backbone_Network.cpp:227)
                                   needs the unit pass solved tighter than a loose real-pass tolerance. */
} cicy_params;

/* A window-trimmed CNT network: exactly the inputs that
 * Contact_grid::Generate_contact_grid, Hoshen_Kopelman::Determine_clusters_and_percolation
 * and Electrical_analysis::Perform_analysis_on_clusters read
 * (points_cnt, structure_cnt, radii, Cutoff_Wins::cnts_inside, boundary_cnt, boundary_cnt_pts).
 * Each structure list must be a run of consecutive point ids (upstream assumes
 * this too: Direct_Electrifying.cpp:620-624 walks P1..P2 by id). */
typedef struct {
    int64_t n_points;
    const double* x;               /* points_cnt[i].x */
    const double* y;
    const double* z;
    const int32_t* flag;           /* points_cnt[i].flag: CNT id of the point */
    int32_t n_cnts;
    const int64_t* structure_ptr;  /* n_cnts + 1 offsets into structure_idx */
    const int64_t* structure_idx;  /* point ids of each CNT, in order */
    const double* radii;           /* n_cnts */
    int32_t n_inside;
    const int32_t* cnts_inside;    /* Cutoff_Wins::cnts_inside */
    const int64_t* boundary_cnt_ptr;  /* 7 offsets: faces 0..5 (0 z_max, 1 z_min, 2 x_max, 3 y_max, 4 x_min, 5 y_min) */
    const int32_t* boundary_cnt_idx;  /* Cutoff_Wins::boundary_cnt */
    const int64_t* boundary_pts_ptr;  /* 7 offsets */
    const int64_t* boundary_pts_idx;  /* Cutoff_Wins::boundary_cnt_pts */
    cicy_cuboid window;            /* observation window (Geom_sample::update_observation_window_geometry) */
} cicy_network;

/* Solver choices for the DEA conjugate gradient (no upstream counterpart:
 * upstream always runs FP64 Jacobi-PCG, Direct_Electrifying.cpp:1538-1659). */
typedef enum {
    CICY_PRECISION_FP64 = 0,  /* FP64 everywhere (upstream arithmetic) */
    CICY_PRECISION_MIXED = 1  /* FP32 SpMV and preconditioner apply; FP64 dots, residual replacement, refinement */
} cicy_precision;

typedef enum {
    CICY_PRECOND_JACOBI = 0,  /* M^-1 = 1/diag (Direct_Electrifying.cpp:1662-1668) */
    CICY_PRECOND_LEARNED = 1, /* chain blocks plus a learned sparse approximate inverse T^-1 + T^-1 E_w T^-1 (graph network
                                 weights w on the couplings outside the blocks); Jacobi-PCG when it fails to converge */
    CICY_PRECOND_CHAIN = 2,   /* block-Jacobi over CNT element chains (tridiagonal blocks, explicit inverses) */
    CICY_PRECOND_MG = 3       /* chain-aggregation multigrid V-cycle: chain blocks as the fine smoother, one coarse
                                 unknown per chain block, pairwise aggregation below, dense coarsest inverse */
} cicy_preconditioner;

typedef struct {
    int32_t precision;        /* cicy_precision */
    int32_t preconditioner;   /* cicy_preconditioner */
    int32_t max_iter_factor;  /* max iterations = factor * nodes (upstream 300, Direct_Electrifying.cpp:1559) */
    int32_t flags;            /* bit 0: never use the cluster-resident solver (grid-wide persistent kernel only);
                                 bit 1: multigrid above 20,000 rows keeps its first pairwise prolongator piecewise
                                 constant (no smoothing) */
} cicy_solver_opts;

#define CICY_SOLVER_NO_CLUSTER 1
#define CICY_SOLVER_NO_SMOOTHED 2

/* One DEA linear solve (unit-resistor or real-resistor pass) of one cluster. */
typedef struct {
    int32_t cluster;          /* percolated cluster index */
    int32_t pass;             /* -1 unit-resistor pass, 0/1/2 real pass along x/y/z */
    int64_t nodes;            /* global nodes incl. reserved */
    int64_t reserved;         /* reserved (prescribed-voltage) nodes */
    int64_t nnz_lower;        /* strict-lower non-zeros of the free block */
    int64_t iterations;       /* CG iterations */
    double rel_residual;      /* FP64 |b - A x| / |b| after the solve */
    double seconds;           /* device time of the solve (CUDA events) */
    int32_t kernel;           /* 0: grid-wide persistent PCG, 1: cluster-resident PCG, 2: multigrid PCG */
    int32_t restarts;         /* FP64 true-residual restarts taken */
    int32_t levels;           /* multigrid levels (0 for one-level preconditioners) */
    int32_t fallback;         /* 1: the learned preconditioner did not reach the tolerance; Jacobi-PCG solved it */
} cicy_solve_info;

typedef struct {
    double resistances[3];     /* resistances.txt row (Electrical_analysis.cpp:873-932) */
    double resistivities[3];   /* resistivities.txt row */
    int64_t n_slots;           /* entries of the sectioned domain */
    int64_t n_point_contacts;  /* distinct (Pa, CNTb) contacts */
    int32_t n_labels;          /* clusters before percolation */
    int32_t n_junctions;       /* compressed CNT-CNT junctions */
    int32_t n_percolated;      /* percolated clusters */
    int32_t n_solves;          /* entries used in `solves` */
    cicy_solve_info solves[32];
    double stage_seconds[6];   /* grid, clusters, unit DEA, backbone, real DEA, total (device events) */
} cicy_result;

/* ---------------- context ---------------- */
cicy_status cicy_ctx_create(cicy_ctx** out, int device);
cicy_status cicy_ctx_destroy(cicy_ctx* ctx);
/* Use an external cudaStream_t (passed as void*) instead of the context's own.  The context keeps
   a second stream of its own for work no later stage reads (the backbone and family volumes);
   each call makes the main stream wait for it, so any later work or read on the main stream
   (the getters included) sees it complete. */
cicy_status cicy_ctx_set_stream(cicy_ctx* ctx, void* cuda_stream);
void* cicy_ctx_stream(cicy_ctx* ctx);
cicy_status cicy_ctx_set_solver(cicy_ctx* ctx, const cicy_solver_opts* opts);
/* Polls a grid-barrier wait of this context's persistent solvers makes before it
 * gives up: the kernel then records a device status, every CTA leaves at its next
 * barrier, and the call returns CICY_E_TIMEOUT with the context still usable.
 * polls <= 0 restores the default (2^28, far above any real wait).  Stands in for
 * upstream's only bound on a solve, the CG's iteration cap
 * (Direct_Electrifying.cpp:1559, 1640-1641), for waits upstream does not have. */
cicy_status cicy_ctx_set_spin_limit(cicy_ctx* ctx, int64_t polls);
const char* cicy_last_error(const cicy_ctx* ctx);
/* Number of kernels this context has launched so far. */
int64_t cicy_ctx_kernel_launches(const cicy_ctx* ctx);

/* ---------------- inputs ---------------- */
/* Copy a window-trimmed network from host memory into the context's device buffers. */
cicy_status cicy_upload_network(cicy_ctx* ctx, const cicy_network* net);

/* ---------------- hot path stages ---------------- */
/* Contact_grid::Generate_contact_grid (Contact_grid.cpp:18-80, CNT branch :104-295). */
cicy_status cicy_contact_grid(cicy_ctx* ctx, const cicy_params* p);
/* Hoshen_Kopelman::Determine_clusters_and_percolation, CNT-only path
 * (Hoshen_Kopelman.cpp:17-201, :203-572, :2331-2738). */
cicy_status cicy_clusters(cicy_ctx* ctx, const cicy_params* p);
/* Electrical_analysis::Perform_analysis_on_clusters (Electrical_analysis.cpp:10-145) with
 * Direct_Electrifying::Compute_voltage_field (Direct_Electrifying.cpp:11-113) and
 * Backbone_Network::Determine_backbone_network (Backbone_Network.cpp:11-62). */
cicy_status cicy_electrical_analysis(cicy_ctx* ctx, const cicy_params* p, cicy_result* out);
/* All three stages (App_Network_3D.cpp:140-179 for one window). */
cicy_status cicy_network_to_conductance(cicy_ctx* ctx, const cicy_params* p, cicy_result* out);

/* ---------------- clusters and percolation of a mixed CNT/GNP network ----------------
 * The state Determine_clusters_and_percolation has for GNP_CNT_mix after Make_mixed_clusters
 * (host arrays, copied): mixed labels of CNTs and GNPs (-1: no cluster), the particles
 * inside the window, the face lists of Cutoff_Wins, the particle pairs of every junction
 * kind, and the GNP point lists with their boundary points (point, face) and the
 * junction-point flags of Add_gnp_junction (bp_flags). */
typedef struct {
    int32_t n_labels;
    int32_t n_cnts; const int32_t* labels_cnt;
    int32_t n_cnts_inside; const int32_t* cnts_inside;
    int32_t n_gnps; const int32_t* labels_gnp;
    int32_t n_gnps_inside; const int32_t* gnps_inside;
    const int64_t* boundary_cnt_ptr; const int32_t* boundary_cnt_idx;   /* 6 faces */
    const int64_t* boundary_gnp_ptr; const int32_t* boundary_gnp_idx;   /* 6 faces */
    int64_t n_junctions_cnt; const int32_t* jc_n1; const int32_t* jc_n2;
    int64_t n_junctions_gnp; const int32_t* jg_n1; const int32_t* jg_n2;
    int64_t n_junctions_mixed; const int32_t* jm_n1; const int32_t* jm_n2; /* CNT, GNP */
    int64_t n_points_gnp;
    const int64_t* structure_gnp_ptr; const int64_t* structure_gnp_idx;
    const int64_t* pts_boundary_ptr; const int64_t* pts_boundary_point; const int32_t* pts_boundary_face;
    const int32_t* bp_flags;
} cicy_mixed_state;
typedef struct cicy_mixed_clusters cicy_mixed_clusters;
/* Upstream's public members after Determine_clusters_and_percolation (borrowed, valid until
 * cicy_mixed_clusters_free).  Lists as CSR; junction groups index the junction arrays;
 * structure_gnp and pts_boundary as Remove_gnp_points_in_non_relevant_boundaries leaves them. */
typedef struct {
    int32_t n_percolated;
    const int32_t* family;
    const int64_t* clusters_cnt_ptr; const int32_t* clusters_cnt_idx;
    const int64_t* clusters_gnp_ptr; const int32_t* clusters_gnp_idx;
    int32_t n_isolated_cnt; const int64_t* isolated_cnt_ptr; const int32_t* isolated_cnt_idx;
    int32_t n_isolated_gnp; const int64_t* isolated_gnp_ptr; const int32_t* isolated_gnp_idx;
    const int64_t* cnt_junctions_ptr; const int32_t* cnt_junctions_idx;
    const int64_t* gnp_junctions_ptr; const int32_t* gnp_junctions_idx;
    const int64_t* mix_junctions_ptr; const int32_t* mix_junctions_idx;
    const int64_t* structure_gnp_ptr; const int64_t* structure_gnp_idx;
    const int64_t* pts_boundary_ptr; const int64_t* pts_boundary_point; const int32_t* pts_boundary_face;
} cicy_mixed_clusters_list;
/* Make_particle_clusters for CNTs and GNPs, Find_percolated_clusters with CNT and GNP faces
 * (direction codes 10 d + 1, families by their sum), Group_junctions for the three junction
 * kinds and Remove_gnp_points_in_non_relevant_boundaries (Hoshen_Kopelman.cpp:17-201,
 * 2331-2903), on the device.  A junction whose particles carry different labels is
 * CICY_E_INPUT, as upstream's error. */
cicy_status cicy_mixed_percolation(cicy_ctx* ctx, const cicy_mixed_state* in, cicy_mixed_clusters** out);
cicy_status cicy_mixed_clusters_view(const cicy_mixed_clusters* h, cicy_mixed_clusters_list* view);
void cicy_mixed_clusters_free(cicy_mixed_clusters* h);

/* ---------------- electrical stage of a mixed CNT/GNP network (GNP_CNT_mix) ----------------
 * Upstream's public members after Hoshen_Kopelman::Determine_clusters_and_percolation
 * and Cutoff_Wins for a mixed network (Hoshen_Kopelman.h:27-51, Cutoff_Wins.h), the
 * state Electrical_analysis::Perform_analysis_on_clusters reads.  Host arrays, copied.
 * CSR lists: *_ptr has one offset more than lists.  Junctions: (P1, N1, P2, N2, distance);
 * mixed junctions have the CNT point and CNT first.  The CNT points, radii and face
 * point lists are the context's uploaded network. */
typedef struct {
    int32_t n_clusters;
    const int32_t* family;                                                   /* [n_clusters] */
    const int64_t* clusters_cnt_ptr; const int32_t* clusters_cnt_idx;        /* clusters_cnt */
    const int64_t* clusters_gnp_ptr; const int32_t* clusters_gnp_idx;        /* clusters_gnp */
    const int64_t* cnt_junctions_ptr; const int32_t* cnt_junctions_idx;      /* cluster_cnt_junctions */
    const int64_t* gnp_junctions_ptr; const int32_t* gnp_junctions_idx;      /* cluster_gnp_junctions */
    const int64_t* mix_junctions_ptr; const int32_t* mix_junctions_idx;      /* cluster_mix_junctions */
    int64_t n_junctions_cnt;
    const int64_t* jc_p1; const int32_t* jc_n1; const int64_t* jc_p2; const int32_t* jc_n2; const double* jc_dist;
    int64_t n_junctions_gnp;
    const int64_t* jg_p1; const int32_t* jg_n1; const int64_t* jg_p2; const int32_t* jg_n2; const double* jg_dist;
    int64_t n_junctions_mixed;
    const int64_t* jm_p1; const int32_t* jm_n1; const int64_t* jm_p2; const int32_t* jm_n2; const double* jm_dist;
    const int64_t* elements_ptr; const int64_t* elements_idx;                /* elements_cnt of every CNT (ascending) */
    int32_t n_gnps;
    int64_t n_points_gnp;
    const double* points_gnp;                                                /* xyz per GNP point */
    const int64_t* structure_gnp_ptr; const int64_t* structure_gnp_idx;      /* structure_gnp */
    const int32_t* pts_boundary_count;                                       /* GNP::pts_boundary.size() */
    const double* gnp_t; const double* gnp_volume;                           /* GNP::t, GNP::volume */
    const double* gnp_frame;  /* 16 per GNP: side l, centre[3], rotation[9] (row-major), face-0 normal[3] */
    const int64_t* boundary_gnp_ptr; const int32_t* boundary_gnp_idx;        /* Cutoff_Wins::boundary_gnp (6 faces) */
    const int64_t* boundary_gnp_pts_ptr; const int64_t* boundary_gnp_pts_idx;/* Cutoff_Wins::boundary_gnp_pts (6 faces) */
} cicy_hybrid_state;
/* Electrical_analysis::Perform_analysis_on_clusters for GNP_CNT_mix (Electrical_analysis.cpp:10-145,
 * 229-675) on the device: per percolated cluster the unit-resistor DEA (LM_matrix_for_cnts and
 * LM_matrix_for_gnps, CNT, CNT-CNT, CNT-GNP and GNP-GNP junction resistors and the resistors of
 * each GNP's triangulation, Direct_Electrifying.cpp:11-1394), the backbone of CNTs and GNPs
 * (Backbone_Network.cpp:11-1127) and the real-resistor DEA and parallel resistor per
 * percolated direction with CNT and GNP boundary currents; GNP in-plane / through-plane
 * resistivities as Electric_para::resistivity_GNP_surf / resistivity_GNP_t.  Needs the uploaded
 * CNT network (cicy_upload_network); simulation_scope 0.  A GNP with more points than the
 * triangulation holds (256) gives CICY_E_CAPACITY; upstream's failures give CICY_E_INPUT. */
cicy_status cicy_hybrid_electrical(cicy_ctx* ctx, const cicy_hybrid_state* st, const cicy_params* p, double resistivity_gnp_surf,
                                   double resistivity_gnp_t, cicy_result* out);
/* After cicy_hybrid_electrical: structure_gnp as the backbone left it (CSR over GNPs; size query
 * with NULL buffers), and the volume members volumes_cnt[8], volumes_gnp[8], dead_branches[7],
 * dead_gnps[7] before the fractions step (Backbone_Network.h:26-34). */
cicy_status cicy_get_hybrid_structure(cicy_ctx* ctx, int64_t* n_idx, int64_t* ptr, int64_t* idx);
cicy_status cicy_get_hybrid_volumes(cicy_ctx* ctx, double* volumes30);
/* The GNP and mixed junction lists of a percolated cluster after its backbone (cluster_gnp_junctions,
 * cluster_mix_junctions); sizes in n_gnp / n_mix (NULL buffers: size query). */
cicy_status cicy_get_hybrid_junctions(cicy_ctx* ctx, int32_t cluster, int64_t* n_gnp, int32_t* gnp, int64_t* n_mix, int32_t* mix);

/* ---------------- copy-out (size query: pass NULL buffers, read the counts) ----------------
 * These fill the public members the upstream classes expose to later stages. */
/* The context's network (after an upload, cicy_ctx_generate_cnt_network or
 * cicy_ctx_extract_window): points (x, y, z, flag; n_points), each CNT's run
 * (cnt_start, cnt_len; n_cnts), radii, cnts_inside (n_inside), the six faces'
 * boundary CNT and point lists (Cutoff_Wins::boundary_cnt / boundary_flags_cnt as
 * CSR: 7 offsets each, n_bcnt / n_bpts entries) and the window cuboid.  Any buffer
 * may be NULL. */
cicy_status cicy_get_network(cicy_ctx* ctx, int64_t* n_points, int32_t* n_cnts, int32_t* n_inside, int64_t* n_bcnt, int64_t* n_bpts,
                             double* x, double* y, double* z, int32_t* flag, int32_t* cnt_start, int32_t* cnt_len, double* radii,
                             int32_t* cnts_inside, int64_t* bcnt_ptr, int32_t* bcnt_idx, int64_t* bpts_ptr, int32_t* bpts_idx,
                             cicy_cuboid* window);
/* Contact_grid::sectioned_domain_cnts as CSR (n_regions + 1 offsets). */
cicy_status cicy_get_sectioned_domain(cicy_ctx* ctx, int64_t* n_regions, int64_t* n_slots, int64_t* ptr, int64_t* idx);
/* The point_contacts / point_contacts_dist maps of Hoshen_Kopelman::Label_cnts_in_window
 * (Hoshen_Kopelman.cpp:249-372), sorted by (Pa, CNTb). */
cicy_status cicy_get_point_contacts(cicy_ctx* ctx, int64_t* n, int64_t* pa, int32_t* cnt_b, int64_t* pb, double* dist);
/* labels_cnt after Cleanup_labels (Hoshen_Kopelman.cpp:374-425); n = number of CNTs. */
cicy_status cicy_get_labels(cicy_ctx* ctx, int32_t* n_cnts, int32_t* n_labels, int32_t* labels);
/* Hoshen_Kopelman::junctions_cnt (Hoshen_Kopelman.cpp:443-554). */
cicy_status cicy_get_junctions(cicy_ctx* ctx, int64_t* n, int64_t* p1, int32_t* n1, int64_t* p2, int32_t* n2, double* dist);
/* Hoshen_Kopelman::elements_cnt as CSR over all CNTs; which = 0 after labelling,
 * which = 1 the backbone-trimmed elements (Backbone_Network.cpp:412-556). */
cicy_status cicy_get_elements(cicy_ctx* ctx, int32_t which, int64_t* n_cnts, int64_t* n_idx, int64_t* ptr, int64_t* idx);
/* clusters_cnt (percolated clusters, CSR), family, cluster_cnt_junctions (CSR);
 * which = 0 after percolation, 1 after backbone extraction. */
cicy_status cicy_get_clusters(cicy_ctx* ctx, int32_t which, int32_t* n_clusters, int64_t* n_idx, int64_t* ptr, int32_t* idx,
                              int32_t* family, int64_t* n_junc_idx, int64_t* junc_ptr, int32_t* junc_idx);
/* Backbone_Network's volume members after Perform_analysis_on_clusters
 * (Backbone_Network.h:26-34, filled by Calculate_cnt_volumes, Backbone_Network.cpp:412-574,
 * and Calculate_percolated_families_fractions, Electrical_analysis.cpp:678-786):
 * volumes_cnt[8] (backbone volume per family 0-6; [7] dead branches plus isolated and
 * non-percolated CNTs), dead_branches[7] (per family), and the fractions step's
 * total_volumes[8] and fractions[8] (volumes.txt, fractions.txt).  CNT networks: the GNP
 * members are 0.  Any pointer may be NULL.  After cicy_electrical_analysis. */
cicy_status cicy_get_volumes(cicy_ctx* ctx, double* volumes_cnt, double* dead_branches, double* total_volumes, double* fractions);
/* One DEA system and its solution, as upstream builds it in SSS form
 * (strict-lower CSR of the free block, diagonal, right-hand side after the BC
 * elimination, initial guess, prescribed voltages, voltages of all nodes).
 * solve = index into cicy_result::solves. */
cicy_status cicy_get_system(cicy_ctx* ctx, int32_t solve, int64_t* nodes, int64_t* reserved, int64_t* nnz_lower,
                            int64_t* row_ptr, int64_t* col_ind, double* values, double* diag, double* b, double* x0,
                            double* voltages);

/* Chains (consecutive free nodes of one CNT) of a solve's system: start node and
 * length of each, in the order of the system's CNTs. */
cicy_status cicy_get_chains(cicy_ctx* ctx, int32_t solve, int32_t* n_chains, int32_t* start, int32_t* len);

/* ---------------- learned preconditioner (no upstream counterpart) ----------------
 * A graph network (3 message-passing layers, width 32, BF16 weights and
 * activations, FP32 accumulation) that weights the couplings left out by the
 * chain block-Jacobi T, giving M^-1 = T^-1 + T^-1 E_w T^-1.  Parameters are one
 * flat FP32 vector of cicy_gnn_param_count() entries.  The training entry points
 * take device pointers and a cudaStream_t (as void*); systems are full symmetric
 * CSR with ascending columns, diagonal included. */
int32_t cicy_gnn_param_count(void);
/* Parameters the solver uses for CICY_PRECOND_LEARNED (host array, copied). */
cicy_status cicy_ctx_set_learned_params(cicy_ctx* ctx, const float* params, int32_t n);

typedef struct cicy_gnn cicy_gnn;
typedef struct {
    int32_t n, nnz;
    const int32_t* row_ptr;   /* device, n + 1 */
    const int32_t* col_ind;   /* device, nnz */
    const double* values;     /* device, nnz */
    int32_t n_chains;
    const int32_t* chain_start; /* device */
    const int32_t* chain_len;   /* device */
} cicy_gnn_system;
cicy_status cicy_gnn_create(cicy_gnn** out, int device);
cicy_status cicy_gnn_destroy(cicy_gnn* g);
/* Features and chain blocks of one system (kept until the next call).  The CSR
 * structure and the chains are checked on the device first (CICY_E_INPUT when
 * row_ptr is not 0 .. nnz non-decreasing, a column index is outside [0, n), or
 * the chains are not consecutive runs covering the rows). */
cicy_status cicy_gnn_set_system(cicy_gnn* g, const cicy_gnn_system* sys, void* stream);
/* Forward pass: weight of every matrix entry (0 on the blocks and the diagonal) into w[nnz] (device). */
cicy_status cicy_gnn_forward(cicy_gnn* g, const float* params, float* w, void* stream);
/* Mean loss 1 - (r.Az)^2/(|r|^2 |Az|^2), r = A u, z = M^-1 r, over n_probes probe
 * vectors u (device, n_probes x n, FP64), and its gradient grad[param_count] (device, overwritten). */
cicy_status cicy_gnn_loss_grad(cicy_gnn* g, const float* params, int32_t n_probes, const double* probes, double* loss, float* grad,
                               void* stream);
/* u <- u - 0.9 T^-1 A u, `sweeps` times, on each probe vector (leaves the modes the blocks handle worst). */
cicy_status cicy_gnn_smooth_probes(cicy_gnn* g, int32_t n_probes, double* probes, int32_t sweeps, void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on device arrays of n floats; step counts from 1. */
cicy_status cicy_gnn_adam(float* params, const float* grad, float* m, float* v, int32_t n, int32_t step, float lr, void* stream);

/* FP64 CSR sparse matrix-vector product y = A x on device arrays: the CG's SpMV
 * (spM_V_SSS, Direct_Electrifying.cpp:1680-1735, which uses the symmetric
 * SSS storage; here full CSR).  Enqueued on `stream` (a cudaStream_t, or NULL);
 * returns without waiting. */
cicy_status cicy_spmv_csr(int32_t n, const int32_t* row_ptr, const int32_t* col_ind, const double* values, const double* x, double* y,
                          void* stream);

/* ---------------- batched Monte-Carlo solves (no upstream counterpart) ----------------
 * Many independent DEA systems (e.g. the real-resistor systems of hundreds of
 * seeded realisations) solved together.  Methods 0 and 1 stop at
 * |r| <= tol min(|r0|, |b|) confirmed on the FP64 true residual (the test of
 * Direct_Electrifying.cpp:1571, 1619, and |b - A x| <= tol |b|); method 2 is
 * the per-network solver and uses the upstream test |r| <= tol |r0|.
 * Methods:
 *   0  one persistent kernel launch replayed from a CUDA graph; each CTA takes
 *      the next system of a largest-first queue and runs preconditioned CG on
 *      it alone, with the preconditioner and precision of cicy_batch_set_solver
 *      (the largest systems optionally on 16-CTA clusters, cicy_batch_set_split);
 *   1  one 16-CTA cluster per system running the chain-aggregation multigrid
 *      PCG (after cicy_batch_enable_multigrid; FP64);
 *   2  one system after another through the per-network grid-wide persistent
 *      PCG (the path cicy_electrical_analysis uses), same preconditioner and
 *      precision as method 0; seconds = the sum of its kernels' device times.
 * All pointers are device memory the caller keeps alive, of the stated sizes;
 * the chains must be consecutive runs of rows covering 0 .. n-1.
 * cicy_batch_create checks the CSR structure and the chains on the device
 * and returns CICY_E_INPUT naming the first bad system. */
typedef struct {
    int32_t n, nnz;
    const int32_t* row_ptr;    /* full symmetric CSR, diagonal included, ascending columns */
    const int32_t* col_ind;
    const double* values;
    const double* b;
    const double* x0;          /* initial guess */
    double* x;                 /* solution (written by every solve) */
    int32_t n_chains;
    const int32_t* chain_start;
    const int32_t* chain_len;
    const float* edge_weights; /* CICY_PRECOND_LEARNED: weight of every CSR entry, 0 on the chain blocks
                                  and the diagonal (cicy_gnn_forward's output); NULL otherwise */
} cicy_batch_system;
typedef struct cicy_batch cicy_batch;
cicy_status cicy_batch_create(cicy_batch** out, int device, const cicy_batch_system* systems, int32_t count, double tol,
                              int32_t max_iter_factor, int32_t precision);
cicy_status cicy_batch_destroy(cicy_batch* b);
/* Launch shape of method 0: threads per CTA (256, 512, 1024) and CTAs per SM. */
cicy_status cicy_batch_set_shape(cicy_batch* b, int32_t threads, int32_t ctas_per_sm);
/* Preconditioner of methods 0 and 2: CICY_PRECOND_JACOBI (plain Jacobi-PCG, the
 * upstream algorithm), CICY_PRECOND_CHAIN (whole-chain block-Jacobi; method 2
 * splits chains into blocks of at most 32 nodes), CICY_PRECOND_LEARNED (chain
 * blocks of at most 32 nodes plus the learned sparse approximate inverse,
 * needs every system's edge_weights).  Precision: CICY_PRECISION_FP64, or
 * CICY_PRECISION_MIXED (FP32 conductances in a difference-form SpMV and FP32
 * preconditioner factors; FP64 vectors, dots and residual replacement).
 * Default: CICY_PRECOND_CHAIN and the precision given to create. */
cicy_status cicy_batch_set_solver(cicy_batch* b, int32_t preconditioner, int32_t precision);
/* Method 0: systems of at least `rows` rows each run on one 16-CTA cluster
 * (chain-aligned row ranges per CTA, hardware cluster barriers), concurrently
 * with the one-CTA solves of the rest, in the same graph launch; 0 (the
 * default): every system on one CTA. */
cicy_status cicy_batch_set_split(cicy_batch* b, int32_t rows);
/* Builds a multigrid hierarchy per system (setup time returned) so the batch can
 * also run method 1. */
cicy_status cicy_batch_enable_multigrid(cicy_batch* b, double* setup_seconds);
/* 0, 1 or 2 (above). */
cicy_status cicy_batch_set_method(cicy_batch* b, int32_t method);
/* Times method 0's launch shapes (with the current preconditioner and
 * precision) and, when multigrid is enabled, method 1, on this batch, then for
 * method 0 the cluster split at 131072, 32768 and 8192 rows, and keeps the
 * fastest (for method 1 ctas_per_sm returns the number of concurrent clusters;
 * split_rows is 0 when no system runs on a cluster). */
cicy_status cicy_batch_autotune(cicy_batch* b, int32_t* method, int32_t* threads, int32_t* ctas_per_sm, int32_t* split_rows,
                                double* seconds);
/* One solve of every system by the current method; seconds = its device time (CUDA events). */
cicy_status cicy_batch_solve(cicy_batch* b, double* seconds);
/* Per system: iterations, FP64 |b - A x| / |b|, flag (1 converged, 2 iteration cap, 0 breakdown or restart limit). */
cicy_status cicy_batch_results(cicy_batch* b, int64_t* iterations, double* rel_residual, int32_t* flags);

/* ---------------- host-side network sources (CPU, upstream of the hot path) ---------------- */
/* Seeded synthetic CNT network (no upstream counterpart; emits the same layout
 * Read_Network::Read_cnt_data_from_dat builds, Read_Network.cpp:348-467):
 * start U(sample), isotropic initial direction, polyline of `step` steps with
 * polar turn U[0, max_turn] at uniform azimuth, length U[len_min, len_max],
 * 1 + floor(L/step) points. Counter-based (Philox-4x32-10) so each CNT is
 * reproducible by index. */
typedef struct {
    cicy_cuboid sample;
    int32_t n_cnts;
    int32_t n_threads;   /* host threads (0: all) */
    uint64_t seed;
    double step;
    double len_min, len_max;
    double radius;
    double max_turn_rad;
} cicy_gen_params;
cicy_status cicy_generate_cnt_network(const cicy_gen_params* g, cicy_host_network** out);

/* Window extraction for window 0 of a single-window run: Shells::Generate_shells
 * (Shells.cpp:21-69) + Cutoff_Wins::Trim_boundary_cnts / Add_cnt_segment_to_structure /
 * Substitute_boundary_point / Add_cnt_point_to_boundary_vectors / Fill_cnts_inside
 * (Cutoff_Wins.cpp:82-831), CNT_wires branch. */
typedef struct {
    cicy_cuboid sample;     /* Geom_sample::sample */
    double win_max[3];      /* Geom_sample::win_max_x/y/z */
    double win_min[3];      /* Geom_sample::win_min_x/y/z */
    double win_delt[3];     /* Geom_sample::win_delt_x/y/z */
    double step_length;     /* Nanotube_Geo::step_length */
    int32_t min_points;     /* Nanotube_Geo::min_points */
    int32_t reserved0;
} cicy_window_params;
cicy_status cicy_extract_window(const cicy_host_network* in, const cicy_window_params* w, cicy_host_network** out);
/* The seeded synthetic network of cicy_generate_cnt_network generated on the device
 * into the context (replaces its network; only the per-CNT point counts and runs
 * travel to the host, for the context's bookkeeping).  Same Philox streams: point counts, structure,
 * flags and start points equal the host generator's; later points follow from the
 * device's sin/cos, so coordinates agree with the host generator's to rounding
 * (checked within 1e-10 um), not bit for bit.  The result is the untrimmed network (window =
 * sample, no CNTs inside yet): call cicy_ctx_extract_window before the stages. */
cicy_status cicy_ctx_generate_cnt_network(cicy_ctx* ctx, const cicy_gen_params* g);
/* Window 0 of a single-window run trimmed on the device, in place on the context's
 * network: Shells::Generate_shells / Find_shell (Shells.cpp:21-149) and
 * Cutoff_Wins::Trim_boundary_cnts (Cutoff_Wins.cpp:82-276),
 * Add_cnt_segment_to_structure (:298-467), Substitute_boundary_point (:468-548),
 * Where_is_with_boundary (:683-743), Add_cnt_point_to_boundary_vectors (:745-769)
 * and Fill_cnts_inside (:803-831), CNT_wires branch; equal bit for bit to
 * cicy_extract_window on the same network.  The network must be in the layout the
 * generator and Read_Network emit (CNT i is the i-th run of consecutive points and
 * its points carry flag i), as after cicy_ctx_generate_cnt_network or the upload of
 * an untrimmed network; else CICY_E_INPUT.  Limits: at most 16 segments per CNT
 * (CICY_E_CAPACITY), min_points >= 2.  Upstream's errors (a cut point off the
 * window, a CNT left with one point) return CICY_E_INPUT with its message. */
cicy_status cicy_ctx_extract_window(cicy_ctx* ctx, const cicy_window_params* w);

/* Read_Network::Generate_nanoparticle_network_from_file, CNT branch
 * (Read_sample_geometry + Read_cnt_data_from_dat / Read_cnt_data_from_csv,
 * Read_Network.cpp:154-467): sample_geom.csv and cnt_struct / cnt_coordinates
 * (.dat when file_type = 0, .csv when 1) of `directory`, read whole and parsed
 * in memory, into the layout the generator emits (window = the sample).  The
 * upstream error cases return CICY_E_INPUT with the upstream message
 * (cicy_host_last_error); so does a CSV line that does not hold its numbers
 * (upstream would read it as zeros and shift the points after it).  CSV
 * coordinates are parsed on host threads.  GNP files are not read. */
cicy_status cicy_read_network(const char* directory, int32_t file_type, cicy_host_network** out);
/* GNPs (graphene nanoplatelets) of a directory's gnp_data.dat as
 * Read_Network::Read_gnp_data_from_dat builds them (Read_Network.cpp:576-679):
 * rotation matrix from the stored (theta, phi) of the normal
 * (Generate_Network::Get_transformation_matrix), the 8 vertices
 * (Obtain_gnp_vertex_coordinates) and the 6 face planes
 * (Update_gnp_plane_equations), in upstream's operation order on the host, so
 * the doubles equal upstream's.  Input of the GNP contact search (the hybrid
 * CNT/GNP configuration). */
typedef struct cicy_gnp_set cicy_gnp_set;
typedef struct {
    int32_t n;
    const double* l;         /* side [n] */
    const double* t;         /* thickness [n] */
    const double* center;    /* [3n] */
    const double* rotation;  /* row-major 3x3 per GNP [9n] */
    const double* vertices;  /* 8 vertices x (x, y, z) per GNP [24n] */
    const double* planes;    /* 6 faces x (nx, ny, nz, d) per GNP [24n], n.p + d = 0 on the face */
} cicy_gnps;
cicy_status cicy_read_gnps(const char* directory, cicy_gnp_set** out);
/* Borrowed view; valid until cicy_gnp_set_free. */
cicy_status cicy_gnp_set_view(const cicy_gnp_set* set, cicy_gnps* view);
void cicy_gnp_set_free(cicy_gnp_set* set);

/* GNP part of the window extraction (window 0, single-window runs), on the
 * host: Shells::Add_to_gnp_shells and Cutoff_Wins::Fill_gnps_inside with
 * Find_gnp_boundary_points (Shells.cpp:150-178, Cutoff_Wins.cpp:833-1318).
 * GNPs deeper than the boundary shell are inside; a GNP in it with a vertex
 * inside the window is inside too and gets, per window face it crosses, one
 * boundary point: the average of its vertices on the face, its edges' cuts
 * through the face, the window edges through it and a window corner inside it
 * (upstream's points_gnp / structure_gnp / boundary_gnp / boundary_gnp_pts
 * before the contact search; n_points is gnp_pts_bdds), and those GNPs'
 * volume inside the window. */
typedef struct cicy_gnp_window cicy_gnp_window;
typedef struct {
    int32_t n_inside;
    const int32_t* gnps_inside;        /* [n_inside] */
    const int32_t* boundary_gnp_ptr;   /* [7]: GNPs at face f are boundary_gnp_idx[ptr[f]..ptr[f+1]) */
    const int32_t* boundary_gnp_idx;
    int64_t n_points;
    const double* points;              /* [3 n_points] boundary points */
    const int32_t* point_gnp;          /* [n_points] */
    const int32_t* point_boundary;     /* [n_points] face of the point */
    const int32_t* boundary_pts_ptr;   /* [7] */
    const int32_t* boundary_pts_idx;
    int32_t n_gnps;
    const int32_t* structure_ptr;      /* [n_gnps + 1] each GNP's boundary points */
    const int32_t* structure_idx;
    const double* volume;              /* [n_gnps] volume inside the window (Approximate_gnp_volume_inside_sample)
                                          of the GNPs crossing a face, NaN for the others */
} cicy_gnp_window_list;
cicy_status cicy_gnp_extract_window(const cicy_gnp_set* gnps, const cicy_window_params* w, cicy_gnp_window** out);
/* Borrowed view; valid until cicy_gnp_window_free. */
cicy_status cicy_gnp_window_view(const cicy_gnp_window* h, cicy_gnp_window_list* view);
void cicy_gnp_window_free(cicy_gnp_window* h);

/* GNP part of the contact grid on the device: Contact_grid::Fill_sectioned_domain_gnps
 * (Contact_grid.cpp:297-512) on the region grid of Generate_contact_grid +
 * Adjust_regions_if_needed (:18-102).  The GNPs of `inside` (indices into the
 * set, in order) are sampled on upstream's grid of their volume; each sample
 * point strictly inside `window` adds its GNP to its region and the overlap
 * neighbours.  Region t = a + b sx + c sx sy lists each GNP once, in `inside`
 * order (the upstream sectioned_domain_gnps), as CSR of GNP indices.  FP64
 * without contraction, so the lists equal upstream's.  Limits: regions x
 * GNPs < 2^32, at most 2^29 sample points (CICY_E_CAPACITY). */
typedef struct cicy_gnp_grid cicy_gnp_grid;
cicy_status cicy_gnp_sectioned_domain(int device, const cicy_gnp_set* gnps, const int32_t* inside, int32_t n_inside,
                                      const cicy_cuboid* window, const double* gs_min, double overlap_cnt, double overlap_gnp,
                                      cicy_gnp_grid** out);
/* Region counts, sizes and the CSR (ptr[sx sy sz + 1], idx[n_entries]); valid until cicy_gnp_grid_free. */
cicy_status cicy_gnp_grid_view(const cicy_gnp_grid* g, int32_t* n_regions, double* l_regions, const int32_t** ptr, const int32_t** idx,
                               int64_t* n_entries);
void cicy_gnp_grid_free(cicy_gnp_grid* g);

/* Closest GNP point to each query point on the device, the CNT-GNP distance of
 * the mixed contact search (Generate_Network::Get_gnp_point_closest_to_point,
 * Generate_Network.cpp:5577-5856, called by Hoshen_Kopelman::Find_adjacent_labels):
 * host arrays xyz[3n] and GNP indices gnp[n] in, distance dist[n], closest
 * point closest[3n] and flag[n] (0, or -1 with distance 0 and the origin when
 * the point is inside the GNP) out.  Upstream's decision tree and arithmetic
 * order without contraction, so the results equal upstream's. */
cicy_status cicy_gnp_point_distance(int device, const cicy_gnp_set* gnps, int32_t n, const double* xyz, const int32_t* gnp, double* dist,
                                    double* closest, int32_t* flag);

/* GNP-GNP distance on the device, Hoshen_Kopelman::Get_distance_between_GNPs
 * (Hoshen_Kopelman.cpp:770-823): GJK distance (Collision_detection::GJK_distance,
 * Collision_detection.cpp:751-1703) and, for interpenetrating GNPs, the EPA
 * penetration depth and direction (:1704-1946), upstream's steps and FP64
 * operation order, so the doubles equal upstream's.  Pair i is GNPs a[i], b[i]:
 * dist[i] (the van der Waals distance when they interpenetrate), the direction
 * direction[3i..] (GJK's last search direction, or EPA's face normal), the move
 * of b displacement[3i..] (direction x (depth + vdw); 0 when separate) and
 * penetrating[i].  A pair upstream fails on (GJK beyond 50 iterations) returns
 * CICY_E_INPUT naming it; an EPA polytope beyond 72 vertices / 160 faces,
 * CICY_E_CAPACITY. */
cicy_status cicy_gnp_pair_distance(int device, const cicy_gnp_set* gnps, int32_t n, const int32_t* a, const int32_t* b, double vdw, double* dist,
                                   double* direction, double* displacement, int32_t* penetrating);

/* Junction points of GNP pairs on the device: the distance step above, then
 * Hoshen_Kopelman::Find_junction_points_for_gnps (Hoshen_Kopelman.cpp:826-1825)
 * on GNP a and GNP b moved apart when they interpenetrate (Move_gnp), the point
 * on b moved back, as Label_gnps_in_window does (:712-746).  Per pair: the
 * points point_a[3i..], point_b[3i..], outside[i] (1: point_a outside `sample`,
 * 2: point_b, Point_3D::is_outside_cuboid; -1 when the step failed) and
 * status[i] (0, or the step upstream fails in: 1 simplex size, 2 intersection
 * outside [0, 1], 3 no vertex inside the other face, 4 no edge for the
 * two-intersection average, 5 no face for the vertex sum).  allow_simplex3 is
 * Simu_para::allow_simplex3 (false for App_Network_3D). */
cicy_status cicy_gnp_junction_points(int device, const cicy_gnp_set* gnps, int32_t n, const int32_t* a, const int32_t* b, double vdw,
                                     const cicy_cuboid* sample, int32_t allow_simplex3, double* point_a, double* point_b, int32_t* outside,
                                     int32_t* status);

/* GNP-GNP contact pass of Hoshen_Kopelman::Label_gnps_in_window
 * (Hoshen_Kopelman.cpp:626-767) on the device: every pair of GNPs sharing a
 * region of `grid` (cicy_gnp_sectioned_domain), measured once; the pairs within
 * the tunnelling cutoff (dist <= tunnel) in upstream's visiting order (regions,
 * then j < k within the region, first visit), each as (a < b) with the results
 * of cicy_gnp_pair_distance and the junction points of
 * cicy_gnp_junction_points.  Upstream links a pair (HK76) when neither point
 * is outside the sample; a junction step that fails returns CICY_E_INPUT naming
 * the pair, where upstream stops.  Upstream orders a pair as (min(GNP1, GNP2),
 * GNP2); with region lists in ascending GNP order (an ascending `inside`) that
 * is (a < b) too. */
typedef struct cicy_gnp_pairs cicy_gnp_pairs;
typedef struct {
    int64_t n;                    /* contact pairs */
    int64_t n_visits;             /* region pair visits */
    int64_t n_pairs;              /* distinct pairs measured */
    const int32_t* a;             /* [n] */
    const int32_t* b;             /* [n] */
    const int32_t* penetrating;   /* [n] */
    const double* dist;           /* [n] */
    const double* direction;      /* [3n] */
    const double* displacement;   /* [3n] */
    const double* point_a;        /* [3n] junction point on a */
    const double* point_b;        /* [3n] junction point on b */
    const int32_t* outside;       /* [n] 1: point_a outside the sample, 2: point_b, 3: both */
} cicy_gnp_pair_list;
cicy_status cicy_gnp_contact_pairs(int device, const cicy_gnp_set* gnps, const cicy_gnp_grid* grid, double vdw, double tunnel,
                                   const cicy_cuboid* sample, int32_t allow_simplex3, cicy_gnp_pairs** out);
/* Borrowed view; valid until cicy_gnp_pairs_free. */
cicy_status cicy_gnp_pairs_view(const cicy_gnp_pairs* p, cicy_gnp_pair_list* view);
void cicy_gnp_pairs_free(cicy_gnp_pairs* p);

/* GNP labels on the device: the HK76 pass of Label_gnps_in_window over the
 * contact pairs whose junction points are both inside the sample (outside ==
 * 0), in list order, then Cleanup_labels and Renumber_gnp_labels
 * (Hoshen_Kopelman.cpp:594-616): labels_gnp[n_gnps] (-1: no cluster) numbered
 * from n_labels_cnt, and n_total_labels = n_labels_cnt + the GNP clusters. */
cicy_status cicy_gnp_labels(int device, const cicy_gnp_pairs* pairs, int32_t n_gnps, int32_t n_labels_cnt, int32_t* labels_gnp,
                            int32_t* n_total_labels);

/* Labels of mixed CNT/GNP clusters on the device, Make_mixed_clusters
 * (Hoshen_Kopelman.cpp:1925-1987): the context's CNT labels (cicy_clusters on
 * the hybrid grid) and GNP labels `labels_gnp` (cicy_gnp_labels, n_total_labels
 * labels in all) joined by the context's CNT-GNP contacts
 * (cicy_gnp_cnt_contacts) in contact-number order (HK76), then Cleanup_labels:
 * labels_cnt[n_cnts] and labels_gnp_out[n_gnps] (either may be NULL),
 * n_clusters.  The context's CNT labels become the mixed ones. */
cicy_status cicy_mixed_labels(cicy_ctx* ctx, const int32_t* labels_gnp, int32_t n_gnps, int32_t n_total_labels, int32_t* labels_cnt,
                              int32_t* labels_gnp_out, int32_t* n_clusters);

/* GNP point structures on the device, Add_gnp_junction and
 * Add_gnp_point_to_vectors_if_not_repeated (Hoshen_Kopelman.cpp:1837-1923)
 * over the contact pairs whose junction points are both inside the sample, in
 * list order: the point on a, then on b, joins its GNP's point list; a point of
 * an interpenetrating pair reuses the first point of that list within squared
 * distance tol_gnp2 (Cutoff_dist::tol_gnp2), else it is appended with the next
 * global number.  Initial points (upstream's points_gnp before the pass, e.g.
 * window boundary points; gnp_pts_bdds = n_init_points) and per-GNP lists
 * (CSR; NULL for none) may be given. */
typedef struct cicy_gnp_points cicy_gnp_points;
typedef struct {
    int64_t n_points;
    const double* points;          /* [3 n_points]: initial points, then the junction points */
    int32_t n_gnps;
    const int32_t* structure_ptr;  /* [n_gnps + 1] structure_gnp as CSR */
    const int32_t* structure_idx;
    int64_t n_junctions;
    const int32_t* junctions;      /* [4 n_junctions]: Pa, GNPa, Pb, GNPb (junctions_gnp) */
    const double* junction_dist;   /* [n_junctions] */
    int32_t n_boundary;            /* gnp_pts_bdds */
    const int32_t* boundary_used;  /* [n_boundary] bp_flags */
} cicy_gnp_point_list;
cicy_status cicy_gnp_junction_structures(int device, const cicy_gnp_pairs* pairs, int32_t n_gnps, double tol_gnp2, int32_t n_init_points,
                                         const double* init_points, const int32_t* init_ptr, const int32_t* init_idx, cicy_gnp_points** out);
/* Borrowed view; valid until cicy_gnp_points_free. */
cicy_status cicy_gnp_points_view(const cicy_gnp_points* p, cicy_gnp_point_list* view);
void cicy_gnp_points_free(cicy_gnp_points* p);

/* Compress_mixed_contacts / Add_mixed_junction (Hoshen_Kopelman.cpp:2181-2306)
 * on the device, over the context's CNT-GNP contacts (cicy_gnp_cnt_contacts):
 * GNPs ascending, the CNTs in contact with each ascending, their contact
 * points ascending, cut into runs at min_points past a run's first point, each
 * run kept at its first point of least junction distance.  Junction j joins CNT
 * point cnt_point[j] of CNT cnt[j] to the new GNP point gnp_point[j] =
 * n_points_gnp + j of GNP gnp[j] (its closest point points[3j..]); upstream
 * appends these points to points_gnp and structure_gnp[gnp[j]] in this order
 * and adds cnt_point[j] to elements_cnt[cnt[j]].  Results via
 * cicy_get_mixed_junctions (size query: NULL buffers). */
cicy_status cicy_mixed_junctions(cicy_ctx* ctx, int64_t n_points_gnp, int32_t min_points, int64_t* n_junctions);
cicy_status cicy_get_mixed_junctions(cicy_ctx* ctx, int64_t* n, int64_t* cnt_point, int32_t* cnt, int64_t* gnp_point, int32_t* gnp, double* dist,
                                     double* points);

/* CNT-GNP contacts of the hybrid CNT/GNP sample on the device:
 * Hoshen_Kopelman::Find_adjacent_labels (Hoshen_Kopelman.cpp:1989-2142) over
 * Contact_grid::Generate_contact_grid with particle type GNP_CNT_mix.  The
 * context holds the CNT network and its contact grid (cicy_upload_network,
 * cicy_contact_grid with the hybrid overlaps); `grid` is the GNP part of the
 * same grid (cicy_gnp_sectioned_domain with the same window, region sizes and
 * overlaps; other regions: CICY_E_INPUT).  A (point, GNP) pair of a region is a
 * contact when max(closest distance - CNT radius, van der Waals) is within the
 * tunnelling cutoff (+1e-10); contacts are numbered in upstream's visiting
 * order (regions, the region's GNPs, the region's points).  A point inside a
 * GNP is no contact (upstream's ignore_eror_cnt_inside_gnp = 1), or, with
 * inside_is_error = 1, fails with CICY_E_INPUT as upstream's default does.
 * At most 2^31 point-GNP visits (CICY_E_CAPACITY). */
cicy_status cicy_gnp_cnt_contacts(cicy_ctx* ctx, const cicy_gnp_set* gnps, const cicy_gnp_grid* grid, const cicy_params* p,
                                  int32_t inside_is_error, int64_t* n_contacts);
/* The contacts by contact-point number i: CNT point point[i], GNP gnp[i], junction
 * distance dist[i] (point_contacts / point_contacts_dist) and the closest GNP point
 * closest[3i..3i+2] (contact_points_gnp).  Size query: NULL buffers. */
cicy_status cicy_get_gnp_cnt_contacts(cicy_ctx* ctx, int64_t* n, int64_t* point, int32_t* gnp, double* dist, double* closest);

/* Wrap caller-owned arrays (copied) as a host network, e.g. a network read from files. */
cicy_status cicy_host_network_from_arrays(const cicy_network* net, cicy_host_network** out);
/* Borrowed view of a host network; valid until cicy_host_network_free. */
cicy_status cicy_host_network_view(const cicy_host_network* h, cicy_network* view);
void cicy_host_network_free(cicy_host_network* h);
/* Message of the last failing host-side call on this thread. */
const char* cicy_host_last_error(void);

/* ---------------- allocation-free solve ----------------
 * No counterpart in the reference.  FP64 Jacobi-PCG (the algorithm of
 * Solve_DEA_equations_CG_SSS) on a system the caller already holds in device
 * memory as full symmetric CSR (row_ptr[n+1], col_ind/values[nnz], diagonal
 * included), right-hand side b[n] and solution x[n] (in: initial guess, out:
 * solution), that allocates no device memory: for callers that may not let
 * cudaMalloc/cudaFree synchronize the device or take the allocator's lock
 * mid-loop, or whose host owns all device memory.  All scratch lives in one
 * fixed static device array of about 5.3 MB that every GPU loading the library
 * holds until exit; systems above 131072 rows are rejected with
 * CICY_E_CAPACITY.  Runs on the current device and `stream` (a cudaStream_t, or
 * NULL); returns once the solve is complete.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) and keeps it for the
 * life of the process, so make that first call before any stream capture; after
 * a cudaDeviceReset the kept address is stale (do not call it again on that
 * device).  Every call shares the one array and the call resets the words that
 * must start at zero, so calls that overlap on the GPU (other streams, other
 * host threads) race: serialize them.  The CSR is checked on the device first
 * (row_ptr 0 .. nnz non-decreasing, columns in [0, n)); a malformed system
 * returns CICY_E_INPUT before any kernel uses its indices.  Stops when
 * |r| <= tol |r0|; `rel_residual` gets |r| / |r0|.  When `max_iter` runs out
 * first the call still returns CICY_OK, as upstream's CG does, with
 * `iterations` = max_iter and `rel_residual` > tol.  Errors: message via
 * cicy_host_last_error(). */
cicy_status cicy_jacobi_pcg_static(int32_t n, int32_t nnz, const int32_t* row_ptr, const int32_t* col_ind, const double* values,
                                   const double* b, double* x, double tol, int64_t max_iter, void* stream, int64_t* iterations,
                                   double* rel_residual);

#ifdef __cplusplus
}
#endif
#endif /* CICY_B200_H */
