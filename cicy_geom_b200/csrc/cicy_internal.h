// Internal declarations shared by the host-side sources of libcicy_b200.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cicy_b200.h"

struct cicy_host_network;

namespace cicy {

// Host-owned CNT network in the layout of cicy_network.
struct HostNetwork {
    std::vector<double> x, y, z;
    std::vector<int32_t> flag;
    std::vector<double> radii;
    std::vector<int64_t> structure_ptr, structure_idx;
    std::vector<int32_t> cnts_inside;
    std::vector<int64_t> boundary_cnt_ptr;
    std::vector<int32_t> boundary_cnt_idx;
    std::vector<int64_t> boundary_pts_ptr, boundary_pts_idx;
    cicy_cuboid window;
};

HostNetwork* generate_cnt_network(const cicy_gen_params& g);
cicy_status extract_window(const HostNetwork& in, const cicy_window_params& w, HostNetwork** out, std::string& err);
HostNetwork* host_network_from_view(const cicy_network& n);
cicy_status read_network_files(const std::string& dir, int file_type, HostNetwork** out, std::string& err);

// GNPs of a gnp_data.dat with their upstream vertices and face planes.
struct GnpSet {
    int32_t n = 0;
    std::vector<double> l, t, center, rotation, vertices, planes;  // per GNP: 1, 1, 3, 9, 24, 24
};
cicy_status read_gnp_file(const std::string& dir, GnpSet** out, std::string& err);

// GNP part of the contact grid (gnp_grid.cu): region grid and region lists (CSR, GNP indices).
struct GnpGrid {
    int n_regions[3] = {0, 0, 0};
    double l_regions[3] = {0, 0, 0};
    std::vector<int32_t> ptr, idx;
    int64_t launches = 0;
};
void gnp_sectioned_domain(const GnpSet& g, const std::vector<int32_t>& inside, const cicy_cuboid& w, const double gs_min[3],
                          double overlap_cnt, double overlap_gnp, GnpGrid& out);
// GNP-GNP contact pass (gnp_pairs.cu): pairs within the tunnelling cutoff in
// upstream's visiting order, with distance, direction and the move of b.
struct GnpPairs {
    std::vector<int32_t> a, b, penetrating;
    std::vector<double> dist, direction, displacement;  // 1, 3, 3 per pair
    std::vector<double> point_a, point_b;               // junction points, 3 per pair
    std::vector<int32_t> outside;                       // 1: point_a outside the sample, 2: point_b
    int64_t n_visits = 0, n_pairs = 0, launches = 0;
};
void gnp_contact_pairs(const GnpSet& g, const GnpGrid& grid, double vdw, double tunnel, const cicy_cuboid& sample, bool allow_simplex3,
                       GnpPairs& out);
// GNP point structures after Add_gnp_junction (gnp_labels.cu).
struct GnpStructures {
    std::vector<double> points;                   // 3 per point: the initial ones, then the junction points
    std::vector<int32_t> structure_ptr, structure_idx;
    std::vector<int32_t> junctions;               // Pa, GNPa, Pb, GNPb per junction
    std::vector<double> junction_dist;
    int32_t n_boundary = 0;                       // initial points (gnp_pts_bdds)
    std::vector<int32_t> boundary_used;           // bp_flags
    int64_t launches = 0;
};
void gnp_junction_structures(const GnpPairs& pairs, int n_gnps, double tol_gnp2, const std::vector<double>& init_points,
                             const std::vector<int32_t>& init_ptr, const std::vector<int32_t>& init_idx, GnpStructures& out);
// GNP part of the window extraction (host_network.cpp): gnps_inside, boundary_gnp,
// and the GNP boundary points (points_gnp, structure_gnp, boundary_gnp_pts).
struct GnpWindow {
    std::vector<int32_t> inside;
    std::vector<std::vector<int32_t>> boundary_gnp, boundary_pts, structure;
    std::vector<double> points;  // 3 per point
    std::vector<int32_t> point_gnp, point_boundary;
    std::vector<double> volume;  // per GNP: the volume inside the window where the extraction sets it, else NaN
    std::vector<int32_t> flat_bgnp_ptr, flat_bgnp_idx, flat_bpts_ptr, flat_bpts_idx, flat_st_ptr, flat_st_idx;
};
cicy_status gnp_window(const GnpSet& g, const cicy_window_params& w, GnpWindow& out, std::string& err);
// Message returned by cicy_host_last_error() on this thread.
void set_host_error(const std::string& msg);
void host_network_view(const HostNetwork& h, cicy_network& v);

}  // namespace cicy

struct cicy_host_network {
    cicy::HostNetwork net;
};

struct cicy_gnp_set {
    cicy::GnpSet g;
};

struct cicy_gnp_grid {
    cicy::GnpGrid grid;
};

struct cicy_gnp_pairs {
    cicy::GnpPairs pairs;
};

struct cicy_gnp_window {
    cicy::GnpWindow w;
};

struct cicy_gnp_points {
    cicy::GnpStructures s;
};
