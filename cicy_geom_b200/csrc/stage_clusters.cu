// Network upload, contact grid, tunnelling-contact search, Hoshen-Kopelman
// labelling, junction compression, elements, percolation (device).
#include <algorithm>
#include <cmath>

#include "ctx.cuh"
#include "trace.cuh"
#include "uf.cuh"

namespace cicy {

namespace {

constexpr double kZero = 1.0e-10;  // MathMatrix.h:18

// ---------------------------------------------------------------------------
// Contact grid (Contact_grid.cpp:104-295).  Region coordinates and overlap flags
// use the exact upstream operation sequence (FP64, no contraction).
struct PointRegions {
    long long t[4];
    int n;
};

__device__ __forceinline__ PointRegions regions_of(double px, double py, double pz, const GridGeom g) {
    // Calculate_region_coordinates (Contact_grid.cpp:163-184)
    int a = (int)((px - g.min[0]) / g.l[0]);
    if (a < 0) a = 0; else if (a >= g.n[0]) a = g.n[0] - 1;
    int b = (int)((py - g.min[1]) / g.l[1]);
    if (b < 0) b = 0; else if (b >= g.n[1]) b = g.n[1] - 1;
    int c = (int)((pz - g.min[2]) / g.l[2]);
    if (c < 0) c = 0; else if (c >= g.n[2]) c = g.n[2] - 1;
    // Calculate_overlapping_flags (Contact_grid.cpp:186-212)
    double x1 = (double)a * g.l[0] + g.min[0];
    double x2 = x1 + g.l[0];
    double y1 = (double)b * g.l[1] + g.min[1];
    double y2 = y1 + g.l[1];
    double z1 = (double)c * g.l[2] + g.min[2];
    double z2 = z1 + g.l[2];
    const double ov = g.overlap;
    int f0 = 0, f1 = 0, f2 = 0;
    if ((a > 0) && (px >= x1) && (px <= x1 + ov)) f0 = -1;
    else if ((a < g.n[0] - 1) && (px >= x2 - ov) && (px <= x2)) f0 = 1;
    if ((b > 0) && (py >= y1) && (py <= y1 + ov)) f1 = -1;
    else if ((b < g.n[1] - 1) && (py >= y2 - ov) && (py <= y2)) f1 = 1;
    if ((c > 0) && (pz >= z1) && (pz <= z1 + ov)) f2 = -1;
    else if ((c < g.n[2] - 1) && (pz >= z2 - ov) && (pz <= z2)) f2 = 1;
    // Assign_point_to_regions_cnts + Calculate_t (Contact_grid.cpp:214-295)
    const long long sx = g.n[0], sxy = (long long)g.n[0] * g.n[1];
    PointRegions r;
    r.n = 0;
    r.t[r.n++] = a + b * sx + c * sxy;
    if (f0) r.t[r.n++] = (a + f0) + b * sx + c * sxy;
    if (f1) r.t[r.n++] = a + (b + f1) * sx + c * sxy;
    if (f2) r.t[r.n++] = a + b * sx + (c + f2) * sxy;
    return r;
}

__device__ __forceinline__ int trav_rank(const int32_t* __restrict__ off, int n, int q) {
    int lo = 0, hi = n;  // find last i with off[i] <= q
    while (hi - lo > 1) {
        int m = (lo + hi) >> 1;
        if (off[m] <= q) lo = m; else hi = m;
    }
    return lo;
}

// Points in traversal order q = (rank in cnts_inside, position in structure):
// the order Fill_sectioned_domain_cnts pushes them (Contact_grid.cpp:114-160).
__global__ void k_grid_count(int n_trav, const int32_t* __restrict__ trav_off, int n_inside, const int32_t* __restrict__ inside,
                             const int32_t* __restrict__ cstart, const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, GridGeom g, int32_t* __restrict__ trav_pt,
                             int32_t* __restrict__ cnt) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_trav; q += gridDim.x * blockDim.x) {
        int r = trav_rank(trav_off, n_inside, q);
        int P = cstart[inside[r]] + (q - trav_off[r]);
        trav_pt[q] = P;
        PointRegions pr = regions_of(x[P], y[P], z[P], g);
        for (int i = 0; i < pr.n; i++) atomicAdd(&cnt[pr.t[i]], 1);
    }
}

__global__ void k_grid_scatter(int n_trav, const int32_t* __restrict__ trav_pt, const double* __restrict__ x,
                               const double* __restrict__ y, const double* __restrict__ z, GridGeom g,
                               int32_t* __restrict__ cursor, uint32_t* __restrict__ slot_q, int32_t* __restrict__ slot_region) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_trav; q += gridDim.x * blockDim.x) {
        int P = trav_pt[q];
        PointRegions pr = regions_of(x[P], y[P], z[P], g);
        for (int i = 0; i < pr.n; i++) {
            int pos = atomicAdd(&cursor[pr.t[i]], 1);
            slot_q[pos] = (uint32_t)q;
            slot_region[pos] = (int32_t)pr.t[i];
        }
    }
}

// ---------------------------------------------------------------------------
// Tunnelling-contact search: every j<k pair of every region, as
// Hoshen_Kopelman::Label_cnts_in_window (Hoshen_Kopelman.cpp:255-369) scans
// them.  A block stages the points of a contiguous run of slots in shared
// memory; each thread owns one slot j and walks k = j+1 .. end of its region.
constexpr int kPairThreads = 256;
constexpr int kPairTile = 512;      // slots owned by one block
constexpr int kPairStage = 1024;    // slots staged in shared memory (tile + region tail): 40 KB, five blocks per SM

struct StagedPt {
    double x, y, z, r;
    int32_t cnt, pt;
};

__device__ __forceinline__ StagedPt load_slot(int s, const uint32_t* __restrict__ slot_sorted, const int32_t* __restrict__ trav_pt,
                                              const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                                              const int32_t* __restrict__ flag, const double* __restrict__ radii) {
    StagedPt sp;
    int P = trav_pt[slot_sorted[s]];
    sp.pt = P;
    sp.x = x[P];
    sp.y = y[P];
    sp.z = z[P];
    sp.cnt = flag[P];
    sp.r = radii[sp.cnt];
    return sp;
}

__global__ void __launch_bounds__(kPairThreads) k_pairs(int n_slots, const int32_t* __restrict__ region_ptr,
                                                        const int32_t* __restrict__ slot_region,
                                                        const uint32_t* __restrict__ slot_sorted,
                                                        const int32_t* __restrict__ trav_pt, const double* __restrict__ x,
                                                        const double* __restrict__ y, const double* __restrict__ z,
                                                        const int32_t* __restrict__ flag, const double* __restrict__ radii,
                                                        double vdw, double tunnel, int cap, int32_t* __restrict__ count,
                                                        int32_t* __restrict__ ra, int32_t* __restrict__ rb,
                                                        int32_t* __restrict__ rpa, int32_t* __restrict__ rpb,
                                                        double* __restrict__ rd, uint64_t* __restrict__ rkey) {
    extern __shared__ unsigned char smem_raw[];
    StagedPt* st = reinterpret_cast<StagedPt*>(smem_raw);
    const int s0 = blockIdx.x * kPairTile;
    if (s0 >= n_slots) return;
    const int s_last = min(s0 + kPairTile, n_slots) - 1;
    int stage_end = region_ptr[slot_region[s_last] + 1];
    stage_end = min(stage_end, s0 + kPairStage);
    for (int s = s0 + threadIdx.x; s < stage_end; s += blockDim.x)
        st[s - s0] = load_slot(s, slot_sorted, trav_pt, x, y, z, flag, radii);
    __syncthreads();
    for (int s = s0 + threadIdx.x; s <= s_last; s += blockDim.x) {
        const int t = slot_region[s];
        const int r0 = region_ptr[t], r1 = region_ptr[t + 1];
        const StagedPt p1 = st[s - s0];
        for (int k = s + 1; k < r1; k++) {
            StagedPt p2 = (k < stage_end) ? st[k - s0] : load_slot(k, slot_sorted, trav_pt, x, y, z, flag, radii);
            if (p1.cnt == p2.cnt) continue;
            // Point_3D::distance_to (Geometry_3D.cpp:64-70), then the junction distance
            double dx = p1.x - p2.x, dy = p1.y - p2.y, dz = p1.z - p2.z;
            double dist_cnts = sqrt(dx * dx + dy * dy + dz * dz);
            double dj = dist_cnts - p1.r - p2.r;
            if (dj < vdw) dj = vdw;
            if (dj <= tunnel) {
                int pos = atomicAdd(count, 1);
                if (pos < cap) {
                    const bool lo1 = p1.cnt < p2.cnt;
                    ra[pos] = lo1 ? p1.cnt : p2.cnt;
                    rb[pos] = lo1 ? p2.cnt : p1.cnt;
                    rpa[pos] = lo1 ? p1.pt : p2.pt;
                    rpb[pos] = lo1 ? p2.pt : p1.pt;
                    rd[pos] = dj;
                    rkey[pos] = ((uint64_t)t << 26) | ((uint64_t)(s - r0) << 13) | (uint64_t)(k - r0);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// point_contacts: for each (Pa, CNTb) keep the strictly smallest junction
// distance, first in scan order on ties (Hoshen_Kopelman.cpp:353-364).
__global__ void k_contact_keys(int n, const int32_t* __restrict__ ra, const int32_t* __restrict__ rb,
                               const int32_t* __restrict__ rpa, int bp, int bc, uint64_t* __restrict__ keys,
                               uint32_t* __restrict__ vals) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        keys[i] = ((uint64_t)ra[i] << (bc + bp)) | ((uint64_t)rb[i] << bp) | (uint64_t)rpa[i];
        vals[i] = (uint32_t)i;
    }
}

__global__ void k_run_heads(int n, const uint64_t* __restrict__ keys, int32_t* __restrict__ head) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

__global__ void k_contact_unique(int n, const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                                 const int32_t* __restrict__ head, const int32_t* __restrict__ head_scan,
                                 const int32_t* __restrict__ ra, const int32_t* __restrict__ rb,
                                 const int32_t* __restrict__ rpa, const int32_t* __restrict__ rpb,
                                 const double* __restrict__ rd, const uint64_t* __restrict__ rkey,
                                 int32_t* __restrict__ ua, int32_t* __restrict__ ub, int32_t* __restrict__ upa,
                                 int32_t* __restrict__ upb, double* __restrict__ ud) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        uint32_t best = vals[i];
        double bd = rd[best];
        uint64_t bk = rkey[best];
        for (int j = i + 1; j < n && keys[j] == keys[i]; j++) {
            uint32_t v = vals[j];
            double d = rd[v];
            uint64_t k = rkey[v];
            if (d < bd || (d == bd && k < bk)) { best = v; bd = d; bk = k; }
        }
        int u = head_scan[i];
        ua[u] = ra[best];
        ub[u] = rb[best];
        upa[u] = rpa[best];
        upb[u] = rpb[best];
        ud[u] = bd;
    }
}

// ---------------------------------------------------------------------------
// Union-find over CNTs (uf.cuh)
__global__ void k_uf_init(int n, int32_t* parent, unsigned long long* minkey) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        parent[i] = i;
        minkey[i] = ~0ull;
    }
}

__global__ void k_uf_union(int n, const int32_t* __restrict__ ua, const int32_t* __restrict__ ub, int32_t* parent) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uf_unite(parent, ua[i], ub[i]);
    }
}

// Roots into a separate array so no thread ever reads a half-flattened parent[].
__global__ void k_uf_flatten(int n, const int32_t* __restrict__ parent, int32_t* __restrict__ root) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) root[i] = uf_root(parent, i);
}

// The upstream label of a cluster is the rank of its first contact in scan
// order (HK76 creates labels in scan order and Merge_labels keeps the smaller
// root, Hoshen_Kopelman.cpp:2908-2989; Cleanup_labels renumbers roots in
// ascending order, :374-425).
__global__ void k_min_scan_key(int n, const int32_t* __restrict__ ra, const uint64_t* __restrict__ rkey,
                               const int32_t* __restrict__ parent, unsigned long long* minkey) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicMin(&minkey[parent[ra[i]]], (unsigned long long)rkey[i]);
}

__global__ void k_root_flags(int n, const int32_t* __restrict__ parent, const unsigned long long* __restrict__ minkey,
                             int32_t* __restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        flag[i] = (parent[i] == i && minkey[i] != ~0ull) ? 1 : 0;
}

__global__ void k_root_keys(int n, const int32_t* __restrict__ flag, const int32_t* __restrict__ scan,
                            const unsigned long long* __restrict__ minkey, uint64_t* keys, uint32_t* vals) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) {
            keys[scan[i]] = minkey[i];
            vals[scan[i]] = (uint32_t)i;
        }
}

__global__ void k_root_rank(int n, const uint32_t* __restrict__ vals, int32_t* __restrict__ rank) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) rank[vals[i]] = i;
}

__global__ void k_labels(int n, const int32_t* __restrict__ parent, const unsigned long long* __restrict__ minkey,
                         const int32_t* __restrict__ rank, int32_t* __restrict__ labels) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int r = parent[i];
        labels[i] = (minkey[r] != ~0ull) ? rank[r] : -1;
    }
}

// ---------------------------------------------------------------------------
// Compress_cnt_cnt_contact_segments (Hoshen_Kopelman.cpp:443-554): one thread per
// (CNT i, CNT j) group walks its contacts in ascending Pa.
__global__ void k_group_heads(int n, const int32_t* __restrict__ ua, const int32_t* __restrict__ ub, int32_t* __restrict__ head) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        head[i] = (i == 0 || ua[i] != ua[i - 1] || ub[i] != ub[i - 1]) ? 1 : 0;
}

__global__ void k_group_starts(int n, const int32_t* __restrict__ head, const int32_t* __restrict__ scan, int32_t* __restrict__ gs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (head[i]) gs[scan[i]] = i;
}

template <bool kWrite>
__global__ void k_compress(int n_groups, int n_uc, const int32_t* __restrict__ gs, const int32_t* __restrict__ ua,
                           const int32_t* __restrict__ ub, const int32_t* __restrict__ upa, const int32_t* __restrict__ upb,
                           const double* __restrict__ ud, int min_points, int32_t* __restrict__ jcnt,
                           const int32_t* __restrict__ jofs, int32_t* __restrict__ jp1, int32_t* __restrict__ jn1,
                           int32_t* __restrict__ jp2, int32_t* __restrict__ jn2, double* __restrict__ jd) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n_groups; g += gridDim.x * blockDim.x) {
        const int b = gs[g], e = (g + 1 < n_groups) ? gs[g + 1] : n_uc;
        const int ci = ua[b], cj = ub[b];
        long long Pi0 = upa[b], Pj0 = upb[b];
        double dmin = ud[b];
        long long Pi_j = Pi0, Pj_j = Pj0;
        int out = 0, base = kWrite ? jofs[g] : 0;
        for (int k = b + 1; k < e; k++) {
            long long Pi1 = upa[k], Pj1 = upb[k];
            double d = ud[k];
            long long dj = Pj1 - Pj0;
            if (dj < 0) dj = -dj;
            if (Pi1 - Pi0 >= min_points || dj >= min_points) {
                if (kWrite) {
                    jp1[base + out] = (int32_t)Pi_j; jn1[base + out] = ci;
                    jp2[base + out] = (int32_t)Pj_j; jn2[base + out] = cj;
                    jd[base + out] = dmin;
                }
                out++;
                dmin = d; Pi_j = Pi1; Pj_j = Pj1;
            } else if (d < dmin) {
                dmin = d; Pi_j = Pi1; Pj_j = Pj1;
            }
            Pi0 = Pi1;
            Pj0 = Pj1;
        }
        if (kWrite) {
            jp1[base + out] = (int32_t)Pi_j; jn1[base + out] = ci;
            jp2[base + out] = (int32_t)Pj_j; jn2[base + out] = cj;
            jd[base + out] = dmin;
        }
        out++;
        if (!kWrite) jcnt[g] = out;
    }
}

// elements_cnt: junction points plus first/last structure point of each CNT with a
// junction (Hoshen_Kopelman.cpp:527-553, Complete_cnt_elements :557-572).
__global__ void k_mark_junctions(int nj, const int32_t* __restrict__ jp1, const int32_t* __restrict__ jn1,
                                 const int32_t* __restrict__ jp2, const int32_t* __restrict__ jn2, int32_t* mark,
                                 int32_t* has_junc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nj; i += gridDim.x * blockDim.x) {
        mark[jp1[i]] = 1;
        mark[jp2[i]] = 1;
        has_junc[jn1[i]] = 1;
        has_junc[jn2[i]] = 1;
    }
}

__global__ void k_mark_ends(int nc, const int32_t* __restrict__ has_junc, const int32_t* __restrict__ cstart,
                            const int32_t* __restrict__ clen, int32_t* mark) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
        if (has_junc[c] && clen[c] > 0) {
            mark[cstart[c]] = 1;
            mark[cstart[c] + clen[c] - 1] = 1;
        }
}

__global__ void k_fill_elements(int np, const int32_t* __restrict__ mark, const int32_t* __restrict__ scan, int32_t* __restrict__ elem) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x)
        if (mark[i]) elem[scan[i]] = i;
}

// ---------------------------------------------------------------------------
// Percolation (Hoshen_Kopelman.cpp:2366-2589): faces {2,4} x, {3,5} y, {0,1} z.
__global__ void k_face_touch(const int32_t* __restrict__ bptr, const int32_t* __restrict__ bidx, const int32_t* __restrict__ labels,
                             int32_t* face_bits) {
    const int first_face[3] = {2, 3, 0};
    for (int d = 0; d < 3; d++) {
        int f = first_face[d];
        for (int i = bptr[f] + blockIdx.x * blockDim.x + threadIdx.x; i < bptr[f + 1]; i += gridDim.x * blockDim.x) {
            int L = labels[bidx[i]];
            if (L != -1) atomicOr(&face_bits[L], 1 << d);
        }
    }
}

__global__ void k_face_perc(const int32_t* __restrict__ bptr, const int32_t* __restrict__ bidx, const int32_t* __restrict__ labels,
                            const int32_t* __restrict__ face_bits, int32_t* perc_bits) {
    const int second_face[3] = {4, 5, 1};
    for (int d = 0; d < 3; d++) {
        int f = second_face[d];
        for (int i = bptr[f] + blockIdx.x * blockDim.x + threadIdx.x; i < bptr[f + 1]; i += gridDim.x * blockDim.x) {
            int L = labels[bidx[i]];
            if (L != -1 && (face_bits[L] >> d & 1)) atomicOr(&perc_bits[L], 1 << d);
        }
    }
}

__global__ void k_nonzero(int n, const int32_t* __restrict__ v, int32_t* __restrict__ f) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) f[i] = v[i] != 0;
}

// Percolated clusters in cnts_inside order (Make_particle_clusters :2331-2363,
// Determine_family_of_percolated_clusters :2524-2589).
__global__ void k_cluster_members(int n_inside, const int32_t* __restrict__ inside, const int32_t* __restrict__ labels,
                                  const int32_t* __restrict__ perc_bits, const int32_t* __restrict__ perc_index,
                                  int bits_rank, int32_t* __restrict__ flag, uint64_t* __restrict__ key) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_inside; i += gridDim.x * blockDim.x) {
        int L = labels[inside[i]];
        bool in = (L >= 0) && perc_bits[L] != 0;
        flag[i] = in ? 1 : 0;
        key[i] = in ? (((uint64_t)perc_index[L] << bits_rank) | (uint64_t)i) : 0;
    }
}

// Group_junctions_same_particle (Hoshen_Kopelman.cpp:2686-2710).
__global__ void k_junction_members(int nj, const int32_t* __restrict__ jn1, const int32_t* __restrict__ labels,
                                   const int32_t* __restrict__ perc_bits, const int32_t* __restrict__ perc_index, int bits_j,
                                   int32_t* __restrict__ flag, uint64_t* __restrict__ key) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nj; i += gridDim.x * blockDim.x) {
        int L = labels[jn1[i]];
        bool in = (L >= 0) && perc_bits[L] != 0;
        flag[i] = in ? 1 : 0;
        key[i] = in ? (((uint64_t)perc_index[L] << bits_j) | (uint64_t)i) : 0;
    }
}

__global__ void k_compact_kv(int n, const int32_t* __restrict__ flag, const int32_t* __restrict__ scan, const uint64_t* __restrict__ kin,
                             uint64_t* __restrict__ kout, uint32_t* __restrict__ vout) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) {
            kout[scan[i]] = kin[i];
            vout[scan[i]] = (uint32_t)i;
        }
}

// CSR from keys sorted by (group << shift | member): counts per group and the member ids.
__global__ void k_group_count(int n, const uint64_t* __restrict__ keys, int shift, int32_t* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) atomicAdd(&cnt[keys[i] >> shift], 1);
}

__global__ void k_member_values(int n, const uint64_t* __restrict__ keys, uint64_t mask, const int32_t* __restrict__ map,
                                int32_t* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int m = (int)(keys[i] & mask);
        out[i] = map ? map[m] : m;
    }
}

int grid_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)b;
}

}  // namespace

Ctx::~Ctx() {
    for (auto* s : systems) delete s;
    for (auto* s : sys_pool) delete s;
    delete hy;
}

int32_t read_i32(Ctx& c, const int32_t* dptr) {
    int32_t v = 0;
    CICY_CUDA(cudaMemcpyAsync(&v, dptr, sizeof(v), cudaMemcpyDeviceToHost, c.stream));
    CICY_CUDA(cudaStreamSynchronize(c.stream));
    return v;
}

void check_status(Ctx& c, const char* where) {
    int st = 0;
    CICY_CUDA(cudaMemcpyAsync(&st, c.status.get(), sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CICY_CUDA(cudaStreamSynchronize(c.stream));
    if (st == DEV_OK) return;
    CICY_CUDA(cudaMemsetAsync(c.status.get(), 0, sizeof(int), c.stream));
    if (st == DEV_TIMEOUT) throw Fail{CICY_E_TIMEOUT, std::string(where) + ": a bounded device wait gave up"};
    if (st == DEV_CAPACITY) throw Fail{CICY_E_CAPACITY, std::string(where) + ": a grid region holds more than 8192 points"};
    if (st == DEV_ZERO_DIAG) throw Fail{CICY_E_ZERO_DIAGONAL, std::string(where) + ": zero on the stiffness diagonal"};
    throw Fail{CICY_E_INTERNAL, std::string(where) + ": device status " + std::to_string(st)};
}

// ---------------------------------------------------------------------------
void upload_network(Ctx& c, const cicy_network& n) {
    if (n.n_points < 0 || n.n_cnts < 0 || n.n_inside < 0 || !n.structure_ptr || !n.radii)
        throw Fail{CICY_E_INPUT, "cicy_upload_network: missing arrays"};
    if (n.n_points >= (1LL << 31) - 1) throw Fail{CICY_E_CAPACITY, "cicy_upload_network: 2^31 or more points"};
    cudaStream_t s = c.stream;
    c.n_points = (int)n.n_points;
    c.n_cnts = n.n_cnts;
    c.n_inside = n.n_inside;
    c.window = n.window;
    // structure lists -> (start, length) runs of consecutive point ids
    c.h_cstart.assign(n.n_cnts, 0);
    c.h_clen.assign(n.n_cnts, 0);
    for (int i = 0; i < n.n_cnts; i++) {
        int64_t b = n.structure_ptr[i], e = n.structure_ptr[i + 1];
        if (e < b) throw Fail{CICY_E_INPUT, "cicy_upload_network: structure_ptr not ascending"};
        if (e > b) {
            int64_t p0 = n.structure_idx[b];
            if (p0 < 0 || p0 + (e - b) > n.n_points) throw Fail{CICY_E_INPUT, "cicy_upload_network: point id out of range"};
            for (int64_t k = b + 1; k < e; k++)
                if (n.structure_idx[k] != n.structure_idx[k - 1] + 1)
                    throw Fail{CICY_E_INPUT, "cicy_upload_network: CNT " + std::to_string(i) + " is not a run of consecutive point ids"};
            c.h_cstart[i] = (int32_t)p0;
        }
        c.h_clen[i] = (int32_t)(e - b);
    }
    std::vector<int32_t> trav_off(n.n_inside + 1, 0);
    for (int i = 0; i < n.n_inside; i++) {
        int ci = n.cnts_inside[i];
        if (ci < 0 || ci >= n.n_cnts) throw Fail{CICY_E_INPUT, "cicy_upload_network: cnts_inside out of range"};
        trav_off[i + 1] = trav_off[i] + c.h_clen[ci];
    }
    c.n_trav = trav_off[n.n_inside];
    c.h_bcnt_ptr.assign(7, 0);
    c.h_bpts_ptr.assign(7, 0);
    if (n.boundary_cnt_ptr)
        for (int f = 0; f < 7; f++) c.h_bcnt_ptr[f] = (int32_t)n.boundary_cnt_ptr[f];
    if (n.boundary_pts_ptr)
        for (int f = 0; f < 7; f++) c.h_bpts_ptr[f] = (int32_t)n.boundary_pts_ptr[f];
    std::vector<int32_t> bpts(c.h_bpts_ptr[6]);
    for (int i = 0; i < c.h_bpts_ptr[6]; i++) bpts[i] = (int32_t)n.boundary_pts_idx[i];

    const size_t np = std::max<int64_t>(n.n_points, 1), nc = std::max(n.n_cnts, 1);
    c.x.ensure(np); c.y.ensure(np); c.z.ensure(np); c.flag.ensure(np);
    c.radii.ensure(nc); c.cstart.ensure(nc); c.clen.ensure(nc);
    c.inside.ensure(std::max(n.n_inside, 1));
    c.trav_off.ensure(n.n_inside + 1);
    c.bcnt_ptr.ensure(7); c.bpts_ptr.ensure(7);
    c.bcnt_idx.ensure(std::max(c.h_bcnt_ptr[6], 1));
    c.bpts_idx.ensure(std::max(c.h_bpts_ptr[6], 1));
    c.status.ensure(1);
    c.i32_scalar.ensure(8);
    c.i64_scalar.ensure(8);
    auto up = [&](void* d, const void* h, size_t bytes) {
        if (bytes) CICY_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s));
    };
    up(c.x.get(), n.x, sizeof(double) * n.n_points);
    up(c.y.get(), n.y, sizeof(double) * n.n_points);
    up(c.z.get(), n.z, sizeof(double) * n.n_points);
    up(c.flag.get(), n.flag, sizeof(int32_t) * n.n_points);
    up(c.radii.get(), n.radii, sizeof(double) * n.n_cnts);
    up(c.cstart.get(), c.h_cstart.data(), sizeof(int32_t) * n.n_cnts);
    up(c.clen.get(), c.h_clen.data(), sizeof(int32_t) * n.n_cnts);
    up(c.inside.get(), n.cnts_inside, sizeof(int32_t) * n.n_inside);
    up(c.trav_off.get(), trav_off.data(), sizeof(int32_t) * (n.n_inside + 1));
    up(c.bcnt_ptr.get(), c.h_bcnt_ptr.data(), sizeof(int32_t) * 7);
    up(c.bpts_ptr.get(), c.h_bpts_ptr.data(), sizeof(int32_t) * 7);
    up(c.bcnt_idx.get(), n.boundary_cnt_idx, sizeof(int32_t) * c.h_bcnt_ptr[6]);
    up(c.bpts_idx.get(), bpts.data(), sizeof(int32_t) * c.h_bpts_ptr[6]);
    CICY_CUDA(cudaMemsetAsync(c.status.get(), 0, sizeof(int), s));
    CICY_CUDA(cudaStreamSynchronize(s));
    c.stage = 1;
    c.have_backbone = false;
    c.have_volumes = false;
    c.have_hybrid = false;
}

// ---------------------------------------------------------------------------
void run_contact_grid(Ctx& c, const cicy_params& p) {
    if (c.stage < 1) throw Fail{CICY_E_STATE, "cicy_contact_grid: no network uploaded"};
    cudaStream_t s = c.stream;
    CICY_TRACE("contact_grid", s);
    const cicy_cuboid& w = c.window;
    // Generate_contact_grid + Adjust_regions_if_needed (Contact_grid.cpp:18-102)
    GridGeom& g = c.grid;
    g.n[0] = std::max(1, (int)(w.len_x / p.gs_min[0]));
    g.n[1] = std::max(1, (int)(w.len_y / p.gs_min[1]));
    g.n[2] = std::max(1, (int)(w.len_z / p.gs_min[2]));
    g.l[0] = p.gs_min[0]; g.l[1] = p.gs_min[1]; g.l[2] = p.gs_min[2];
    const double max_ov = std::max(p.gs_overlap_cnt, p.gs_overlap_gnp);
    const double lens[3] = {w.len_x, w.len_y, w.len_z};
    for (int a = 0; a < 3; a++)
        if (p.gs_min[a] < 2 * max_ov) {
            g.l[a] = 2.0 * (max_ov + kZero);
            g.n[a] = 1 + (int)(lens[a] / g.l[a]);
        }
    g.min[0] = w.min_x; g.min[1] = w.min_y; g.min[2] = w.min_z;
    g.overlap = p.gs_overlap_cnt;
    g.total = (long long)g.n[0] * g.n[1] * g.n[2];
    if (g.total <= 0) throw Fail{CICY_E_INPUT, "Generate_contact_grid: invalid number of subregions"};
    if (g.total >= (1LL << 31) - 2 || g.total >= (1LL << 38)) throw Fail{CICY_E_CAPACITY, "Generate_contact_grid: too many regions"};
    const int R = (int)g.total;
    c.region_cnt.ensure(R + 1);
    c.region_ptr.ensure(R + 1);
    c.region_cur.ensure(R + 1);
    c.trav_pt.ensure(std::max(c.n_trav, 1));
    CICY_CUDA(cudaMemsetAsync(c.region_cnt.get(), 0, sizeof(int32_t) * (R + 1), s));
    if (c.n_trav > 0) {
        k_grid_count<<<grid_for(c.n_trav), 256, 0, s>>>(c.n_trav, c.trav_off.get(), c.n_inside, c.inside.get(), c.cstart.get(),
                                                      c.x.get(), c.y.get(), c.z.get(), g, c.trav_pt.get(), c.region_cnt.get());
        c.launches++;
    }
    exclusive_scan_i32(c.region_cnt.get(), c.region_ptr.get(), R + 1, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
    c.n_slots = read_i32(c, c.i32_scalar.get());
    const int S = c.n_slots;
    c.slot_q.ensure(std::max(S, 1));
    c.slot_sorted.ensure(std::max(S, 1));
    c.slot_region.ensure(std::max(S, 1));
    c.seg_large.ensure(R + 1);
    CICY_CUDA(cudaMemcpyAsync(c.region_cur.get(), c.region_ptr.get(), sizeof(int32_t) * (R + 1), cudaMemcpyDeviceToDevice, s));
    if (c.n_trav > 0) {
        k_grid_scatter<<<grid_for(c.n_trav), 256, 0, s>>>(c.n_trav, c.trav_pt.get(), c.x.get(), c.y.get(), c.z.get(), g,
                                                        c.region_cur.get(), c.slot_q.get(), c.slot_region.get());
        c.launches++;
    }
    segmented_sort_u32(c.region_ptr.get(), R, c.slot_q.get(), c.slot_sorted.get(), c.seg_large.get(), c.i32_scalar.get() + 1,
                       c.status.get(), s, c.launches);
    CICY_LAUNCH_CHECK();
    check_status(c, "Generate_contact_grid");
    c.stage = 2;
}

// ---------------------------------------------------------------------------
void run_clusters(Ctx& c, const cicy_params& p) {
    if (c.stage < 2) throw Fail{CICY_E_STATE, "cicy_clusters: run cicy_contact_grid first"};
    cudaStream_t s = c.stream;
    CICY_TRACE("clusters", s);
    TraceSeq tr(s);
    const int S = c.n_slots, NC = std::max(c.n_cnts, 1), NP = std::max(c.n_points, 1);
    // ---- pair tests ----
    int cap = std::max(1 << 16, S / 4);
    c.raw_count.ensure(1);
    for (int attempt = 0; attempt < 2; attempt++) {
        c.raw_a.ensure(cap); c.raw_b.ensure(cap); c.raw_pa.ensure(cap); c.raw_pb.ensure(cap);
        c.raw_d.ensure(cap); c.raw_key.ensure(cap);
        CICY_CUDA(cudaMemsetAsync(c.raw_count.get(), 0, sizeof(int32_t), s));
        if (S > 0) {
            const int blocks = ceil_div(S, kPairTile);
            const size_t smem = sizeof(StagedPt) * kPairStage;
            static bool attr_set = false;
            if (!attr_set) {
                CICY_CUDA(cudaFuncSetAttribute(k_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                attr_set = true;
            }
            k_pairs<<<blocks, kPairThreads, smem, s>>>(S, c.region_ptr.get(), c.slot_region.get(), c.slot_sorted.get(),
                                                       c.trav_pt.get(), c.x.get(), c.y.get(), c.z.get(), c.flag.get(),
                                                       c.radii.get(), p.van_der_waals_dist, p.tunneling_dist, cap,
                                                       c.raw_count.get(), c.raw_a.get(), c.raw_b.get(), c.raw_pa.get(),
                                                       c.raw_pb.get(), c.raw_d.get(), c.raw_key.get());
            c.launches++;
            CICY_LAUNCH_CHECK();
        }
        c.n_raw = read_i32(c, c.raw_count.get());
        if (c.n_raw <= cap) break;
        cap = c.n_raw + c.n_raw / 8 + 1024;
        if (attempt == 1) throw Fail{CICY_E_INTERNAL, "contact buffer overflow"};
    }
    const int NR = c.n_raw;
    tr.mark("clusters.pairs");
    // ---- point_contacts ----
    const int bp = bits_for((uint64_t)NP), bc = bits_for((uint64_t)NC);
    if (bp + 2 * bc > 64) throw Fail{CICY_E_CAPACITY, "too many points/CNTs for the 64-bit contact key"};
    c.sort_k.ensure(std::max(NR, NC) + 1);
    c.sort_v.ensure(std::max(NR, NC) + 1);
    c.flags.ensure(std::max(std::max(NR, NC), c.n_inside) + 1);
    c.flags_scan.ensure(std::max(std::max(NR, NC), c.n_inside) + 1);
    c.uc_a.ensure(std::max(NR, 1)); c.uc_b.ensure(std::max(NR, 1)); c.uc_pa.ensure(std::max(NR, 1));
    c.uc_pb.ensure(std::max(NR, 1)); c.uc_d.ensure(std::max(NR, 1));
    if (NR > 0) {
        k_contact_keys<<<grid_for(NR), 256, 0, s>>>(NR, c.raw_a.get(), c.raw_b.get(), c.raw_pa.get(), bp, bc, c.sort_k.get(), c.sort_v.get());
        c.launches++;
        radix_sort_pairs(c.sort_k.get(), c.sort_v.get(), NR, bp + 2 * bc, c.rs, s, c.launches);
        k_run_heads<<<grid_for(NR), 256, 0, s>>>(NR, c.sort_k.get(), c.flags.get());
        c.launches++;
        exclusive_scan_i32(c.flags.get(), c.flags_scan.get(), NR, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
        k_contact_unique<<<grid_for(NR), 256, 0, s>>>(NR, c.sort_k.get(), c.sort_v.get(), c.flags.get(), c.flags_scan.get(),
                                                    c.raw_a.get(), c.raw_b.get(), c.raw_pa.get(), c.raw_pb.get(), c.raw_d.get(),
                                                    c.raw_key.get(), c.uc_a.get(), c.uc_b.get(), c.uc_pa.get(), c.uc_pb.get(),
                                                    c.uc_d.get());
        c.launches++;
        c.n_uc = read_i32(c, c.i32_scalar.get());
    } else {
        c.n_uc = 0;
    }
    const int NU = c.n_uc;
    tr.mark("clusters.point_contacts");
    // ---- labels ----
    c.parent.ensure(NC); c.minkey.ensure(NC); c.labels.ensure(NC); c.root_rank.ensure(NC);
    k_uf_init<<<grid_for(NC), 256, 0, s>>>(c.n_cnts, c.parent.get(), c.minkey.get());
    c.launches++;
    if (NU > 0) {
        k_uf_union<<<grid_for(NU), 256, 0, s>>>(NU, c.uc_a.get(), c.uc_b.get(), c.parent.get());
        c.launches++;
    }
    c.uf_root.ensure(NC);
    k_uf_flatten<<<grid_for(NC), 256, 0, s>>>(c.n_cnts, c.parent.get(), c.uf_root.get());
    CICY_CUDA(cudaMemcpyAsync(c.parent.get(), c.uf_root.get(), sizeof(int32_t) * c.n_cnts, cudaMemcpyDeviceToDevice, s));
    c.launches++;
    if (NR > 0) {
        k_min_scan_key<<<grid_for(NR), 256, 0, s>>>(NR, c.raw_a.get(), c.raw_key.get(), c.parent.get(), c.minkey.get());
        c.launches++;
    }
    k_root_flags<<<grid_for(NC), 256, 0, s>>>(c.n_cnts, c.parent.get(), c.minkey.get(), c.flags.get());
    exclusive_scan_i32(c.flags.get(), c.flags_scan.get(), c.n_cnts, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
    k_root_keys<<<grid_for(NC), 256, 0, s>>>(c.n_cnts, c.flags.get(), c.flags_scan.get(), c.minkey.get(), c.sort_k.get(), c.sort_v.get());
    c.launches += 2;
    c.n_labels = read_i32(c, c.i32_scalar.get());
    if (c.n_labels > 0) {
        radix_sort_pairs(c.sort_k.get(), c.sort_v.get(), c.n_labels, bits_for((uint64_t)c.grid.total) + 26, c.rs, s, c.launches);
        k_root_rank<<<grid_for(c.n_labels), 256, 0, s>>>(c.n_labels, c.sort_v.get(), c.root_rank.get());
        c.launches++;
    }
    k_labels<<<grid_for(NC), 256, 0, s>>>(c.n_cnts, c.parent.get(), c.minkey.get(), c.root_rank.get(), c.labels.get());
    c.launches++;
    tr.mark("clusters.labels");
    // ---- junction compression ----
    c.grp_start.ensure(std::max(NU, 1)); c.junc_cnt.ensure(std::max(NU, 1) + 1); c.junc_ofs.ensure(std::max(NU, 1) + 1);
    int n_groups = 0;
    if (NU > 0) {
        k_group_heads<<<grid_for(NU), 256, 0, s>>>(NU, c.uc_a.get(), c.uc_b.get(), c.flags.get());
        exclusive_scan_i32(c.flags.get(), c.flags_scan.get(), NU, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
        k_group_starts<<<grid_for(NU), 256, 0, s>>>(NU, c.flags.get(), c.flags_scan.get(), c.grp_start.get());
        c.launches += 2;
        n_groups = read_i32(c, c.i32_scalar.get());
        k_compress<false><<<grid_for(n_groups), 256, 0, s>>>(n_groups, NU, c.grp_start.get(), c.uc_a.get(), c.uc_b.get(), c.uc_pa.get(),
                                                         c.uc_pb.get(), c.uc_d.get(), p.min_points, c.junc_cnt.get(), nullptr,
                                                         nullptr, nullptr, nullptr, nullptr, nullptr);
        exclusive_scan_i32(c.junc_cnt.get(), c.junc_ofs.get(), n_groups, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
        c.launches++;
        c.n_junc = read_i32(c, c.i32_scalar.get());
    } else {
        c.n_junc = 0;
    }
    const int NJ = c.n_junc;
    c.j_p1.ensure(std::max(NJ, 1)); c.j_n1.ensure(std::max(NJ, 1)); c.j_p2.ensure(std::max(NJ, 1));
    c.j_n2.ensure(std::max(NJ, 1)); c.j_d.ensure(std::max(NJ, 1));
    if (NJ > 0) {
        k_compress<true><<<grid_for(n_groups), 256, 0, s>>>(n_groups, NU, c.grp_start.get(), c.uc_a.get(), c.uc_b.get(), c.uc_pa.get(),
                                                        c.uc_pb.get(), c.uc_d.get(), p.min_points, nullptr, c.junc_ofs.get(),
                                                        c.j_p1.get(), c.j_n1.get(), c.j_p2.get(), c.j_n2.get(), c.j_d.get());
        c.launches++;
    }
    tr.mark("clusters.junctions");
    // ---- elements ----
    c.mark.ensure(NP + 1); c.mark_scan.ensure(NP + 1); c.has_junc.ensure(NC);
    CICY_CUDA(cudaMemsetAsync(c.mark.get(), 0, sizeof(int32_t) * (NP + 1), s));
    CICY_CUDA(cudaMemsetAsync(c.has_junc.get(), 0, sizeof(int32_t) * NC, s));
    if (NJ > 0) {
        k_mark_junctions<<<grid_for(NJ), 256, 0, s>>>(NJ, c.j_p1.get(), c.j_n1.get(), c.j_p2.get(), c.j_n2.get(), c.mark.get(), c.has_junc.get());
        k_mark_ends<<<grid_for(NC), 256, 0, s>>>(c.n_cnts, c.has_junc.get(), c.cstart.get(), c.clen.get(), c.mark.get());
        c.launches += 2;
    }
    exclusive_scan_i32(c.mark.get(), c.mark_scan.get(), c.n_points + 1, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
    int n_elem = read_i32(c, c.i32_scalar.get());
    c.elem_idx.ensure(std::max(n_elem, 1));
    k_fill_elements<<<grid_for(NP), 256, 0, s>>>(c.n_points, c.mark.get(), c.mark_scan.get(), c.elem_idx.get());
    c.launches++;
    tr.mark("clusters.elements");
    // ---- percolation and families ----
    const int NL = std::max(c.n_labels, 1);
    c.face_bits.ensure(NL); c.perc_bits.ensure(NL); c.perc_index.ensure(NL + 1);
    CICY_CUDA(cudaMemsetAsync(c.face_bits.get(), 0, sizeof(int32_t) * NL, s));
    CICY_CUDA(cudaMemsetAsync(c.perc_bits.get(), 0, sizeof(int32_t) * NL, s));
    if (c.h_bcnt_ptr[6] > 0) {
        k_face_touch<<<grid_for(c.h_bcnt_ptr[6]), 256, 0, s>>>(c.bcnt_ptr.get(), c.bcnt_idx.get(), c.labels.get(), c.face_bits.get());
        k_face_perc<<<grid_for(c.h_bcnt_ptr[6]), 256, 0, s>>>(c.bcnt_ptr.get(), c.bcnt_idx.get(), c.labels.get(), c.face_bits.get(), c.perc_bits.get());
        c.launches += 2;
    }
    k_nonzero<<<grid_for(NL), 256, 0, s>>>(c.n_labels, c.perc_bits.get(), c.flags.get());
    exclusive_scan_i32(c.flags.get(), c.perc_index.get(), c.n_labels, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
    c.launches++;
    c.n_perc = read_i32(c, c.i32_scalar.get());
    // families in percolated order (Family_map, Hoshen_Kopelman.cpp:2591-2622)
    c.h_family.clear();
    if (c.n_perc > 0) {
        std::vector<int32_t> bits(c.n_labels);
        CICY_CUDA(cudaMemcpyAsync(bits.data(), c.perc_bits.get(), sizeof(int32_t) * c.n_labels, cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaStreamSynchronize(s));
        static const int fam_of_bits[8] = {-1, 0, 1, 3, 2, 4, 5, 6};
        for (int L = 0; L < c.n_labels; L++)
            if (bits[L]) c.h_family.push_back(fam_of_bits[bits[L]]);
    }
    tr.mark("clusters.percolation");
    // percolated clusters (CNTs in cnts_inside order) and their junctions
    const int NP_ = std::max(c.n_perc, 1);
    c.clu_ptr.ensure(NP_ + 1); c.cj_ptr.ensure(NP_ + 1);
    c.h_clu_ptr.assign(c.n_perc + 1, 0);
    c.h_cj_ptr.assign(c.n_perc + 1, 0);
    if (c.n_perc > 0) {
        const int br = bits_for((uint64_t)std::max(c.n_inside, 1));
        c.work_i32a.ensure(std::max(c.n_inside, NJ) + 1);
        c.rs.keys_tmp.ensure(std::max(c.n_inside, NJ) + 1);
        // members
        uint64_t* kin = c.rs.keys_tmp.get();  // reuse as staging; radix uses its own tmp buffers below
        DBuf<uint64_t> stage_keys;
        stage_keys.ensure(std::max(c.n_inside, NJ) + 1);
        k_cluster_members<<<grid_for(c.n_inside), 256, 0, s>>>(c.n_inside, c.inside.get(), c.labels.get(), c.perc_bits.get(),
                                                             c.perc_index.get(), br, c.flags.get(), stage_keys.get());
        exclusive_scan_i32(c.flags.get(), c.flags_scan.get(), c.n_inside, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
        k_compact_kv<<<grid_for(c.n_inside), 256, 0, s>>>(c.n_inside, c.flags.get(), c.flags_scan.get(), stage_keys.get(), c.sort_k.get(), c.sort_v.get());
        c.launches += 2;
        (void)kin;
        int nm = read_i32(c, c.i32_scalar.get());
        radix_sort_pairs(c.sort_k.get(), c.sort_v.get(), nm, br + bits_for((uint64_t)c.n_perc), c.rs, s, c.launches);
        c.clu_idx.ensure(std::max(nm, 1));
        CICY_CUDA(cudaMemsetAsync(c.work_i32a.get(), 0, sizeof(int32_t) * (c.n_perc + 1), s));
        k_group_count<<<grid_for(nm), 256, 0, s>>>(nm, c.sort_k.get(), br, c.work_i32a.get());
        exclusive_scan_i32(c.work_i32a.get(), c.clu_ptr.get(), c.n_perc + 1, nullptr, c.scan_tmp32, s, c.launches);
        k_member_values<<<grid_for(nm), 256, 0, s>>>(nm, c.sort_k.get(), (1ull << br) - 1, c.inside.get(), c.clu_idx.get());
        c.launches += 2;
        CICY_CUDA(cudaMemcpyAsync(c.h_clu_ptr.data(), c.clu_ptr.get(), sizeof(int32_t) * (c.n_perc + 1), cudaMemcpyDeviceToHost, s));
        // junctions
        const int bj = bits_for((uint64_t)std::max(NJ, 1));
        int njm = 0;
        if (NJ > 0) {
            k_junction_members<<<grid_for(NJ), 256, 0, s>>>(NJ, c.j_n1.get(), c.labels.get(), c.perc_bits.get(), c.perc_index.get(),
                                                          bj, c.flags.get(), stage_keys.get());
            exclusive_scan_i32(c.flags.get(), c.flags_scan.get(), NJ, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
            k_compact_kv<<<grid_for(NJ), 256, 0, s>>>(NJ, c.flags.get(), c.flags_scan.get(), stage_keys.get(), c.sort_k.get(), c.sort_v.get());
            c.launches += 2;
            njm = read_i32(c, c.i32_scalar.get());
            radix_sort_pairs(c.sort_k.get(), c.sort_v.get(), njm, bj + bits_for((uint64_t)c.n_perc), c.rs, s, c.launches);
        }
        c.cj_idx.ensure(std::max(njm, 1));
        CICY_CUDA(cudaMemsetAsync(c.work_i32a.get(), 0, sizeof(int32_t) * (c.n_perc + 1), s));
        if (njm > 0) {
            k_group_count<<<grid_for(njm), 256, 0, s>>>(njm, c.sort_k.get(), bj, c.work_i32a.get());
            k_member_values<<<grid_for(njm), 256, 0, s>>>(njm, c.sort_k.get(), (1ull << bj) - 1, nullptr, c.cj_idx.get());
            c.launches += 2;
        }
        exclusive_scan_i32(c.work_i32a.get(), c.cj_ptr.get(), c.n_perc + 1, nullptr, c.scan_tmp32, s, c.launches);
        CICY_CUDA(cudaMemcpyAsync(c.h_cj_ptr.data(), c.cj_ptr.get(), sizeof(int32_t) * (c.n_perc + 1), cudaMemcpyDeviceToHost, s));
        CICY_CUDA(cudaStreamSynchronize(s));
        stage_keys.release();
    }
    CICY_LAUNCH_CHECK();
    check_status(c, "Determine_clusters_and_percolation");
    tr.mark("clusters.members");
    c.stage = 3;
    c.have_backbone = false;
    c.have_volumes = false;
    c.have_hybrid = false;
}

}  // namespace cicy
