// Electrical stage of a mixed CNT/GNP network on the device (GNP_CNT_mix):
// Electrical_analysis::Perform_analysis_on_clusters (Electrical_analysis.cpp:10-145,
// 229-675) with the GNP branches of Direct_Electrifying (LM_matrix_for_gnps,
// Fill_2d_matrices_mixed_junctions, Fill_2d_matrices_gnp with each GNP's
// triangulation, Fill_2d_matrices_gnp_junctions; Direct_Electrifying.cpp:307-348,
// 903-1319) and Backbone_Network (Find_zero_current, Find_backbone_gnps and its
// removal cascade, Backbone_Network.cpp:64-245, 577-1127).
//
// Included at the end of stage_dea.cu (same translation unit, built without FMA
// contraction): the CNT part of every system is stage_dea.cu's solve_dea, which
// calls the three hooks below for the GNP part, so both kinds of resistors go
// through one sort-and-reduce assembly in upstream's insertion order.
//
// Layout: GNP point lists are a CSR of fixed capacity per GNP with the current
// length in scount (the backbone keeps points at the front); node numbers of GNP
// points in lmm_g; each GNP's triangulation in a fixed slot of kTriCap edges with
// its edge count in tri_cnt (0: none, as upstream's empty gnps[].triangulation).
#pragma once

#include "gnp_triangulation.cuh"

namespace cicy {

namespace {

constexpr int kTriMaxPoints = 256;          // points per GNP the triangulation holds
constexpr int kTriCap = 3 * kTriMaxPoints;  // edges per GNP triangulation slot
// GNP volume members in HybridDev::vol_acc (the CNT ones are Ctx::vol_acc's)
enum HybVol : int { HV_GNP = 0, HV_DEAD_GNP = 8, HV_WORDS = 15 };

// LM_matrix_for_gnps (Direct_Electrifying.cpp:307-348): points of the cluster's GNPs in
// list order; a point without a node (not on a prescribed face) takes the next one.
__global__ void k_gnp_node_counts(int ng, const int32_t* __restrict__ gnps, const int32_t* __restrict__ sptr,
                                  const int32_t* __restrict__ sidx, const int32_t* __restrict__ scount, const int32_t* __restrict__ lmm_g,
                                  int32_t* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
        const int g = gnps[i], b = sptr[g];
        int k = 0;
        for (int m = 0; m < scount[g]; m++) k += lmm_g[sidx[b + m]] < 0 ? 1 : 0;
        cnt[i] = k;
    }
}

__global__ void k_gnp_node_assign(int ng, int first, const int32_t* __restrict__ gnps, const int32_t* __restrict__ sptr,
                                  const int32_t* __restrict__ sidx, const int32_t* __restrict__ scount, const int32_t* __restrict__ base,
                                  int32_t* __restrict__ lmm_g) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
        const int g = gnps[i], b = sptr[g];
        int node = first + base[i];
        for (int m = 0; m < scount[g]; m++) {
            const int P = sidx[b + m];
            if (lmm_g[P] < 0) lmm_g[P] = node++;
        }
    }
}

// Triangulation::Generate_3d_trangulation of each GNP of the cluster whose triangulation is
// empty, or of all of them in the unit-resistor pass (Fill_2d_matrices_gnp, :1040-1058).
__global__ void k_gnp_triangulate(int ng, int all, const int32_t* __restrict__ gnps, const double* __restrict__ pts,
                                  const int32_t* __restrict__ sptr, const int32_t* __restrict__ sidx, const int32_t* __restrict__ scount,
                                  const double* __restrict__ frame, gnp::TriWork<kTriMaxPoints>* work, int32_t* __restrict__ tri,
                                  int32_t* __restrict__ tri_cnt, int* status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
        const int g = gnps[i];
        if (!all && tri_cnt[g] > 0) continue;
        const double* q = frame + 16 * (size_t)g;  // l, centre[3], rotation[9], face-0 normal[3]
        const int n = scount[g];
        const int k = gnp::triangulate<kTriMaxPoints>(pts, sidx + sptr[g], n, q[0], q + 1, q + 4, gnp::P3{q[13], q[14], q[15]}, work[i],
                                                      tri + 2 * (size_t)kTriCap * g, kTriCap);
        if (k < 0) {
            atomicCAS(status, 0, (int)DEV_CAPACITY);
            tri_cnt[g] = 0;
            continue;
        }
        if (n > 4 && k == 0) atomicCAS(status, 0, (int)DEV_INPUT);  // Bowyer-Watson gave no triangulation
        tri_cnt[g] = k;
    }
}

__global__ void k_gnp_tri_counts(int ng, const int32_t* __restrict__ gnps, const int32_t* __restrict__ tri_cnt, int32_t* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) cnt[i] = tri_cnt[gnps[i]];
}

// Fill_2d_matrices_mixed_junctions (:903-1019): a junction whose two points have nodes is a
// resistor; it joins the free block by overwriting, or adds to a prescribed node's entries
// when more than two faces are prescribed, or is dropped; its GNP point takes the CNT's
// radius (points_cnt_rad, the last such junction of the list wins).
__global__ void k_mix_edges(int nm, int base, int r_flag, int reserved, int jtype, double jres, double C1, double C2,
                            const int32_t* __restrict__ mix, const int32_t* __restrict__ p1, const int32_t* __restrict__ n1c,
                            const int32_t* __restrict__ p2, const int32_t* __restrict__ n2g, const double* __restrict__ jd,
                            const double* __restrict__ radii, const double* __restrict__ gt, const int32_t* __restrict__ lmm,
                            const int32_t* __restrict__ lmm_g, int32_t* __restrict__ rad_from, int32_t* __restrict__ n1,
                            int32_t* __restrict__ n2, int32_t* __restrict__ op, double* __restrict__ g) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += gridDim.x * blockDim.x) {
        const int idx = mix[i];
        const int a = lmm[p1[idx]], b = lmm_g[p2[idx]];
        const int o = base + i;
        n1[o] = a;
        n2[o] = b;
        g[o] = 0;
        op[o] = OP_SKIP;
        if (a < 0 || b < 0) continue;
        double ginv = 1.0;
        if (r_flag == 1) {
            double Re;
            if (jtype == 0) {
                Re = jres;
            } else {
                const double l1 = radii[n1c[idx]];
                const double jl1 = l1 + l1, jl2 = gt[n2g[idx]];  // CNT diameter, GNP thickness
                const double A = (jl1 - jl2 < kZero) ? jl1 * jl1 : jl2 * jl2;
                const double d = jd[idx];
                Re = C1 * d * exp(C2 * d) / A;
            }
            ginv = 1 / Re;
        }
        if (a >= reserved && b >= reserved) {
            op[o] = OP_OVERWRITE;
            g[o] = ginv;
        } else if (reserved > 2) {
            op[o] = OP_ADD;
            g[o] = ginv;
        }
        atomicMax(&rad_from[p2[idx]], i);
    }
}

__global__ void k_mix_radius(int nm, const int32_t* __restrict__ mix, const int32_t* __restrict__ n1c, const int32_t* __restrict__ p2,
                             const double* __restrict__ radii, const int32_t* __restrict__ rad_from, double* __restrict__ cnt_rad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += gridDim.x * blockDim.x) {
        const int idx = mix[i];
        if (rad_from[p2[idx]] == i) cnt_rad[p2[idx]] = radii[n1c[idx]];
    }
}

// Calculate_resistance_gnp (:1198-1232): rho L / (pi r1 r2), rho = u . (u_x rho_s, u_y rho_s, u_z rho_t).
__device__ __forceinline__ double gnp_resistance(const double* A, const double* B, double r1, double r2, double rs, double rt, bool& ok) {
    const double dx = A[0] - B[0], dy = A[1] - B[1], dz = A[2] - B[2];
    const double L = sqrt(dx * dx + dy * dy + dz * dz);
    ok = !(L < kZero);
    const double ux = (B[0] - A[0]) / L, uy = (B[1] - A[1]) / L, uz = (B[2] - A[2]) / L;
    const double rho = ux * rs * ux + uy * rs * uy + uz * rt * uz;
    return rho * L / (kPI * r1 * r2);
}

// Fill_2d_matrices_gnp (:1060-1133): each GNP's triangulation edges, last to first.
__global__ void k_gnp_tri_edges(int ng, int base, int r_flag, double rs, double rt, const int32_t* __restrict__ gnps,
                                const int32_t* __restrict__ off, const int32_t* __restrict__ tri, const int32_t* __restrict__ tri_cnt,
                                const double* __restrict__ pts, const double* __restrict__ gt, const int32_t* __restrict__ lmm_g,
                                const int32_t* __restrict__ rad_from, const double* __restrict__ cnt_rad, int32_t* __restrict__ n1,
                                int32_t* __restrict__ n2, int32_t* __restrict__ op, double* __restrict__ g, int* status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
        const int gi = gnps[i], m = tri_cnt[gi];
        const int32_t* e = tri + 2 * (size_t)kTriCap * gi;
        const double t2 = gt[gi] / 2;
        for (int j = m - 1; j >= 0; j--) {
            const int v1 = e[2 * j], v2 = e[2 * j + 1];
            const int o = base + off[i] + (m - 1 - j);
            const int a = lmm_g[v1], b = lmm_g[v2];
            n1[o] = a;
            n2[o] = b;
            op[o] = OP_OVERWRITE;
            g[o] = 1.0;
            if (a < 0 || b < 0) {  // LMM_gnps.at() of a point without a node
                atomicCAS(status, 0, (int)DEV_INPUT);
                op[o] = OP_SKIP;
                continue;
            }
            if (r_flag == 1) {
                const double r1 = rad_from[v1] >= 0 ? cnt_rad[v1] : t2;
                const double r2 = rad_from[v2] >= 0 ? cnt_rad[v2] : t2;
                bool ok;
                const double Re = gnp_resistance(pts + 3 * (size_t)v1, pts + 3 * (size_t)v2, r1, r2, rs, rt, ok);
                if (!ok) atomicCAS(status, 0, (int)DEV_INPUT);
                g[o] = 1 / Re;
            }
        }
    }
}

// Fill_2d_matrices_gnp_junctions (:1234-1319): a junction whose two points have nodes is a resistor.
__global__ void k_gnp_junction_edges(int nj, int base, int r_flag, int jtype, double jres, double C1, double C2,
                                     const int32_t* __restrict__ gj, const int32_t* __restrict__ p1, const int32_t* __restrict__ gn1,
                                     const int32_t* __restrict__ p2, const int32_t* __restrict__ gn2, const double* __restrict__ jd,
                                     const double* __restrict__ gt, const int32_t* __restrict__ lmm_g, int32_t* __restrict__ n1,
                                     int32_t* __restrict__ n2, int32_t* __restrict__ op, double* __restrict__ g) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nj; i += gridDim.x * blockDim.x) {
        const int idx = gj[i];
        const int a = lmm_g[p1[idx]], b = lmm_g[p2[idx]];
        const int o = base + i;
        n1[o] = a;
        n2[o] = b;
        g[o] = 0;
        op[o] = OP_SKIP;
        if (a < 0 || b < 0) continue;
        double ginv = 1.0;
        if (r_flag == 1) {
            double Re;
            if (jtype == 0) {
                Re = jres;
            } else {
                const double jl1 = gt[gn1[idx]], jl2 = gt[gn2[idx]];
                const double A = (jl1 - jl2 < kZero) ? jl1 * jl1 : jl2 * jl2;
                const double d = jd[idx];
                Re = C1 * d * exp(C2 * d) / A;
            }
            ginv = 1 / Re;
        }
        op[o] = OP_OVERWRITE;
        g[o] = ginv;
    }
}

// ---------------------------------------------------------------------------
// Backbone of a mixed cluster (Backbone_Network.cpp:64-245, 577-1127)

// Find_zero_current's GNP terms: triangulation edges, GNP-GNP and CNT-GNP junctions.
__global__ void k_current_max_gnp(int ng, const int32_t* __restrict__ gnps, const int32_t* __restrict__ tri,
                                  const int32_t* __restrict__ tri_cnt, int ngj, const int32_t* __restrict__ gj,
                                  const int32_t* __restrict__ jg_p1, const int32_t* __restrict__ jg_p2, int nmj, const int32_t* __restrict__ mix,
                                  const int32_t* __restrict__ jm_p1, const int32_t* __restrict__ jm_p2, const int32_t* __restrict__ lmm,
                                  const int32_t* __restrict__ lmm_g, const double* __restrict__ volt, unsigned long long* imax) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng + ngj + nmj; i += gridDim.x * blockDim.x) {
        double m = 0;
        if (i < ng) {
            const int g = gnps[i];
            const int32_t* e = tri + 2 * (size_t)kTriCap * g;
            for (int k = 0; k < tri_cnt[g]; k++) m = fmax(m, fabs(volt[lmm_g[e[2 * k]]] - volt[lmm_g[e[2 * k + 1]]]));
        } else if (i < ng + ngj) {
            const int idx = gj[i - ng];
            m = fabs(volt[lmm_g[jg_p1[idx]]] - volt[lmm_g[jg_p2[idx]]]);
        } else {
            const int idx = mix[i - ng - ngj];
            m = fabs(volt[lmm[jm_p1[idx]]] - volt[lmm_g[jm_p2[idx]]]);
        }
        atomic_max_pos(imax, m);
    }
}

// Find_and_remove_gnp_and_mixed_junctions_below_zero_current, CNT-GNP part (:662-735): the
// cluster's mixed junctions last to first.  A junction is removed when its current is below
// the zero current, its CNT is dead or its CNT point is no longer an element; its GNP point
// leaves the GNP's list and its CNT point the CNT's elements (a CNT left with fewer than two
// elements is dead).  Only junctions of the same CNT interact: one thread per CNT walks them
// (segments of the junctions sorted by CNT, positions descending).
__global__ void k_mix_below_zero(int nseg, const int32_t* __restrict__ seg_start, int nm, const uint32_t* __restrict__ order,
                                 const int32_t* __restrict__ mix, const int32_t* __restrict__ jm_p1, const int32_t* __restrict__ jm_n1,
                                 const int32_t* __restrict__ jm_p2, const int32_t* __restrict__ lmm, const int32_t* __restrict__ lmm_g,
                                 const double* __restrict__ volt, const unsigned long long* __restrict__ imax_bits,
                                 const int32_t* __restrict__ elem_pos, int32_t* __restrict__ cur_lo, int32_t* __restrict__ cur_hi,
                                 int32_t* __restrict__ elem_removed, int32_t* __restrict__ removed_cnt, int32_t* __restrict__ mix_alive,
                                 int32_t* __restrict__ pt_removed) {
    const double i_max = fmax(__longlong_as_double((long long)*imax_bits), kZero);
    const double zero_current = i_max * 1e-9;
    for (int sg = blockIdx.x * blockDim.x + threadIdx.x; sg < nseg; sg += gridDim.x * blockDim.x) {
        const int b = seg_start[sg], e = sg + 1 < nseg ? seg_start[sg + 1] : nm;
        for (int k = b; k < e; k++) {
            const int i = (int)order[k];
            const int idx = mix[i];
            const int P1 = jm_p1[idx], c = jm_n1[idx], P2 = jm_p2[idx];
            const double Ij = fabs(volt[lmm[P1]] - volt[lmm_g[P2]]);
            const int lo = cur_lo[c], hi = cur_hi[c];
            const bool empty = lo < 0;
            const int q = elem_pos[P1];
            const bool in_elem = !empty && q >= lo && q <= hi && !elem_removed[q];
            if (Ij - zero_current < kZero || empty || !in_elem) {
                mix_alive[i] = 0;
                pt_removed[P2] = 1;
                if (in_elem) {
                    elem_removed[q] = 1;
                    removed_cnt[c]++;
                    if ((hi - lo + 1) - removed_cnt[c] < 2) {  // the CNT's elements are cleared
                        cur_lo[c] = -1;
                        cur_hi[c] = -2;
                    }
                }
            }
        }
    }
}

// GNP-GNP part (:737-790): a junction below the zero current is removed with both its points.
__global__ void k_gj_below_zero(int nj, const int32_t* __restrict__ gj, const int32_t* __restrict__ jg_p1, const int32_t* __restrict__ jg_p2,
                                const int32_t* __restrict__ lmm_g, const double* __restrict__ volt, const unsigned long long* __restrict__ imax_bits,
                                int32_t* __restrict__ gj_alive, int32_t* __restrict__ pt_removed) {
    const double i_max = fmax(__longlong_as_double((long long)*imax_bits), kZero);
    const double zero_current = i_max * 1e-9;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nj; i += gridDim.x * blockDim.x) {
        const int idx = gj[i];
        const int P1 = jg_p1[idx], P2 = jg_p2[idx];
        if (fabs(volt[lmm_g[P1]] - volt[lmm_g[P2]]) - zero_current < kZero) {
            gj_alive[i] = 0;
            pt_removed[P1] = 1;
            pt_removed[P2] = 1;
        }
    }
}

// Remove_point_from_vector for every removed point (:1041-1055): each GNP's list keeps its
// other points in order, at the front.
__global__ void k_gnp_compact(int ng, const int32_t* __restrict__ gnps, const int32_t* __restrict__ sptr, int32_t* __restrict__ sidx,
                              int32_t* __restrict__ scount, const int32_t* __restrict__ pt_removed) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
        const int g = gnps[i], b = sptr[g];
        int k = 0;
        for (int m = 0; m < scount[g]; m++) {
            const int P = sidx[b + m];
            if (!pt_removed[P]) sidx[b + k++] = P;
        }
        scount[g] = k;
    }
}

// Clear_structure_of_dead_gnps (:792-853): a GNP with no points, one junction and no boundary
// point, or only boundary points is dead; its list is cleared.  Each cleared list and each
// dead GNP with one junction asks for another removal round (to_remove).
__global__ void k_gnp_clear_dead(int ng, const int32_t* __restrict__ gnps, const int32_t* __restrict__ sptr,
                                 const int32_t* __restrict__ sidx, int32_t* __restrict__ scount, const int32_t* __restrict__ nb,
                                 int32_t* __restrict__ pt_removed, int32_t* __restrict__ to_remove, int* status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) {
        const int g = gnps[i];
        const int NT = scount[g], NB = nb[g], NJ = NT - NB;
        if (NT == 0 || (NB == 0 && NJ == 1) || NB == NT) {
            if (NT > 0) {
                for (int m = 0; m < NT; m++) pt_removed[sidx[sptr[g] + m]] = 1;
                scount[g] = 0;
                atomicAdd(to_remove, 1);
            }
            if (NJ == 1) atomicAdd(to_remove, 1);
        } else if (NT < 2) {
            atomicCAS(status, 0, (int)DEV_INPUT);  // "There should be at least two points"
        }
    }
}

// One round of Remove_junctions_with_dead_particles_gnps and _mixed (:994-1127), the lists
// last to first.  A junction removed here can empty a GNP's list that a later junction of the
// same round reads, so one thread runs the round in upstream's order; `live` counts each
// GNP's points during the round (the lists are compacted after it).
__global__ void k_dead_junction_round(int ngj, const int32_t* __restrict__ gj, const int32_t* __restrict__ jg_p1,
                                      const int32_t* __restrict__ jg_n1, const int32_t* __restrict__ jg_p2, const int32_t* __restrict__ jg_n2,
                                      int32_t* __restrict__ gj_alive, int nmj, const int32_t* __restrict__ mix, const int32_t* __restrict__ jm_p1,
                                      const int32_t* __restrict__ jm_n1, const int32_t* __restrict__ jm_p2, const int32_t* __restrict__ jm_n2,
                                      int32_t* __restrict__ mix_alive, const int32_t* __restrict__ cur_lo, const int32_t* __restrict__ cur_hi,
                                      const int32_t* __restrict__ elem_pos, const int32_t* __restrict__ elem_removed,
                                      int32_t* __restrict__ live, int32_t* __restrict__ pt_removed) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    auto remove = [&](int P, int g) {
        if (live[g] > 0 && !pt_removed[P]) {
            pt_removed[P] = 1;
            live[g]--;
        }
    };
    for (int i = ngj - 1; i >= 0; i--) {
        if (!gj_alive[i]) continue;
        const int idx = gj[i];
        const int g1 = jg_n1[idx], g2 = jg_n2[idx];
        if (live[g1] == 0 || live[g2] == 0) {
            gj_alive[i] = 0;
            remove(jg_p1[idx], g1);
            remove(jg_p2[idx], g2);
        }
    }
    for (int i = nmj - 1; i >= 0; i--) {
        if (!mix_alive[i]) continue;
        const int idx = mix[i];
        const int c = jm_n1[idx], g2 = jm_n2[idx], P1 = jm_p1[idx];
        const int lo = cur_lo[c], hi = cur_hi[c];
        if (lo < 0 || live[g2] == 0) {
            mix_alive[i] = 0;
            remove(jm_p2[idx], g2);
        } else {
            const int q = elem_pos[P1];
            if (!(q >= lo && q <= hi && !elem_removed[q])) {
                mix_alive[i] = 0;
                remove(jm_p2[idx], g2);
            }
        }
    }
}

// Calculate_gnp_backbone_volume (:882-948): GNP volumes to the family's backbone or dead
// total in cluster order (one thread: the same sequence of FP64 additions); the
// triangulations of the cluster are cleared.
__global__ void k_gnp_volume_sum(int ng, int family, const int32_t* __restrict__ gnps, const int32_t* __restrict__ scount,
                                 const double* __restrict__ vol, int32_t* __restrict__ tri_cnt, double* acc) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double live = acc[HV_GNP + family], dead = acc[HV_DEAD_GNP + family];
    for (int i = 0; i < ng; i++) {
        const int g = gnps[i];
        if (scount[g] > 0) live = live + vol[g];
        else dead = dead + vol[g];
        tri_cnt[g] = 0;
    }
    acc[HV_GNP + family] = live;
    acc[HV_DEAD_GNP + family] = dead;
}

// The CNT elements after the backbone: kept range of each CNT minus the points the mixed
// junctions took out (marks over points, then the usual scan and fill).
__global__ void k_mark_kept_elements(int n_elem, const int32_t* __restrict__ elem, const int32_t* __restrict__ flag,
                                     const int32_t* __restrict__ cur_lo, const int32_t* __restrict__ cur_hi,
                                     const int32_t* __restrict__ elem_removed, int32_t* __restrict__ mark) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_elem; q += gridDim.x * blockDim.x) {
        const int P = elem[q], c = flag[P];
        mark[P] = (cur_lo[c] >= 0 && q >= cur_lo[c] && q <= cur_hi[c] && !elem_removed[q]) ? 1 : 0;
    }
}

__global__ void k_fill_marked(int np, const int32_t* __restrict__ mark, const int32_t* __restrict__ scan, int32_t* __restrict__ elem) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x)
        if (mark[i]) elem[scan[i]] = i;
}

__global__ void k_cnt_has_elements(int n, const int32_t* __restrict__ members, const int32_t* __restrict__ cur_lo, int32_t* __restrict__ alive) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) alive[i] = cur_lo[members[i]] >= 0 ? 1 : 0;
}

__global__ void k_clear_tri(int ng, const int32_t* __restrict__ gnps, int32_t* __restrict__ tri_cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ng; i += gridDim.x * blockDim.x) tri_cnt[gnps[i]] = 0;
}

// Currents_through_boundary_gnps (Electrical_analysis.cpp:607-675): the edges of each GNP on
// the face (list order) with a node on a prescribed face; the terms are added in that order
// by k_boundary_sum.
__global__ void k_gnp_boundary_terms(int nb, const int32_t* __restrict__ face, const int32_t* __restrict__ off, int node,
                                     const int32_t* __restrict__ tri, const int32_t* __restrict__ tri_cnt, const int32_t* __restrict__ lmm_g,
                                     const int32_t* __restrict__ rad_from, const double* __restrict__ cnt_rad, const double* __restrict__ gt,
                                     const double* __restrict__ pts, const double* __restrict__ volt, double rs, double rt,
                                     double* __restrict__ term, int32_t* __restrict__ valid, int* status) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
        const int g = face[k], m = tri_cnt[g];
        const int32_t* e = tri + 2 * (size_t)kTriCap * g;
        for (int j = 0; j < m; j++) {
            const int o = off[k] + j;
            const int v1 = e[2 * j], v2 = e[2 * j + 1];
            const int nA = lmm_g[v1], nB = lmm_g[v2];
            term[o] = 0;
            valid[o] = 0;
            if (nA < 0 || nB < 0) {
                atomicCAS(status, 0, (int)DEV_INPUT);
                continue;
            }
            if (nA <= 1 || nB <= 1) {
                if (nA == nB) {  // "nodes are at the same boundary"
                    atomicCAS(status, 0, (int)DEV_INPUT);
                    continue;
                }
                const int n1 = (nA == node) ? nA : nB, n2 = (nA == node) ? nB : nA;
                const double t2 = gt[g] / 2;
                const double r1 = rad_from[v1] >= 0 ? cnt_rad[v1] : t2;
                const double r2 = rad_from[v2] >= 0 ? cnt_rad[v2] : t2;
                const double V = volt[n2] - volt[n1];
                bool ok;
                const double Re = gnp_resistance(pts + 3 * (size_t)v1, pts + 3 * (size_t)v2, r1, r2, rs, rt, ok);
                term[o] = V / Re;
                valid[o] = 1;
            }
        }
    }
}

__global__ void k_face_tri_counts(int nb, const int32_t* __restrict__ face, const int32_t* __restrict__ tri_cnt, int32_t* __restrict__ cnt) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) cnt[k] = tri_cnt[face[k]];
}

__global__ void k_fill_value_i32(int n, int32_t v, int32_t* __restrict__ a) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = v;
}

// key (CNT, descending list position) of each mixed junction, for k_mix_below_zero
__global__ void k_mix_keys(int nm, const int32_t* __restrict__ mix, const int32_t* __restrict__ jm_n1, uint64_t* __restrict__ key,
                           uint32_t* __restrict__ val) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += gridDim.x * blockDim.x) {
        key[i] = ((uint64_t)(uint32_t)jm_n1[mix[i]] << 32) | (uint32_t)(nm - 1 - i);
        val[i] = (uint32_t)i;
    }
}

__global__ void k_key_heads(int n, const uint64_t* __restrict__ key, int32_t* __restrict__ head) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        head[i] = (i == 0 || (key[i] >> 32) != (key[i - 1] >> 32)) ? 1 : 0;
}

__global__ void k_head_positions(int n, const int32_t* __restrict__ head, const int32_t* __restrict__ scan, int32_t* __restrict__ start) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (head[i]) start[scan[i]] = i;
}

template <class T>
void upload(Ctx& c, DBuf<T>& d, const T* h, size_t n) {
    d.ensure(std::max<size_t>(n, 1));
    if (n) CICY_CUDA(cudaMemcpyAsync(d.get(), h, sizeof(T) * n, cudaMemcpyHostToDevice, c.stream));
}

// Compact `list` (n entries) by the 0/1 flags in `alive`; returns the kept count.
int compact_list(Ctx& c, int32_t* list, int n, DBuf<int32_t>& alive, DBuf<int32_t>& scan, DBuf<int32_t>& tmp) {
    if (n <= 0) return 0;
    cudaStream_t s = c.stream;
    scan.ensure(n + 1);
    tmp.ensure(n + 1);
    exclusive_scan_i32(alive.get(), scan.get(), n, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
    k_compact_i32<<<grid_for(n), 256, 0, s>>>(n, list, alive.get(), scan.get(), tmp.get());
    c.launches++;
    const int k = read_i32(c, c.i32_scalar.get());
    if (k) CICY_CUDA(cudaMemcpyAsync(list, tmp.get(), sizeof(int32_t) * k, cudaMemcpyDeviceToDevice, s));
    return k;
}

}  // namespace

// ---------------------------------------------------------------------------
// hooks of solve_dea (declared beside it, in the same unnamed namespace)

namespace {

int gnp_lmm(Ctx& c, const GnpPass& gp, const int* bnd, int nbnd, int first_node) {
    HybridDev& H = *gp.hy;
    cudaStream_t s = c.stream;
    H.lmm_g.ensure(std::max(H.n_pts, 1));
    k_fill_value_i32<<<grid_for(H.n_pts), 256, 0, s>>>(H.n_pts, -1, H.lmm_g.get());
    c.launches++;
    for (int k = 0; k < nbnd; k++) {  // Map_points_at_boundaries (:217-246)
        const int f = bnd[k];
        const int b = H.h_bgp_ptr[f], e = H.h_bgp_ptr[f + 1];
        if (e > b) {
            k_lmm_face<<<grid_for(e - b), 256, 0, s>>>(b, e, H.bgp_idx.get(), k, H.lmm_g.get());
            c.launches++;
        }
    }
    if (gp.n_gnps == 0) return 0;
    H.gcnt.ensure(gp.n_gnps + 1);
    H.goff.ensure(gp.n_gnps + 1);
    k_gnp_node_counts<<<grid_for(gp.n_gnps), 256, 0, s>>>(gp.n_gnps, gp.gnps, H.sptr.get(), H.sidx.get(), H.scount.get(), H.lmm_g.get(),
                                                        H.gcnt.get());
    exclusive_scan_i32(H.gcnt.get(), H.goff.get(), gp.n_gnps, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
    k_gnp_node_assign<<<grid_for(gp.n_gnps), 256, 0, s>>>(gp.n_gnps, first_node, gp.gnps, H.sptr.get(), H.sidx.get(), H.scount.get(),
                                                        H.goff.get(), H.lmm_g.get());
    c.launches += 2;
    return read_i32(c, c.i32_scalar.get());
}

int gnp_prepare_edges(Ctx& c, const GnpPass& gp, int r_flag) {
    HybridDev& H = *gp.hy;
    cudaStream_t s = c.stream;
    int n_tri = 0;
    if (gp.n_gnps > 0) {
        H.tri_work.ensure(sizeof(gnp::TriWork<kTriMaxPoints>) * (size_t)gp.n_gnps);
        k_gnp_triangulate<<<grid_for(gp.n_gnps, 64), 64, 0, s>>>(gp.n_gnps, r_flag ? 0 : 1, gp.gnps, H.pts.get(), H.sptr.get(), H.sidx.get(),
                                                                 H.scount.get(), H.geom.get(),
                                                                 reinterpret_cast<gnp::TriWork<kTriMaxPoints>*>(H.tri_work.get()), H.tri.get(),
                                                                 H.tri_cnt.get(), c.status.get());
        k_gnp_tri_counts<<<grid_for(gp.n_gnps), 256, 0, s>>>(gp.n_gnps, gp.gnps, H.tri_cnt.get(), H.gcnt.get());
        exclusive_scan_i32(H.gcnt.get(), H.goff.get(), gp.n_gnps, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
        c.launches += 2;
        CICY_LAUNCH_CHECK();
        check_status(c, "Fill_2d_matrices_gnp (Generate_3d_trangulation)");
        n_tri = read_i32(c, c.i32_scalar.get());
    }
    H.n_tri_pass = n_tri;
    return gp.n_mix + n_tri + gp.n_gj;
}

void gnp_fill_edges(Ctx& c, const GnpPass& gp, int base, int r_flag, int reserved, const cicy_params& p) {
    HybridDev& H = *gp.hy;
    cudaStream_t s = c.stream;
    H.rad_from.ensure(std::max(H.n_pts, 1));
    H.cnt_rad.ensure(std::max(H.n_pts, 1));
    k_fill_value_i32<<<grid_for(H.n_pts), 256, 0, s>>>(H.n_pts, -1, H.rad_from.get());
    c.launches++;
    if (gp.n_mix > 0) {
        k_mix_edges<<<grid_for(gp.n_mix), 256, 0, s>>>(gp.n_mix, base, r_flag, reserved, p.junction_type, p.junction_resistance, p.C1, p.C2,
                                                     gp.mix, H.jm_p1.get(), H.jm_n1.get(), H.jm_p2.get(), H.jm_n2.get(), H.jm_d.get(),
                                                     c.radii.get(), H.t.get(), c.lmm.get(), H.lmm_g.get(), H.rad_from.get(), c.e_n1.get(),
                                                     c.e_n2.get(), c.e_op.get(), c.e_g.get());
        k_mix_radius<<<grid_for(gp.n_mix), 256, 0, s>>>(gp.n_mix, gp.mix, H.jm_n1.get(), H.jm_p2.get(), c.radii.get(), H.rad_from.get(),
                                                      H.cnt_rad.get());
        c.launches += 2;
    }
    const int n_tri = H.n_tri_pass;
    if (gp.n_gnps > 0) {
        k_gnp_tri_edges<<<grid_for(gp.n_gnps, 64), 64, 0, s>>>(gp.n_gnps, base + gp.n_mix, r_flag, H.rs, H.rt, gp.gnps, H.goff.get(),
                                                             H.tri.get(), H.tri_cnt.get(), H.pts.get(), H.t.get(), H.lmm_g.get(),
                                                             H.rad_from.get(), H.cnt_rad.get(), c.e_n1.get(), c.e_n2.get(), c.e_op.get(),
                                                             c.e_g.get(), c.status.get());
        c.launches++;
    }
    if (gp.n_gj > 0) {
        k_gnp_junction_edges<<<grid_for(gp.n_gj), 256, 0, s>>>(gp.n_gj, base + gp.n_mix + n_tri, r_flag, p.junction_type, p.junction_resistance,
                                                             p.C1, p.C2, gp.gj, H.jg_p1.get(), H.jg_n1.get(), H.jg_p2.get(), H.jg_n2.get(),
                                                             H.jg_d.get(), H.t.get(), H.lmm_g.get(), c.e_n1.get(), c.e_n2.get(), c.e_op.get(),
                                                             c.e_g.get());
        c.launches++;
    }
    CICY_LAUNCH_CHECK();
    check_status(c, "Fill_2d_matrices_gnp");
}

}  // namespace


// ---------------------------------------------------------------------------
// Perform_analysis_on_clusters for GNP_CNT_mix (Electrical_analysis.cpp:10-145)

namespace {

// Host checks of the caller's mixed-network state: every index a kernel uses as an address
// is in range before anything is uploaded.
void check_hybrid_state(const Ctx& c, const cicy_hybrid_state& h) {
    auto bad = [](const std::string& m) { throw Fail{CICY_E_INPUT, "cicy_hybrid_electrical: " + m}; };
    auto csr = [&](const int64_t* ptr, const int32_t* idx, int rows, int64_t limit, const char* what) {
        if (rows > 0 && !ptr) bad(std::string(what) + " missing");
        for (int r = 0; r < rows; r++) {
            if (ptr[r + 1] < ptr[r] || (r == 0 && ptr[0] != 0)) bad(std::string(what) + ": offsets are not 0 .. n non-decreasing");
            for (int64_t k = ptr[r]; k < ptr[r + 1]; k++)
                if (idx[k] < 0 || idx[k] >= limit) bad(std::string(what) + ": index out of range");
        }
    };
    const int NC = h.n_clusters;
    if (NC < 0 || h.n_gnps < 0 || h.n_points_gnp < 0 || h.n_junctions_cnt < 0 || h.n_junctions_gnp < 0 || h.n_junctions_mixed < 0)
        bad("negative sizes");
    if (h.n_points_gnp >= (1LL << 31) - 1 || h.n_junctions_mixed >= (1LL << 31) - 1 || h.n_junctions_gnp >= (1LL << 31) - 1)
        throw Fail{CICY_E_CAPACITY, "cicy_hybrid_electrical: 2^31 or more GNP points or junctions"};
    if (NC > 0 && !h.family) bad("family missing");
    for (int j = 0; j < NC; j++)
        if (h.family[j] < 0 || h.family[j] > 6) bad("invalid family");
    csr(h.clusters_cnt_ptr, h.clusters_cnt_idx, NC, c.n_cnts, "clusters_cnt");
    csr(h.clusters_gnp_ptr, h.clusters_gnp_idx, NC, h.n_gnps, "clusters_gnp");
    csr(h.cnt_junctions_ptr, h.cnt_junctions_idx, NC, h.n_junctions_cnt, "cluster_cnt_junctions");
    csr(h.gnp_junctions_ptr, h.gnp_junctions_idx, NC, h.n_junctions_gnp, "cluster_gnp_junctions");
    csr(h.mix_junctions_ptr, h.mix_junctions_idx, NC, h.n_junctions_mixed, "cluster_mix_junctions");
    for (int64_t k = 0; k < h.n_junctions_cnt; k++)
        if (h.jc_p1[k] < 0 || h.jc_p1[k] >= c.n_points || h.jc_p2[k] < 0 || h.jc_p2[k] >= c.n_points || h.jc_n1[k] < 0 ||
            h.jc_n1[k] >= c.n_cnts || h.jc_n2[k] < 0 || h.jc_n2[k] >= c.n_cnts)
            bad("CNT junction out of range");
    for (int64_t k = 0; k < h.n_junctions_gnp; k++)
        if (h.jg_p1[k] < 0 || h.jg_p1[k] >= h.n_points_gnp || h.jg_p2[k] < 0 || h.jg_p2[k] >= h.n_points_gnp || h.jg_n1[k] < 0 ||
            h.jg_n1[k] >= h.n_gnps || h.jg_n2[k] < 0 || h.jg_n2[k] >= h.n_gnps)
            bad("GNP junction out of range");
    for (int64_t k = 0; k < h.n_junctions_mixed; k++)
        if (h.jm_p1[k] < 0 || h.jm_p1[k] >= c.n_points || h.jm_p2[k] < 0 || h.jm_p2[k] >= h.n_points_gnp || h.jm_n1[k] < 0 ||
            h.jm_n1[k] >= c.n_cnts || h.jm_n2[k] < 0 || h.jm_n2[k] >= h.n_gnps)
            bad("mixed junction out of range");
    if (!h.elements_ptr || h.elements_ptr[0] != 0) bad("elements_cnt missing");
    for (int cn = 0; cn < c.n_cnts; cn++) {
        const int b = c.h_cstart[cn], e = b + c.h_clen[cn];
        for (int64_t k = h.elements_ptr[cn]; k < h.elements_ptr[cn + 1]; k++)
            if (h.elements_idx[k] < b || h.elements_idx[k] >= e || (k > h.elements_ptr[cn] && h.elements_idx[k] <= h.elements_idx[k - 1]))
                bad("elements_cnt: a point outside its CNT or not ascending");
    }
    if (h.n_gnps > 0 && (!h.structure_gnp_ptr || !h.points_gnp || !h.gnp_t || !h.gnp_volume || !h.gnp_frame || !h.pts_boundary_count))
        bad("GNP arrays missing");
    std::vector<char> seen(std::max<int64_t>(h.n_points_gnp, 1), 0);
    for (int g = 0; g < h.n_gnps; g++) {
        if (h.structure_gnp_ptr[g + 1] < h.structure_gnp_ptr[g] || (g == 0 && h.structure_gnp_ptr[0] != 0)) bad("structure_gnp offsets");
        for (int64_t k = h.structure_gnp_ptr[g]; k < h.structure_gnp_ptr[g + 1]; k++) {
            const int64_t P = h.structure_gnp_idx[k];
            if (P < 0 || P >= h.n_points_gnp || seen[P]) bad("structure_gnp: a point out of range or listed twice");
            seen[P] = 1;
        }
    }
    for (int f = 0; f < 6; f++) {
        if (!h.boundary_gnp_ptr || !h.boundary_gnp_pts_ptr) bad("GNP face lists missing");
        for (int64_t k = h.boundary_gnp_ptr[f]; k < h.boundary_gnp_ptr[f + 1]; k++)
            if (h.boundary_gnp_idx[k] < 0 || h.boundary_gnp_idx[k] >= h.n_gnps) bad("boundary_gnp out of range");
        for (int64_t k = h.boundary_gnp_pts_ptr[f]; k < h.boundary_gnp_pts_ptr[f + 1]; k++)
            if (h.boundary_gnp_pts_idx[k] < 0 || h.boundary_gnp_pts_idx[k] >= h.n_points_gnp) bad("boundary_gnp_pts out of range");
    }
}

}  // namespace

void run_hybrid_electrical(Ctx& c, const cicy_hybrid_state& h, const cicy_params& p, double rho_gnp_surf, double rho_gnp_t,
                           cicy_result* out) {
    if (c.stage < 1) throw Fail{CICY_E_STATE, "cicy_hybrid_electrical: no network uploaded"};
    if (p.simulation_scope != 0) throw Fail{CICY_E_INPUT, "cicy_hybrid_electrical: simulation_scope 0 only"};
    check_hybrid_state(c, h);
    cudaStream_t s = c.stream;
    if (!c.hy) c.hy = new HybridDev;
    HybridDev& H = *c.hy;
    c.have_hybrid = false;
    c.have_volumes = false;
    for (auto* sy : c.systems) c.sys_pool.push_back(sy);
    c.systems.clear();
    H.rs = rho_gnp_surf;
    H.rt = rho_gnp_t;
    const int NC = h.n_clusters, NG = h.n_gnps, NPG = (int)h.n_points_gnp, NP = std::max(c.n_points, 1);
    H.n_gnps = NG;
    H.n_pts = NPG;
    H.n_clusters = NC;
    // ---- CNT elements (elements_cnt): marks over points, positions, kept ranges ----
    std::vector<int32_t> mark(NP + 1, 0);
    for (int64_t k = 0; k < h.elements_ptr[c.n_cnts]; k++) mark[h.elements_idx[k]] = 1;
    c.mark.ensure(NP + 1);
    c.mark_scan.ensure(NP + 1);
    upload(c, c.mark, mark.data(), (size_t)NP + 1);
    exclusive_scan_i32(c.mark.get(), c.mark_scan.get(), c.n_points + 1, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
    int n_elem = (int)h.elements_ptr[c.n_cnts];
    c.elem_idx.ensure(std::max(n_elem, 1));
    k_fill_marked<<<grid_for(c.n_points), 256, 0, s>>>(c.n_points, c.mark.get(), c.mark_scan.get(), c.elem_idx.get());
    const int NCNT = std::max(c.n_cnts, 1);
    c.bb_lo.ensure(NCNT);
    c.bb_hi.ensure(NCNT);
    k_init_ranges<<<grid_for(NCNT), 256, 0, s>>>(c.n_cnts, c.cstart.get(), c.clen.get(), c.mark_scan.get(), c.bb_lo.get(), c.bb_hi.get());
    c.launches += 2;
    // ---- junctions ----
    auto i32v = [](const int64_t* a, int64_t n) { return std::vector<int32_t>(a, a + n); };
    const int NJC = (int)h.n_junctions_cnt;
    c.n_junc = NJC;
    {
        std::vector<int32_t> a = i32v(h.jc_p1, NJC), b = i32v(h.jc_p2, NJC);
        upload(c, c.j_p1, a.data(), NJC);
        upload(c, c.j_p2, b.data(), NJC);
        upload(c, c.j_n1, h.jc_n1, NJC);
        upload(c, c.j_n2, h.jc_n2, NJC);
        upload(c, c.j_d, h.jc_dist, NJC);
        H.n_jg = (int)h.n_junctions_gnp;
        a = i32v(h.jg_p1, H.n_jg);
        b = i32v(h.jg_p2, H.n_jg);
        upload(c, H.jg_p1, a.data(), H.n_jg);
        upload(c, H.jg_p2, b.data(), H.n_jg);
        upload(c, H.jg_n1, h.jg_n1, H.n_jg);
        upload(c, H.jg_n2, h.jg_n2, H.n_jg);
        upload(c, H.jg_d, h.jg_dist, H.n_jg);
        H.n_jm = (int)h.n_junctions_mixed;
        a = i32v(h.jm_p1, H.n_jm);
        b = i32v(h.jm_p2, H.n_jm);
        upload(c, H.jm_p1, a.data(), H.n_jm);
        upload(c, H.jm_p2, b.data(), H.n_jm);
        upload(c, H.jm_n1, h.jm_n1, H.n_jm);
        upload(c, H.jm_n2, h.jm_n2, H.n_jm);
        upload(c, H.jm_d, h.jm_dist, H.n_jm);
        CICY_CUDA(cudaStreamSynchronize(s));  // the host vectors above go out of scope
    }
    // ---- clusters and their junction lists (working copies the backbone shrinks) ----
    auto flat = [&](const int64_t* ptr, const int32_t* idx, std::vector<int32_t>& hptr, DBuf<int32_t>& d) {
        hptr.assign(NC + 1, 0);
        for (int j = 0; j <= NC; j++) hptr[j] = (int32_t)ptr[j];
        upload(c, d, idx, (size_t)hptr[NC]);
    };
    flat(h.clusters_cnt_ptr, h.clusters_cnt_idx, c.h_clu_ptr, c.bbclu_idx);
    flat(h.cnt_junctions_ptr, h.cnt_junctions_idx, c.h_cj_ptr, c.bbcj_idx);
    flat(h.clusters_gnp_ptr, h.clusters_gnp_idx, H.h_cg_ptr, H.cg_idx);
    flat(h.gnp_junctions_ptr, h.gnp_junctions_idx, H.h_cgj_ptr, H.cgj_idx);
    flat(h.mix_junctions_ptr, h.mix_junctions_idx, H.h_cmj_ptr, H.cmj_idx);
    // the percolation-stage copies the cluster getters read (cicy_get_clusters, which = 0)
    c.clu_idx.ensure(std::max(c.h_clu_ptr[NC], 1));
    c.cj_idx.ensure(std::max(c.h_cj_ptr[NC], 1));
    if (c.h_clu_ptr[NC])
        CICY_CUDA(cudaMemcpyAsync(c.clu_idx.get(), c.bbclu_idx.get(), sizeof(int32_t) * c.h_clu_ptr[NC], cudaMemcpyDeviceToDevice, s));
    if (c.h_cj_ptr[NC])
        CICY_CUDA(cudaMemcpyAsync(c.cj_idx.get(), c.bbcj_idx.get(), sizeof(int32_t) * c.h_cj_ptr[NC], cudaMemcpyDeviceToDevice, s));
    c.h_family.assign(h.family, h.family + NC);
    c.n_perc = NC;
    // ---- GNPs ----
    upload(c, H.pts, h.points_gnp, 3 * (size_t)NPG);
    {
        std::vector<int32_t> sp(NG + 1), sx((size_t)(NG ? h.structure_gnp_ptr[NG] : 0)), sc(NG);
        for (int g = 0; g <= NG; g++) sp[g] = NG ? (int32_t)h.structure_gnp_ptr[g] : 0;
        for (size_t k = 0; k < sx.size(); k++) sx[k] = (int32_t)h.structure_gnp_idx[k];
        for (int g = 0; g < NG; g++) sc[g] = sp[g + 1] - sp[g];
        upload(c, H.sptr, sp.data(), sp.size());
        upload(c, H.sidx, sx.data(), sx.size());
        upload(c, H.scount, sc.data(), sc.size());
        std::vector<int32_t> bgp(h.boundary_gnp_pts_ptr[6]);
        for (size_t k = 0; k < bgp.size(); k++) bgp[k] = (int32_t)h.boundary_gnp_pts_idx[k];
        upload(c, H.bgp_idx, bgp.data(), bgp.size());
        CICY_CUDA(cudaStreamSynchronize(s));
    }
    H.h_bg_ptr.assign(7, 0);
    H.h_bgp_ptr.assign(7, 0);
    for (int f = 0; f <= 6; f++) {
        H.h_bg_ptr[f] = (int32_t)h.boundary_gnp_ptr[f];
        H.h_bgp_ptr[f] = (int32_t)h.boundary_gnp_pts_ptr[f];
    }
    upload(c, H.bg_idx, h.boundary_gnp_idx, (size_t)H.h_bg_ptr[6]);
    upload(c, H.nb, h.pts_boundary_count, NG);
    upload(c, H.t, h.gnp_t, NG);
    upload(c, H.vol, h.gnp_volume, NG);
    upload(c, H.geom, h.gnp_frame, 16 * (size_t)NG);
    H.tri.ensure(2 * (size_t)kTriCap * std::max(NG, 1));
    H.tri_cnt.ensure(std::max(NG, 1));
    H.pt_removed.ensure(std::max(NPG, 1));
    H.live.ensure(std::max(NG, 1));
    CICY_CUDA(cudaMemsetAsync(H.tri_cnt.get(), 0, sizeof(int32_t) * std::max(NG, 1), s));  // Clear_triangulations (:155-170)
    CICY_CUDA(cudaMemsetAsync(H.pt_removed.get(), 0, sizeof(int32_t) * std::max(NPG, 1), s));
    H.vol_acc.ensure(HV_WORDS);
    CICY_CUDA(cudaMemsetAsync(H.vol_acc.get(), 0, sizeof(double) * HV_WORDS, s));
    c.vol_acc.ensure(kVolWords);
    CICY_CUDA(cudaMemsetAsync(c.vol_acc.get(), 0, sizeof(double) * kVolWords, s));
    std::vector<int32_t> clu_len(NC), cj_len(NC);
    H.cgj_len.assign(NC, 0);
    H.cmj_len.assign(NC, 0);
    for (int j = 0; j < NC; j++) {
        clu_len[j] = c.h_clu_ptr[j + 1] - c.h_clu_ptr[j];
        cj_len[j] = c.h_cj_ptr[j + 1] - c.h_cj_ptr[j];
        H.cgj_len[j] = H.h_cgj_ptr[j + 1] - H.h_cgj_ptr[j];
        H.cmj_len[j] = H.h_cmj_ptr[j + 1] - H.h_cmj_ptr[j];
    }
    std::vector<std::vector<double> > parallel(3);
    double t_unit = 0, t_bb = 0, t_real = 0;
    DBuf<int32_t>& eb = c.eb;
    DBuf<int32_t>& ee = c.ee;
    c.imax.ensure(1);
    c.cur_out.ensure(4);
    const int maxl = std::max({c.h_clu_ptr[NC], c.h_cj_ptr[NC], H.h_cgj_ptr[NC], H.h_cmj_ptr[NC], 1}) + 1;
    c.alive.ensure(maxl);
    c.alive_scan.ensure(maxl);
    c.tmp_list.ensure(maxl);
    for (int j = 0; j < NC; j++) {
        int32_t* members = c.bbclu_idx.get() + c.h_clu_ptr[j];
        int32_t* jl = c.bbcj_idx.get() + c.h_cj_ptr[j];
        const int ng = H.h_cg_ptr[j + 1] - H.h_cg_ptr[j];
        const int32_t* gl = H.cg_idx.get() + H.h_cg_ptr[j];
        int32_t* gjl = H.cgj_idx.get() + H.h_cgj_ptr[j];
        int32_t* mxl = H.cmj_idx.get() + H.h_cmj_ptr[j];
        const int fam = c.h_family[j];
        GnpPass gu{&H, gl, ng, mxl, H.cmj_len[j], gjl, H.cgj_len[j]};
        SolveInput u{j, -1, fam, members, clu_len[j], jl, cj_len[j], &gu};
        DeaSystem* su = solve_dea(c, p, u, eb, ee);
        c.systems.push_back(su);
        t_unit += su->seconds;
        // ---- backbone (Backbone_Network::Determine_backbone_network, :11-62) ----
        cudaEvent_t e0, e1;
        CICY_CUDA(cudaEventCreate(&e0));
        CICY_CUDA(cudaEventCreate(&e1));
        CICY_CUDA(cudaEventRecord(e0, s));
        int NM = clu_len[j];
        const int NJ = cj_len[j], ngj = H.cgj_len[j], nmj = H.cmj_len[j];
        CICY_CUDA(cudaMemsetAsync(c.imax.get(), 0, sizeof(unsigned long long), s));
        k_current_max<<<grid_for(NM + NJ), 256, 0, s>>>(NM, eb.get(), ee.get(), c.elem_idx.get(), c.lmm.get(), su->volt.get(), NJ, jl,
                                                      c.j_p1.get(), c.j_p2.get(), c.imax.get());
        k_current_max_gnp<<<grid_for(ng + ngj + nmj), 256, 0, s>>>(ng, gl, H.tri.get(), H.tri_cnt.get(), ngj, gjl, H.jg_p1.get(),
                                                                    H.jg_p2.get(), nmj, mxl, H.jm_p1.get(), H.jm_p2.get(), c.lmm.get(),
                                                                    H.lmm_g.get(), su->volt.get(), c.imax.get());
        c.vol3.ensure(3 * (size_t)std::max(NM, 1));
        c.vol_kind.ensure(std::max(NM, 1));
        k_backbone_cnts<<<grid_for(NM), 256, 0, s>>>(NM, members, eb.get(), ee.get(), c.elem_idx.get(), c.lmm.get(), su->volt.get(),
                                                   c.imax.get(), 1, c.bb_lo.get(), c.bb_hi.get(), c.alive.get(), c.radii.get(), c.x.get(),
                                                   c.y.get(), c.z.get(), c.vol3.get(), c.vol_kind.get());
        k_volume_sum<<<1, kSumThreads, 0, s>>>(NM, fam, c.vol3.get(), c.vol_kind.get(), c.vol_acc.get());
        c.launches += 4;
        NM = compact_list(c, members, NM, c.alive, c.alive_scan, c.tmp_list);  // Find_backbone_cnts drops dead CNTs
        if (ng > 0) {  // Find_backbone_gnps (:577-660)
            H.elem_removed.ensure(std::max(n_elem, 1));
            H.removed_cnt.ensure(NCNT);
            CICY_CUDA(cudaMemsetAsync(H.elem_removed.get(), 0, sizeof(int32_t) * std::max(n_elem, 1), s));
            CICY_CUDA(cudaMemsetAsync(H.removed_cnt.get(), 0, sizeof(int32_t) * NCNT, s));
            H.mix_alive.ensure(std::max(nmj, 1));
            H.gj_alive.ensure(std::max(ngj, 1));
            k_fill_value_i32<<<grid_for(nmj), 256, 0, s>>>(nmj, 1, H.mix_alive.get());
            k_fill_value_i32<<<grid_for(ngj), 256, 0, s>>>(ngj, 1, H.gj_alive.get());
            c.launches += 2;
            if (nmj > 0) {
                H.key.ensure(nmj + 1);
                H.val.ensure(nmj + 1);
                H.alive.ensure(nmj + 1);
                H.alive_scan.ensure(nmj + 1);
                H.seg_start.ensure(nmj + 1);
                k_mix_keys<<<grid_for(nmj), 256, 0, s>>>(nmj, mxl, H.jm_n1.get(), H.key.get(), H.val.get());
                radix_sort_pairs(H.key.get(), H.val.get(), nmj, 32 + bits_for((uint64_t)NCNT), c.rs, s, c.launches);
                k_key_heads<<<grid_for(nmj), 256, 0, s>>>(nmj, H.key.get(), H.alive.get());
                exclusive_scan_i32(H.alive.get(), H.alive_scan.get(), nmj, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
                k_head_positions<<<grid_for(nmj), 256, 0, s>>>(nmj, H.alive.get(), H.alive_scan.get(), H.seg_start.get());
                c.launches += 3;
                const int nseg = read_i32(c, c.i32_scalar.get());
                k_mix_below_zero<<<grid_for(nseg), 256, 0, s>>>(nseg, H.seg_start.get(), nmj, H.val.get(), mxl, H.jm_p1.get(), H.jm_n1.get(),
                                                              H.jm_p2.get(), c.lmm.get(), H.lmm_g.get(), su->volt.get(), c.imax.get(),
                                                              c.mark_scan.get(), c.bb_lo.get(), c.bb_hi.get(), H.elem_removed.get(),
                                                              H.removed_cnt.get(), H.mix_alive.get(), H.pt_removed.get());
                c.launches++;
            }
            if (ngj > 0) {
                k_gj_below_zero<<<grid_for(ngj), 256, 0, s>>>(ngj, gjl, H.jg_p1.get(), H.jg_p2.get(), H.lmm_g.get(), su->volt.get(), c.imax.get(),
                                                            H.gj_alive.get(), H.pt_removed.get());
                c.launches++;
            }
            k_gnp_compact<<<grid_for(ng), 256, 0, s>>>(ng, gl, H.sptr.get(), H.sidx.get(), H.scount.get(), H.pt_removed.get());
            H.to_remove.ensure(1);
            CICY_CUDA(cudaMemsetAsync(H.to_remove.get(), 0, sizeof(int32_t), s));
            k_gnp_clear_dead<<<grid_for(ng), 256, 0, s>>>(ng, gl, H.sptr.get(), H.sidx.get(), H.scount.get(), H.nb.get(), H.pt_removed.get(),
                                                        H.to_remove.get(), c.status.get());
            c.launches += 2;
            int to_remove = read_i32(c, H.to_remove.get());
            for (int round = 0; to_remove && round <= ng + 1; round++) {
                CICY_CUDA(cudaMemcpyAsync(H.live.get(), H.scount.get(), sizeof(int32_t) * std::max(NG, 1), cudaMemcpyDeviceToDevice, s));
                k_dead_junction_round<<<1, 32, 0, s>>>(ngj, gjl, H.jg_p1.get(), H.jg_n1.get(), H.jg_p2.get(), H.jg_n2.get(), H.gj_alive.get(),
                                                     nmj, mxl, H.jm_p1.get(), H.jm_n1.get(), H.jm_p2.get(), H.jm_n2.get(), H.mix_alive.get(),
                                                     c.bb_lo.get(), c.bb_hi.get(), c.mark_scan.get(), H.elem_removed.get(), H.live.get(),
                                                     H.pt_removed.get());
                k_gnp_compact<<<grid_for(ng), 256, 0, s>>>(ng, gl, H.sptr.get(), H.sidx.get(), H.scount.get(), H.pt_removed.get());
                CICY_CUDA(cudaMemsetAsync(H.to_remove.get(), 0, sizeof(int32_t), s));
                k_gnp_clear_dead<<<grid_for(ng), 256, 0, s>>>(ng, gl, H.sptr.get(), H.sidx.get(), H.scount.get(), H.nb.get(),
                                                            H.pt_removed.get(), H.to_remove.get(), c.status.get());
                c.launches += 3;
                to_remove = read_i32(c, H.to_remove.get());
            }
            check_status(c, "Clear_structure_of_dead_gnps");
            // the junction lists without the removed junctions (order kept)
            if (nmj > 0) {
                CICY_CUDA(cudaMemcpyAsync(H.alive.get(), H.mix_alive.get(), sizeof(int32_t) * nmj, cudaMemcpyDeviceToDevice, s));
                H.cmj_len[j] = compact_list(c, mxl, nmj, H.alive, H.alive_scan, H.tmp_list);
            }
            if (ngj > 0) {
                CICY_CUDA(cudaMemcpyAsync(H.alive.get(), H.gj_alive.get(), sizeof(int32_t) * ngj, cudaMemcpyDeviceToDevice, s));
                H.cgj_len[j] = compact_list(c, gjl, ngj, H.alive, H.alive_scan, H.tmp_list);
            }
            // Remove_additional_cnts_from_cluster (:855-880)
            k_cnt_has_elements<<<grid_for(NM), 256, 0, s>>>(NM, members, c.bb_lo.get(), c.alive.get());
            c.launches++;
            NM = compact_list(c, members, NM, c.alive, c.alive_scan, c.tmp_list);
            k_gnp_volume_sum<<<1, 32, 0, s>>>(ng, fam, gl, H.scount.get(), H.vol.get(), H.tri_cnt.get(), H.vol_acc.get());
            // elements: kept ranges minus the points the mixed junctions took out
            CICY_CUDA(cudaMemsetAsync(c.mark.get(), 0, sizeof(int32_t) * (NP + 1), s));
            k_mark_kept_elements<<<grid_for(n_elem), 256, 0, s>>>(n_elem, c.elem_idx.get(), c.flag.get(), c.bb_lo.get(), c.bb_hi.get(),
                                                                 H.elem_removed.get(), c.mark.get());
            exclusive_scan_i32(c.mark.get(), c.mark_scan.get(), c.n_points + 1, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
            n_elem = read_i32(c, c.i32_scalar.get());
            k_fill_marked<<<grid_for(c.n_points), 256, 0, s>>>(c.n_points, c.mark.get(), c.mark_scan.get(), c.elem_idx.get());
            k_init_ranges<<<grid_for(NCNT), 256, 0, s>>>(c.n_cnts, c.cstart.get(), c.clen.get(), c.mark_scan.get(), c.bb_lo.get(), c.bb_hi.get());
            c.launches += 4;
        }
        clu_len[j] = NM;
        if (NJ > 0) {  // Remove_junctions_with_dead_particles_cnts (:950-992)
            k_junction_alive<<<grid_for(NJ), 256, 0, s>>>(NJ, jl, c.j_p1.get(), c.j_n1.get(), c.j_p2.get(), c.j_n2.get(), c.bb_lo.get(),
                                                        c.bb_hi.get(), c.mark_scan.get(), c.alive.get());
            c.launches++;
            cj_len[j] = compact_list(c, jl, NJ, c.alive, c.alive_scan, c.tmp_list);
        }
        CICY_CUDA(cudaEventRecord(e1, s));
        CICY_CUDA(cudaEventSynchronize(e1));
        t_bb += seconds_between(e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        CICY_LAUNCH_CHECK();
        // ---- real-resistor passes (Electrical_analysis.cpp:83-109, 229-289) ----
        if (j > 0) {  // Clear_triangulations_of_cluster(j - 1)
            const int ngp = H.h_cg_ptr[j] - H.h_cg_ptr[j - 1];
            k_clear_tri<<<grid_for(ngp), 256, 0, s>>>(ngp, H.cg_idx.get() + H.h_cg_ptr[j - 1], H.tri_cnt.get());
            c.launches++;
        }
        const int dir_bits[7] = {1, 2, 4, 3, 5, 6, 7};
        for (int d = 0; d < 3; d++) {
            if (!((dir_bits[fam] >> d) & 1) || !p.resistances[d]) continue;
            GnpPass gr{&H, gl, ng, mxl, H.cmj_len[j], gjl, H.cgj_len[j]};
            SolveInput r{j, d, d, members, clu_len[j], jl, cj_len[j], &gr};
            DeaSystem* sr = solve_dea(c, p, r, eb, ee);
            c.systems.push_back(sr);
            t_real += sr->seconds;
            // Calculate_parallel_resistor (:355-473): CNT and GNP currents through face b1
            const int b1 = d == 0 ? 2 : d == 1 ? 3 : 0;
            double I_cnt = 0, I_gnp = 0;
            if (clu_len[j] > 0) {
                const int nb = (int)(c.h_bcnt_ptr[b1 + 1] - c.h_bcnt_ptr[b1]);
                c.bterm.ensure(2 * (size_t)std::max(nb, 1));
                c.bvalid.ensure(2 * (size_t)std::max(nb, 1));
                k_boundary_terms<<<grid_for(2 * nb), 128, 0, s>>>((int)c.h_bcnt_ptr[b1], (int)c.h_bcnt_ptr[b1 + 1], c.bcnt_idx.get(),
                                                                 c.bb_lo.get(), c.bb_hi.get(), c.elem_idx.get(), c.lmm.get(), sr->volt.get(),
                                                                 c.radii.get(), p.resistivity_cnt, c.x.get(), c.y.get(), c.z.get(),
                                                                 c.bterm.get(), c.bvalid.get());
                k_boundary_sum<<<1, kSumThreads, 0, s>>>(2 * nb, c.bterm.get(), c.bvalid.get(), c.cur_out.get());
                c.launches += 2;
                CICY_CUDA(cudaMemcpyAsync(&I_cnt, c.cur_out.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
                CICY_CUDA(cudaStreamSynchronize(s));
            }
            if (ng > 0) {
                const int fb = H.h_bg_ptr[b1], nbg = H.h_bg_ptr[b1 + 1] - fb;
                H.boff.ensure(nbg + 1);
                H.gcnt.ensure(nbg + 1);
                k_face_tri_counts<<<grid_for(nbg), 256, 0, s>>>(nbg, H.bg_idx.get() + fb, H.tri_cnt.get(), H.gcnt.get());
                exclusive_scan_i32(H.gcnt.get(), H.boff.get(), nbg, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
                c.launches++;
                const int m = read_i32(c, c.i32_scalar.get());
                H.bterm.ensure(std::max(m, 1));
                H.bvalid.ensure(std::max(m, 1));
                k_gnp_boundary_terms<<<grid_for(nbg, 64), 64, 0, s>>>(nbg, H.bg_idx.get() + fb, H.boff.get(), 0, H.tri.get(), H.tri_cnt.get(),
                                                                    H.lmm_g.get(), H.rad_from.get(), H.cnt_rad.get(), H.t.get(), H.pts.get(),
                                                                    sr->volt.get(), H.rs, H.rt, H.bterm.get(), H.bvalid.get(), c.status.get());
                k_boundary_sum<<<1, kSumThreads, 0, s>>>(m, H.bterm.get(), H.bvalid.get(), c.cur_out.get() + 1);
                c.launches += 2;
                CICY_CUDA(cudaMemcpyAsync(&I_gnp, c.cur_out.get() + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
                check_status(c, "Currents_through_boundary_gnps");
            }
            parallel[d].push_back(p.applied_voltage / (I_cnt + I_gnp));
        }
    }
    c.h_bbclu_ptr.assign(NC + 1, 0);
    c.h_bbcj_ptr.assign(NC + 1, 0);
    for (int j = 0; j < NC; j++) {
        c.h_bbclu_ptr[j + 1] = c.h_bbclu_ptr[j] + clu_len[j];
        c.h_bbcj_ptr[j + 1] = c.h_bbcj_ptr[j] + cj_len[j];
    }
    c.bb_clu_len = clu_len;
    c.bb_cj_len = cj_len;
    c.have_backbone = true;
    c.have_hybrid = true;
    if (out) {
        const cicy_cuboid& w = c.window;
        const double L[3] = {w.len_x, w.len_y, w.len_z};
        const double A[3] = {w.len_y * w.len_z, w.len_x * w.len_z, w.len_x * w.len_y};
        for (int d = 0; d < 3; d++) {
            double R;
            if (parallel[d].empty()) {
                out->resistivities[d] = p.resistivity_matrix;
                out->resistances[d] = p.resistivity_matrix * L[d] / A[d];
                continue;
            } else if (parallel[d].size() == 1) {
                R = parallel[d][0];
            } else {
                double sum = 0;
                for (double r : parallel[d]) sum = sum + 1 / r;
                R = 1 / sum;
            }
            out->resistances[d] = R;
            out->resistivities[d] = R * A[d] / L[d];
        }
        out->n_percolated = NC;
        out->n_solves = (int32_t)std::min<size_t>(c.systems.size(), 32);
        for (int i = 0; i < out->n_solves; i++) {
            DeaSystem* sy = c.systems[i];
            cicy_solve_info& si = out->solves[i];
            si.cluster = sy->cluster;
            si.pass = sy->pass;
            si.nodes = sy->nodes;
            si.reserved = sy->reserved;
            si.nnz_lower = sy->nnz_lower;
            si.iterations = sy->iterations;
            si.rel_residual = sy->rel_residual;
            si.seconds = sy->seconds;
            si.kernel = sy->mg_levels > 0 ? 2 : sy->cluster_solver ? 1 : 0;
            si.levels = sy->mg_levels;
            si.fallback = sy->fallback;
            si.restarts = sy->restarts;
        }
        out->stage_seconds[2] = t_unit;
        out->stage_seconds[3] = t_bb;
        out->stage_seconds[4] = t_real;
    }
    c.stage = 4;
}

}  // namespace cicy
