// Direct Electrifying Algorithm on the device: node numbering, resistor
// assembly by sort-and-reduce, boundary-condition elimination, the Jacobi-PCG
// voltage solve, backbone extraction and boundary currents
// (Direct_Electrifying.cpp, Backbone_Network.cpp, Electrical_analysis.cpp).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <cmath>
#include <cooperative_groups.h>

#include "ctx.cuh"
#include "solver.cuh"
#include "trace.cuh"

namespace cicy {

namespace {

constexpr double kZero = 1.0e-10;                         // MathMatrix.h:18
constexpr double kPI = 3.1415926535897932384626433832795;  // Input_Reader.h:23
enum EdgeOp : int { OP_SKIP = 0, OP_OVERWRITE = 1, OP_ADD = 2 };

int grid_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)b;
}

// Get_vector_of_boundaries (Direct_Electrifying.cpp:249-305)
int boundaries_of_family(int family, int out[6]) {
    static const int tab[7][6] = {{2, 4}, {3, 5}, {0, 1}, {2, 4, 3, 5}, {2, 4, 0, 1}, {3, 5, 0, 1}, {2, 4, 3, 5, 0, 1}};
    static const int len[7] = {2, 2, 2, 4, 4, 4, 6};
    if (family < 0 || family > 6) return -1;
    for (int i = 0; i < len[family]; i++) out[i] = tab[family][i];
    return len[family];
}

// Per-CNT element ranges of the cluster being solved: [eb, ee) into elem_idx.
__global__ void k_cluster_ranges(int n, const int32_t* __restrict__ members, const int32_t* __restrict__ cur_lo,
                                 const int32_t* __restrict__ cur_hi, int32_t* __restrict__ eb, int32_t* __restrict__ ee,
                                 int* status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int c = members[i];
        int lo = cur_lo[c], hi = cur_hi[c];
        eb[i] = lo;
        ee[i] = hi + 1;
        // LM_matrix_for_cnts: "There is a CNT with not enough points to form an element"
        if (lo < 0 || hi - lo + 1 <= 1) atomicCAS(status, 0, (int)DEV_INPUT);
    }
}

__global__ void k_lmm_face(int b, int e, const int32_t* __restrict__ bpts, int node, int32_t* lmm) {
    for (int i = b + blockIdx.x * blockDim.x + threadIdx.x; i < e; i += gridDim.x * blockDim.x) lmm[bpts[i]] = node;
}

// LM_matrix_for_cnts (Direct_Electrifying.cpp:139-215): new nodes per CNT.
// Upstream walks the cluster's CNTs in order and gives the first and last
// element point a node only if the point has none yet.  Two CNTs can share an
// end point (window trimming splits a CNT at a boundary point and both segments
// keep it); the CNT earlier in the cluster then numbers it and the later one
// reuses it.  Here the CNTs run in parallel, so each shared end point is first
// claimed by the smallest cluster position (claim[P] = min i), and only the
// claimant counts and numbers it.
__global__ void k_claim_init(int n, const int32_t* __restrict__ eb, const int32_t* __restrict__ ee, const int32_t* __restrict__ elem,
                             int32_t* __restrict__ claim) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        claim[elem[eb[i]]] = 0x7fffffff;
        claim[elem[ee[i] - 1]] = 0x7fffffff;
    }
}

__global__ void k_claim(int n, const int32_t* __restrict__ eb, const int32_t* __restrict__ ee, const int32_t* __restrict__ elem,
                        int32_t* __restrict__ claim) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        atomicMin(&claim[elem[eb[i]]], i);
        atomicMin(&claim[elem[ee[i] - 1]], i);
    }
}

// new[i]: bit 0 first point numbered by CNT i, bit 1 last point numbered by CNT i
__global__ void k_node_counts(int n, const int32_t* __restrict__ eb, const int32_t* __restrict__ ee,
                              const int32_t* __restrict__ elem, const int32_t* __restrict__ lmm, const int32_t* __restrict__ claim,
                              int32_t* __restrict__ cnt, int32_t* __restrict__ fresh) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int b = eb[i], e = ee[i];
        int m = e - b;
        const int P0 = elem[b], P1 = elem[e - 1];
        const bool f0 = lmm[P0] < 0 && claim[P0] == i;
        const bool f1 = lmm[P1] < 0 && claim[P1] == i && P1 != P0;
        cnt[i] = (f0 ? 1 : 0) + (m - 2) + (f1 ? 1 : 0);
        fresh[i] = (f0 ? 1 : 0) | (f1 ? 2 : 0);
    }
}

__global__ void k_node_assign(int n, int reserved, const int32_t* __restrict__ eb, const int32_t* __restrict__ ee,
                              const int32_t* __restrict__ elem, const int32_t* __restrict__ base, const int32_t* __restrict__ fresh,
                              int32_t* lmm) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int b = eb[i], e = ee[i];
        int node = reserved + base[i];
        if (fresh[i] & 1) lmm[elem[b]] = node++;
        for (int k = b + 1; k < e - 1; k++) lmm[elem[k]] = node++;
        if (fresh[i] & 2) lmm[elem[e - 1]] = node++;
    }
}

// Calculate_resistance_cnt (Direct_Electrifying.cpp:611-646): rho L / (pi r^2), L summed point by point.
__device__ __forceinline__ double cnt_resistance(int P1, int P2, double radius, double rho, const double* __restrict__ x,
                                                 const double* __restrict__ y, const double* __restrict__ z) {
    double length = 0;
    for (int i = P1; i < P2; i++) {
        double dx = x[i] - x[i + 1], dy = y[i] - y[i + 1], dz = z[i] - z[i + 1];
        length = length + sqrt(dx * dx + dy * dy + dz * dz);
    }
    return rho * length / (kPI * radius * radius);
}

// CNT_volume_between_two_points (Backbone_Network.cpp:558-574): the same point-by-point
// length, times PI r^2 as (length * PI * r) * r.
__device__ __forceinline__ double cnt_volume(int P1, int P2, double radius, const double* __restrict__ x, const double* __restrict__ y,
                                             const double* __restrict__ z) {
    double length = 0;
    for (int i = P1; i < P2; i++) {
        double dx = x[i] - x[i + 1], dy = y[i] - y[i + 1], dz = z[i] - z[i + 1];
        length = length + sqrt(dx * dx + dy * dy + dz * dz);
    }
    return length * kPI * radius * radius;
}

__global__ void k_cnt_edge_counts(int n, const int32_t* __restrict__ eb, const int32_t* __restrict__ ee,
                                  const int32_t* __restrict__ elem, const int32_t* __restrict__ lmm, int32_t* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int b = eb[i], m = ee[i] - b;
        bool three = (m == 3) && lmm[elem[b]] == lmm[elem[b + 2]];
        cnt[i] = three ? 1 : m - 1;
    }
}

// Fill_2d_matrices_cnts + Three_points_in_element (Direct_Electrifying.cpp:489-608).
__global__ void k_cnt_edges(int n, int r_flag, double rho, const int32_t* __restrict__ members, const int32_t* __restrict__ eb,
                            const int32_t* __restrict__ ee, const int32_t* __restrict__ elem, const int32_t* __restrict__ lmm,
                            const int32_t* __restrict__ ofs, const double* __restrict__ radii, const double* __restrict__ x,
                            const double* __restrict__ y, const double* __restrict__ z, int32_t* __restrict__ n1,
                            int32_t* __restrict__ n2, int32_t* __restrict__ op, double* __restrict__ g) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int b = eb[i], m = ee[i] - b, o = ofs[i];
        double r = radii[members[i]];
        if (m == 3 && lmm[elem[b]] == lmm[elem[b + 2]]) {
            double g1 = 1.0, g2 = 1.0;
            if (r_flag == 1) {
                g1 = 1 / cnt_resistance(elem[b], elem[b + 1], r, rho, x, y, z);
                g2 = 1 / cnt_resistance(elem[b + 1], elem[b + 2], r, rho, x, y, z);
            }
            n1[o] = lmm[elem[b]];
            n2[o] = lmm[elem[b + 1]];
            op[o] = OP_OVERWRITE;
            g[o] = g1 + g2;
            continue;
        }
        for (int k = 0; k < m - 1; k++) {
            int P1 = elem[b + k], P2 = elem[b + k + 1];
            double gi = r_flag ? 1 / cnt_resistance(P1, P2, r, rho, x, y, z) : 1.0;
            n1[o + k] = lmm[P1];
            n2[o + k] = lmm[P2];
            op[o + k] = OP_OVERWRITE;
            g[o + k] = gi;
        }
    }
}

// Fill_2d_matrices_cnt_junctions + Calculate_junction_resistance (Direct_Electrifying.cpp:737-901).
__global__ void k_junction_edges(int nj, int base, int r_flag, int reserved, int jtype, double jres, double C1, double C2,
                                 const int32_t* __restrict__ jlist, const int32_t* __restrict__ jp1, const int32_t* __restrict__ jn1,
                                 const int32_t* __restrict__ jp2, const int32_t* __restrict__ jn2, const double* __restrict__ jd,
                                 const double* __restrict__ radii, const int32_t* __restrict__ lmm, int32_t* __restrict__ n1,
                                 int32_t* __restrict__ n2, int32_t* __restrict__ op, double* __restrict__ g) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nj; i += gridDim.x * blockDim.x) {
        int idx = jlist[i];
        int a = lmm[jp1[idx]], b = lmm[jp2[idx]];
        int o = base + i;
        n1[o] = a;
        n2[o] = b;
        g[o] = 0;
        op[o] = OP_SKIP;
        if (a == -1 || b == -1) continue;
        double ginv = 1.0;
        if (r_flag == 1) {
            double Re;
            if (jtype == 0) {
                Re = jres;
            } else {
                double l1 = radii[jn1[idx]], l2 = radii[jn2[idx]];
                double jl1 = l1 + l1, jl2 = l2 + l2;  // CNT diameters
                double A = (jl1 - jl2 < kZero) ? jl1 * jl1 : jl2 * jl2;
                double d = jd[idx];
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
    }
}

// Off-diagonal keys (row = max node, col = min node) and diagonal contributions.
// Skipped edges get the key 1 << (2 bn) (off-diagonal) / 1 << bn (diagonal) and sort last.
__global__ void k_edge_keys(int ne, int bn, const int32_t* __restrict__ n1, const int32_t* __restrict__ n2,
                            const int32_t* __restrict__ op, uint64_t* __restrict__ okey, uint32_t* __restrict__ oval,
                            uint64_t* __restrict__ dkey, uint32_t* __restrict__ dval) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += gridDim.x * blockDim.x) {
        int a = n1[i], b = n2[i];
        bool live = op[i] != OP_SKIP;
        uint64_t hi = (uint64_t)max(a, b), lo = (uint64_t)min(a, b);
        okey[i] = live ? ((hi << bn) | lo) : (1ull << (2 * bn));
        oval[i] = (uint32_t)i;
        dkey[2 * i] = live ? (uint64_t)a : (1ull << bn);
        dval[2 * i] = (uint32_t)i;
        dkey[2 * i + 1] = live ? (uint64_t)b : (1ull << bn);
        dval[2 * i + 1] = (uint32_t)i;
    }
}

// diagonal[node] += g in insertion order (Add_new_elements_to_2d_sparse_matrix et al.).
// Only free nodes: the prescribed nodes' diagonal is dropped (From_2d_to_1d_vectors)
// and their runs, one entry per boundary element, are the longest ones.
__global__ void k_diag_reduce(int n2e, uint64_t skip, uint64_t reserved, const uint64_t* __restrict__ dkey, const uint32_t* __restrict__ dval,
                              const double* __restrict__ g, double* __restrict__ diag_all) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2e; i += gridDim.x * blockDim.x) {
        uint64_t k = dkey[i];
        if (k == skip || k < reserved) continue;
        if (i > 0 && dkey[i - 1] == k) continue;
        double s = 0;
        for (int j = i; j < n2e && dkey[j] == k; j++) s += g[dval[j]];
        diag_all[k] = s;
    }
}

// col_values[row][col]: overwrite / subtract in insertion order.
__global__ void k_offdiag_reduce(int ne, uint64_t skip, const uint64_t* __restrict__ okey, const uint32_t* __restrict__ oval,
                                 const int32_t* __restrict__ op, const double* __restrict__ g, int32_t* __restrict__ head,
                                 double* __restrict__ runval) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += gridDim.x * blockDim.x) {
        uint64_t k = okey[i];
        bool h = (k != skip) && (i == 0 || okey[i - 1] != k);
        head[i] = h ? 1 : 0;
        if (!h) continue;
        double v = 0;
        for (int j = i; j < ne && okey[j] == k; j++) {
            uint32_t e = oval[j];
            if (op[e] == OP_OVERWRITE) v = -g[e];
            else v = v - g[e];
        }
        runval[i] = v;
    }
}

// From_2d_to_1d_vectors (Direct_Electrifying.cpp:1329-1394): split the unique
// (row, col) entries of the free rows into the SSS lower block and the rhs.
__global__ void k_sss_flags(int ne, int bn, int reserved, const uint64_t* __restrict__ okey, const int32_t* __restrict__ head,
                            int32_t* __restrict__ lower_flag) {
    const uint64_t mask = (1ull << bn) - 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += gridDim.x * blockDim.x) {
        bool f = false;
        if (head[i]) {
            long long row = (long long)(okey[i] >> bn), col = (long long)(okey[i] & mask);
            f = row >= reserved && col >= reserved;
        }
        lower_flag[i] = f ? 1 : 0;
    }
}

__global__ void k_sss_fill(int ne, int bn, int reserved, const uint64_t* __restrict__ okey, const int32_t* __restrict__ lower_flag,
                           const int32_t* __restrict__ lower_scan, const double* __restrict__ runval, int32_t* __restrict__ row_cnt,
                           int32_t* __restrict__ col, double* __restrict__ val) {
    const uint64_t mask = (1ull << bn) - 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += gridDim.x * blockDim.x) {
        if (!lower_flag[i]) continue;
        int row = (int)(okey[i] >> bn) - reserved, c = (int)(okey[i] & mask) - reserved;
        int o = lower_scan[i];
        col[o] = c;
        val[o] = runval[i];
        atomicAdd(&row_cnt[row], 1);
    }
}

// rhs: R[i] = R[i] - K_ij * VEF[j] for reserved columns j, ascending j.
__global__ void k_rhs(int ne, int bn, int reserved, const uint64_t* __restrict__ okey, const int32_t* __restrict__ head,
                      const double* __restrict__ runval, const double* __restrict__ vef, double* __restrict__ b) {
    const uint64_t mask = (1ull << bn) - 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        long long row = (long long)(okey[i] >> bn), col = (long long)(okey[i] & mask);
        if (row < reserved || col >= reserved) continue;
        // the first reserved-column entry of a row performs the row's ordered fold
        bool first = true;
        for (int j = i - 1; j >= 0; j--) {
            if (!head[j]) continue;
            long long r2 = (long long)(okey[j] >> bn);
            if (r2 == row) first = false;
            break;
        }
        if (!first) continue;
        double R = 0;
        for (int j = i; j < ne; j++) {
            if (!head[j]) continue;
            long long r2 = (long long)(okey[j] >> bn), c2 = (long long)(okey[j] & mask);
            if (r2 != row || c2 >= reserved) break;
            R = R - runval[j] * vef[c2];
        }
        b[row - reserved] = R;
    }
}

__global__ void k_diag_free(int n, int reserved, const double* __restrict__ diag_all, double* __restrict__ diag, int* status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = diag_all[i + reserved];
        diag[i] = d;
        if (fabs(d) < kZero) atomicCAS(status, 0, (int)DEV_ZERO_DIAG);
    }
}

// Full symmetric CSR (diagonal + lower + upper) for the gather SpMV of the CG.
__global__ void k_full_keys(int n, int m, int bn, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                            uint64_t* __restrict__ key, uint32_t* __restrict__ val) {
    // entries: [0, n) diagonal, [n, n+m) lower (row, col), [n+m, n+2m) upper (col, row)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + 2 * m; i += gridDim.x * blockDim.x) {
        uint64_t r, c;
        if (i < n) {
            r = c = (uint64_t)i;
        } else {
            int e = (i < n + m) ? i - n : i - n - m;
            // row of lower entry e: binary search in rp
            int lo = 0, hi = n;
            while (hi - lo > 1) {
                int mid = (lo + hi) >> 1;
                if (rp[mid] <= e) lo = mid; else hi = mid;
            }
            uint64_t rr = (uint64_t)lo, cc = (uint64_t)col[e];
            if (i < n + m) { r = rr; c = cc; } else { r = cc; c = rr; }
        }
        key[i] = (r << bn) | c;
        val[i] = (uint32_t)i;
    }
}

__global__ void k_full_fill(int n, int m, int bn, const uint64_t* __restrict__ key, const uint32_t* __restrict__ val,
                            const double* __restrict__ diag, const double* __restrict__ lval, int32_t* __restrict__ rcnt,
                            int32_t* __restrict__ fcol, double* __restrict__ fval, double* __restrict__ minv) {
    const uint64_t mask = (1ull << bn) - 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + 2 * m; i += gridDim.x * blockDim.x) {
        uint32_t src = val[i];
        int r = (int)(key[i] >> bn);
        fcol[i] = (int)(key[i] & mask);
        double v;
        if ((int)src < n) {
            v = diag[src];
            minv[src] = 1 / diag[src];  // Jacobi_preconditioner (Direct_Electrifying.cpp:1662-1668)
        } else {
            int e = ((int)src < n + m) ? (int)src - n : (int)src - n - m;
            v = lval[e];
        }
        fval[i] = v;
        atomicAdd(&rcnt[r], 1);
    }
}

// Initial_guess_for_cnt_nodes (Direct_Electrifying.cpp:1434-1470).
__global__ void k_initial_guess(int n, int reserved, int family, double v_p_coord, double max_coord, const int32_t* __restrict__ eb,
                                const int32_t* __restrict__ ee, const int32_t* __restrict__ elem, const int32_t* __restrict__ lmm,
                                const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                                double* __restrict__ x0) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int k = eb[i]; k < ee[i]; k++) {
            int P = elem[k];
            int node = lmm[P];
            if (node >= 2) {
                double c = family == 0 ? x[P] : family == 1 ? y[P] : z[P];
                x0[node - reserved] = v_p_coord * (max_coord - c);
            }
        }
    }
}

__global__ void k_spmv_residual(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                                const double* __restrict__ xin, const double* __restrict__ b, double* __restrict__ r) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++) s += v[k] * xin[ci[k]];
        r[i] = b[i] - s;
    }
}

// block_reduce2 for the residual report
__device__ __forceinline__ void block_reduce2(double a, double b, double* sm, double& ra, double& rb) {
    a = warp_sum(a);
    b = warp_sum(b);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sm[w] = a; sm[32 + w] = b; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        double x = lane < nw ? sm[lane] : 0.0, y = lane < nw ? sm[32 + lane] : 0.0;
        x = warp_sum(x);
        y = warp_sum(y);
        if (lane == 0) { sm[64] = x; sm[65] = y; }
    }
    __syncthreads();
    ra = sm[64];
    rb = sm[65];
    __syncthreads();
}

__global__ void k_true_residual(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ v,
                                const double* __restrict__ xs, const double* __restrict__ b, double* out) {
    __shared__ double sm[72];
    double rr = 0, bb = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = rp[i]; k < rp[i + 1]; k++) s += v[k] * xs[ci[k]];
        double ri = b[i] - s;
        rr += ri * ri;
        bb += b[i] * b[i];
    }
    double s0, s1;
    block_reduce2(rr, bb, sm, s0, s1);
    if (threadIdx.x == 0) {
        atomicAdd(&out[0], s0);
        atomicAdd(&out[1], s1);
    }
}

__global__ void k_voltages(int nodes, int reserved, const double* __restrict__ vef, const double* __restrict__ xs, double* __restrict__ v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nodes; i += gridDim.x * blockDim.x)
        v[i] = i < reserved ? vef[i] : xs[i - reserved];
}

// ---------------------------------------------------------------------------
// Backbone (Backbone_Network.cpp:64-409): element currents on unit resistors,
// zero current = 1e-9 I_max, one kept run per CNT.
__device__ __forceinline__ void atomic_max_pos(unsigned long long* addr, double v) {
    atomicMax(addr, (unsigned long long)__double_as_longlong(v));  // v >= 0: IEEE order == integer order
}

__global__ void k_current_max(int n, const int32_t* __restrict__ eb, const int32_t* __restrict__ ee, const int32_t* __restrict__ elem,
                              const int32_t* __restrict__ lmm, const double* __restrict__ volt, int nj,
                              const int32_t* __restrict__ jlist, const int32_t* __restrict__ jp1, const int32_t* __restrict__ jp2,
                              unsigned long long* imax) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + nj; i += gridDim.x * blockDim.x) {
        double m = 0;
        if (i < n) {
            for (int k = eb[i]; k < ee[i] - 1; k++) m = fmax(m, fabs(volt[lmm[elem[k]]] - volt[lmm[elem[k + 1]]]));
        } else {
            int j = jlist[i - n];
            m = fabs(volt[lmm[jp1[j]]] - volt[lmm[jp2[j]]]);
        }
        atomic_max_pos(imax, m);
    }
}

// Find_backbone_cnts (Backbone_Network.cpp:313-345): the kept element run of every CNT of
// the cluster, and Calculate_cnt_volumes' (:412-556) volumes of its parts: vol3[3i] the dead
// part before the run (the whole CNT when nothing is kept), vol3[3i+1] the run, vol3[3i+2]
// the dead part after it; kind[i] = 0 nothing kept, 1 kept to the end, 2 dead part after.
// The current-carrying run of one backbone member: element offsets idx1 (first element whose
// current exceeds the zero current) and idx2 (first one after it that does not), -1 when absent.
__device__ __forceinline__ void backbone_run(int b, int e, const int32_t* __restrict__ elem, const int32_t* __restrict__ lmm,
                                             const double* __restrict__ volt, double zero_current, int& idx1, int& idx2) {
    idx1 = -1;
    idx2 = -1;
    for (int k = 0; k < e - b - 1; k++) {
        double I = fabs(volt[lmm[elem[b + k]]] - volt[lmm[elem[b + k + 1]]]);
        if (I - zero_current > kZero) {
            if (idx1 == -1) idx1 = k;
        } else if (idx1 != -1 && idx2 == -1) {
            idx2 = k;
            break;
        }
    }
}

// Volumes of member i's parts from its end points Ps, Pe and cut points P1, P2 (-1: absent).
__device__ __forceinline__ void backbone_volumes(int i, double r, int Ps, int P1, int P2, int Pe, const double* __restrict__ x,
                                                 const double* __restrict__ y, const double* __restrict__ z, double* __restrict__ vol3,
                                                 int32_t* __restrict__ kind) {
    if (P1 < 0) {
        vol3[3 * i] = cnt_volume(Ps, Pe, r, x, y, z);
        kind[i] = 0;
    } else {
        vol3[3 * i] = cnt_volume(Ps, P1, r, x, y, z);
        if (P2 < 0) {
            vol3[3 * i + 1] = cnt_volume(P1, Pe, r, x, y, z);
            kind[i] = 1;
        } else {
            vol3[3 * i + 1] = cnt_volume(P1, P2, r, x, y, z);
            vol3[3 * i + 2] = cnt_volume(P2, Pe, r, x, y, z);
            kind[i] = 2;
        }
    }
}

__device__ __forceinline__ void backbone_trim(int i, int c, int b, int e, int idx1, int idx2, int trim, int32_t* __restrict__ cur_lo,
                                              int32_t* __restrict__ cur_hi, int32_t* __restrict__ alive) {
    if (!trim) {
        alive[i] = 1;
        return;
    }
    if (idx1 == -1) {
        cur_lo[c] = -1;
        cur_hi[c] = -2;
        alive[i] = 0;
    } else {
        cur_lo[c] = b + idx1;
        cur_hi[c] = (idx2 == -1) ? e - 1 : b + idx2;
        alive[i] = 1;
    }
}

__global__ void k_backbone_cnts(int n, const int32_t* __restrict__ members, const int32_t* __restrict__ eb, const int32_t* __restrict__ ee,
                                const int32_t* __restrict__ elem, const int32_t* __restrict__ lmm, const double* __restrict__ volt,
                                const unsigned long long* __restrict__ imax_bits, int trim, int32_t* __restrict__ cur_lo,
                                int32_t* __restrict__ cur_hi, int32_t* __restrict__ alive, const double* __restrict__ radii,
                                const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                                double* __restrict__ vol3, int32_t* __restrict__ kind) {
    const double i_max = fmax(__longlong_as_double((long long)*imax_bits), kZero);
    const double zero_current = i_max * 1e-9;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int b = eb[i], e = ee[i];
        int idx1, idx2;
        backbone_run(b, e, elem, lmm, volt, zero_current, idx1, idx2);
        const int c = members[i];
        backbone_volumes(i, radii[c], elem[b], idx1 < 0 ? -1 : elem[b + idx1], idx2 < 0 ? -1 : elem[b + idx2], elem[e - 1], x, y, z, vol3,
                         kind);
        backbone_trim(i, c, b, e, idx1, idx2, trim, cur_lo, cur_hi, alive);
    }
}

// k_backbone_cnts split for the side stream: the run and the trim here, the member's CNT and
// part end points into pts (5 per member) for k_backbone_volumes.
__global__ void k_backbone_scan(int n, const int32_t* __restrict__ members, const int32_t* __restrict__ eb, const int32_t* __restrict__ ee,
                                const int32_t* __restrict__ elem, const int32_t* __restrict__ lmm, const double* __restrict__ volt,
                                const unsigned long long* __restrict__ imax_bits, int trim, int32_t* __restrict__ cur_lo,
                                int32_t* __restrict__ cur_hi, int32_t* __restrict__ alive, int32_t* __restrict__ pts) {
    const double i_max = fmax(__longlong_as_double((long long)*imax_bits), kZero);
    const double zero_current = i_max * 1e-9;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int b = eb[i], e = ee[i];
        int idx1, idx2;
        backbone_run(b, e, elem, lmm, volt, zero_current, idx1, idx2);
        const int c = members[i];
        pts[5 * i] = c;
        pts[5 * i + 1] = elem[b];
        pts[5 * i + 2] = idx1 < 0 ? -1 : elem[b + idx1];
        pts[5 * i + 3] = idx2 < 0 ? -1 : elem[b + idx2];
        pts[5 * i + 4] = elem[e - 1];
        backbone_trim(i, c, b, e, idx1, idx2, trim, cur_lo, cur_hi, alive);
    }
}

__global__ void k_backbone_volumes(int n, const int32_t* __restrict__ pts, const double* __restrict__ radii, const double* __restrict__ x,
                                   const double* __restrict__ y, const double* __restrict__ z, double* __restrict__ vol3,
                                   int32_t* __restrict__ kind) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        backbone_volumes(i, radii[pts[5 * i]], pts[5 * i + 1], pts[5 * i + 2], pts[5 * i + 3], pts[5 * i + 4], x, y, z, vol3, kind);
}

// Volume members of Backbone_Network (acc: volumes_cnt[8], dead_branches[7], then the
// fractions step's total_volumes[8] and fractions[8]).
constexpr int kVolCnt = 0, kVolDead = 8, kVolTotal = 15, kVolFrac = 23, kVolWords = 31;

// Ordered FP64 sums on one CTA of kSumThreads: warps 1.. stage chunk ch + 1 of the
// inputs in shared memory (double-buffered) while thread 0 adds chunk ch in order, so the
// result is the sequence of additions of a sequential loop, at shared-memory latency.
constexpr int kSumThreads = 256;
constexpr int kSumChunk = 512;

template <class Stage, class Consume>
__device__ __forceinline__ void staged_in_order(int n, Stage stage, Consume consume) {
    const int nch = (n + kSumChunk - 1) / kSumChunk;
    const int t = (int)threadIdx.x - 32, T = (int)blockDim.x - 32;
    if (t >= 0 && nch > 0) stage(0, 0, t, T);
    __syncthreads();
    for (int ch = 0; ch < nch; ch++) {
        const int m = min(kSumChunk, n - ch * kSumChunk);
        if (threadIdx.x == 0)
            consume(ch & 1, m);
        else if (t >= 0 && ch + 1 < nch)
            stage(ch + 1, (ch + 1) & 1, t, T);
        __syncthreads();
    }
}

// The cluster's volumes added to its family in upstream's order: CNTs last to first
// (Backbone_Network.cpp:325), per CNT the dead part(s) and then the kept run (:442-543).
// The staging threads turn the parts a CNT does not have into +0.0 terms: the sums start at
// +0.0 and only add volumes >= 0, so x + 0.0 == x and the consumer adds without branches.
__global__ void __launch_bounds__(kSumThreads) k_volume_sum(int n, int family, const double* __restrict__ vol3,
                                                            const int32_t* __restrict__ kind, double* acc) {
    __shared__ double sv[2][3 * kSumChunk];
    double dead = 0, bb = 0;
    if (threadIdx.x == 0) {
        dead = acc[kVolDead + family];
        bb = acc[kVolCnt + family];
    }
    staged_in_order(
        n,
        [&](int ch, int b, int t, int T) {
            const int i0 = n - 1 - ch * kSumChunk, m = min(kSumChunk, i0 + 1);
            for (int j = t; j < m; j += T) {
                const int i = i0 - j, k = kind[i];
                sv[b][3 * j] = vol3[3 * i];
                sv[b][3 * j + 1] = k == 2 ? vol3[3 * i + 2] : 0.0;
                sv[b][3 * j + 2] = k >= 1 ? vol3[3 * i + 1] : 0.0;
            }
        },
        [&](int b, int m) {
            const double* v = sv[b];
#pragma unroll 4
            for (int j = 0; j < m; j++) {
                dead = (dead + v[3 * j]) + v[3 * j + 1];
                bb = bb + v[3 * j + 2];
            }
        });
    if (threadIdx.x == 0) {
        acc[kVolDead + family] = dead;
        acc[kVolCnt + family] = bb;
    }
}

// Sort keys of HoKo->isolated_cnt's order (Hoshen_Kopelman.cpp:2331-2363, 2527-2539): CNTs
// without a label first, then the non-percolated clusters by label, each in cnts_inside
// order; CNTs of percolated clusters sort last (group n_labels + 1).
__global__ void k_isolated_keys(int n_inside, int n_labels, const int32_t* __restrict__ inside, const int32_t* __restrict__ labels,
                                const int32_t* __restrict__ perc_bits, uint64_t* __restrict__ key, uint32_t* __restrict__ val) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_inside; p += gridDim.x * blockDim.x) {
        const int c = inside[p];
        const int L = labels[c];
        const long long g = L < 0 ? 0 : (perc_bits[L] != 0 ? n_labels + 1 : L + 1);
        key[p] = (uint64_t)(g * n_inside + p);
        val[p] = (uint32_t)c;
    }
}

// Whole-CNT volumes of HoKo->isolated_cnt's entries (keys below `end`, a prefix of the
// sorted list) for Calculate_volume_of_non_percolated_cnts; count = their number.
__global__ void k_isolated_volumes(int n_inside, uint64_t end, const uint64_t* __restrict__ key, const uint32_t* __restrict__ cnt,
                                   const int32_t* __restrict__ cstart, const int32_t* __restrict__ clen, const double* __restrict__ radii,
                                   const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                                   double* __restrict__ vol, int32_t* count) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_inside; p += gridDim.x * blockDim.x) {
        if (key[p] >= end) continue;
        const int c = (int)cnt[p];
        vol[p] = cnt_volume(cstart[c], cstart[c] + clen[c] - 1, radii[c], x, y, z);
        atomicMax(count, p + 1);
    }
}

// Calculate_percolated_families_fractions with Calculate_volume_of_non_percolated_cnts
// (Electrical_analysis.cpp:678-786) for CNTs: the isolated list's volumes added in order,
// volumes_cnt[7] = dead branches + that, then total volumes and fractions (no GNPs: their
// volumes are 0), upstream's sequence of additions.
__global__ void __launch_bounds__(kSumThreads) k_family_fractions(const int32_t* __restrict__ count, const double* __restrict__ vol,
                                                                  double* acc) {
    __shared__ double sv[2][kSumChunk];
    double np_cnts = 0;
    staged_in_order(
        *count,
        [&](int ch, int b, int t, int T) {
            const int m = min(kSumChunk, *count - ch * kSumChunk);
            for (int j = t; j < m; j += T) sv[b][j] = vol[ch * kSumChunk + j];
        },
        [&](int b, int m) {
            for (int j = 0; j < m; j++) np_cnts = np_cnts + sv[b][j];
        });
    if (threadIdx.x != 0) return;
    double total_dead = 0, total_dead_gnps = 0;
    for (int i = 0; i < 7; i++) {
        total_dead = total_dead + acc[kVolDead + i];
        total_dead_gnps = total_dead_gnps + 0.0;
    }
    acc[kVolCnt + 7] = total_dead + np_cnts;
    double tv = 0;
    for (int i = 0; i < 8; i++) {
        acc[kVolTotal + i] = 0.0 + acc[kVolCnt + i] + 0.0;
        tv = tv + acc[kVolCnt + i] + 0.0;
    }
    for (int i = 0; i < 8; i++) acc[kVolFrac + i] = acc[kVolTotal + i] / tv;
    (void)total_dead_gnps;
}

// Remove_junctions_with_dead_particles_cnts (Backbone_Network.cpp:950-992).
__global__ void k_junction_alive(int nj, const int32_t* __restrict__ jlist, const int32_t* __restrict__ jp1, const int32_t* __restrict__ jn1,
                                 const int32_t* __restrict__ jp2, const int32_t* __restrict__ jn2, const int32_t* __restrict__ cur_lo,
                                 const int32_t* __restrict__ cur_hi, const int32_t* __restrict__ elem_pos, int32_t* __restrict__ alive) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nj; i += gridDim.x * blockDim.x) {
        int j = jlist[i];
        int c1 = jn1[j], c2 = jn2[j];
        bool ok = cur_lo[c1] >= 0 && cur_lo[c2] >= 0;
        if (ok) {
            int q1 = elem_pos[jp1[j]], q2 = elem_pos[jp2[j]];
            ok = q1 >= cur_lo[c1] && q1 <= cur_hi[c1] && q2 >= cur_lo[c2] && q2 <= cur_hi[c2];
        }
        alive[i] = ok ? 1 : 0;
    }
}

__global__ void k_compact_i32(int n, const int32_t* __restrict__ in, const int32_t* __restrict__ flag, const int32_t* __restrict__ scan,
                              int32_t* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) out[scan[i]] = in[i];
}

// Currents_through_boundary_cnts / Current_of_element_in_boundary (Electrical_analysis.cpp:499-605).
// The terms V/Re (two per boundary CNT) are independent: one thread each computes
// them; k_boundary_sum then adds them in upstream boundary order, so the total is
// the same sequence of FP64 additions as the upstream loop.
__global__ void k_boundary_terms(int b, int e, const int32_t* __restrict__ bcnt, const int32_t* __restrict__ cur_lo,
                                 const int32_t* __restrict__ cur_hi, const int32_t* __restrict__ elem, const int32_t* __restrict__ lmm,
                                 const double* __restrict__ volt, const double* __restrict__ radii, double rho,
                                 const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                                 double* __restrict__ term, int32_t* __restrict__ valid) {
    const int m = 2 * (e - b);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        const int i = b + (t >> 1), side = t & 1;
        int ok = 0;
        double v = 0;
        const int c = bcnt[i];
        const int lo = cur_lo[c], hi = cur_hi[c];
        if (lo >= 0 && hi >= lo) {
            const int P1 = side == 0 ? elem[lo] : elem[hi];
            const int P2 = side == 0 ? elem[lo + 1] : elem[hi - 1];
            const int n1 = lmm[P1];
            if (n1 >= 0 && n1 <= 1) {
                const int n2 = lmm[P2];
                if (n2 >= 0) {
                    const double V = volt[n2] - volt[n1];
                    const double Re = (P1 > P2) ? cnt_resistance(P2, P1, radii[c], rho, x, y, z)
                                                : cnt_resistance(P1, P2, radii[c], rho, x, y, z);
                    v = V / Re;
                    ok = 1;
                }
            }
        }
        term[t] = v;
        valid[t] = ok;
    }
}

__global__ void __launch_bounds__(kSumThreads) k_boundary_sum(int m, const double* __restrict__ term, const int32_t* __restrict__ valid,
                                                              double* out) {
    __shared__ double sv[2][kSumChunk];
    double I = 0;  // starts at +0.0 and never becomes -0.0, so skipped terms can be added as +0.0
    staged_in_order(
        m,
        [&](int ch, int b, int t, int T) {
            const int mm = min(kSumChunk, m - ch * kSumChunk);
            for (int j = t; j < mm; j += T) sv[b][j] = valid[ch * kSumChunk + j] ? term[ch * kSumChunk + j] : 0.0;
        },
        [&](int b, int mm) {
#pragma unroll 4
            for (int j = 0; j < mm; j++) I = I + sv[b][j];
        });
    if (threadIdx.x == 0) *out = I;
}

__global__ void k_init_ranges(int nc, const int32_t* __restrict__ cstart, const int32_t* __restrict__ clen, const int32_t* __restrict__ mscan,
                              int32_t* __restrict__ lo, int32_t* __restrict__ hi) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        int b = mscan[cstart[c]], e = mscan[cstart[c] + clen[c]];
        if (clen[c] == 0) b = e = 0;
        lo[c] = e > b ? b : -1;
        hi[c] = e > b ? e - 1 : -2;
    }
}

// ---------------------------------------------------------------------------
struct SolveInput {
    int cluster;
    int pass;  // -1 unit, 0..2 direction
    int family;
    const int32_t* members;
    int n_members;
    const int32_t* jlist;
    int n_jlist;
    const GnpPass* gnp = nullptr;  // the GNP side of a mixed cluster (hybrid_dea.cuh), or none
};

// GNP side of a mixed cluster's system (hybrid_dea.cuh): GNP point nodes after the CNT
// nodes (returns how many), then the CNT-GNP, triangulation and GNP-GNP resistors
// (count, then fill at `base`), as Compute_voltage_field adds them.
int gnp_lmm(Ctx& c, const GnpPass& g, const int* bnd, int nbnd, int first_node);
int gnp_prepare_edges(Ctx& c, const GnpPass& g, int r_flag);
void gnp_fill_edges(Ctx& c, const GnpPass& g, int base, int r_flag, int reserved, const cicy_params& p);

__global__ void k_singleton_chains(int n, int first_chain, int first_row, int32_t* __restrict__ cs, int32_t* __restrict__ cl) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        cs[first_chain + k] = first_row + k;
        cl[first_chain + k] = 1;
    }
}

double seconds_between(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms * 1e-3;
}

// Direct_Electrifying::Compute_voltage_field (Direct_Electrifying.cpp:11-113), CNT branch.
DeaSystem* solve_dea(Ctx& c, const cicy_params& p, const SolveInput& in, DBuf<int32_t>& eb, DBuf<int32_t>& ee) {
    cudaStream_t s = c.stream;
    const int r_flag = in.pass >= 0 ? 1 : 0;
    int bnd[6];
    const int nbnd = boundaries_of_family(in.family, bnd);
    if (nbnd < 0) throw Fail{CICY_E_INPUT, "Compute_voltage_field: invalid family"};
    const int reserved = nbnd;  // Get_global_nodes: 2/4/6
    const int NM = in.n_members;
    // systems of earlier runs are recycled: their grow-only device buffers stay allocated
    DeaSystem* sys;
    if (!c.sys_pool.empty()) {
        sys = c.sys_pool.back();
        c.sys_pool.pop_back();
        sys->reset();
    } else {
        sys = new DeaSystem;
    }
    sys->cluster = in.cluster;
    sys->pass = in.pass;
    sys->reserved = reserved;
    try {
        eb.ensure(NM + 1);
        ee.ensure(NM + 1);
        k_cluster_ranges<<<grid_for(NM), 256, 0, s>>>(NM, in.members, c.bb_lo.get(), c.bb_hi.get(), eb.get(), ee.get(), c.status.get());
        c.launches++;
        check_status(c, "LM_matrix_for_cnts");
        TraceSeq tr(s);
        // ---- LMM ----
        c.lmm.ensure(std::max(c.n_points, 1));
        CICY_CUDA(cudaMemsetAsync(c.lmm.get(), 0xff, sizeof(int32_t) * std::max(c.n_points, 1), s));
        for (int k = 0; k < nbnd; k++) {
            int f = bnd[k];
            int b = c.h_bpts_ptr[f], e = c.h_bpts_ptr[f + 1];
            if (e > b) {
                k_lmm_face<<<grid_for(e - b), 256, 0, s>>>(b, e, c.bpts_idx.get(), k, c.lmm.get());
                c.launches++;
            }
        }
        c.cnt_nodes.ensure(NM + 1);
        c.cnt_node_base.ensure(NM + 1);
        c.claim.ensure(std::max(c.n_points, 1));
        c.cnt_fresh.ensure(NM + 1);
        k_claim_init<<<grid_for(NM), 256, 0, s>>>(NM, eb.get(), ee.get(), c.elem_idx.get(), c.claim.get());
        k_claim<<<grid_for(NM), 256, 0, s>>>(NM, eb.get(), ee.get(), c.elem_idx.get(), c.claim.get());
        k_node_counts<<<grid_for(NM), 256, 0, s>>>(NM, eb.get(), ee.get(), c.elem_idx.get(), c.lmm.get(), c.claim.get(), c.cnt_nodes.get(),
                                                   c.cnt_fresh.get());
        exclusive_scan_i32(c.cnt_nodes.get(), c.cnt_node_base.get(), NM, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
        k_node_assign<<<grid_for(NM), 256, 0, s>>>(NM, reserved, eb.get(), ee.get(), c.elem_idx.get(), c.cnt_node_base.get(),
                                                   c.cnt_fresh.get(), c.lmm.get());
        c.launches += 4;
        int nodes = reserved + read_i32(c, c.i32_scalar.get());
        const int n_cnt_free = nodes - reserved;
        const int n_gnp_nodes = in.gnp ? gnp_lmm(c, *in.gnp, bnd, nbnd, nodes) : 0;
        nodes += n_gnp_nodes;
        // free nodes of each CNT are one consecutive range: the chains of the block preconditioner;
        // each GNP point node is a chain of its own
        const int NMc = NM + n_gnp_nodes;
        c.chain_start.ensure(NMc + 1);
        c.chain_len.ensure(NMc + 1);
        if (NM > 0) {
            CICY_CUDA(cudaMemcpyAsync(c.chain_start.get(), c.cnt_node_base.get(), sizeof(int32_t) * NM, cudaMemcpyDeviceToDevice, s));
            CICY_CUDA(cudaMemcpyAsync(c.chain_len.get(), c.cnt_nodes.get(), sizeof(int32_t) * NM, cudaMemcpyDeviceToDevice, s));
        }
        if (n_gnp_nodes > 0) {
            k_singleton_chains<<<grid_for(n_gnp_nodes), 256, 0, s>>>(n_gnp_nodes, NM, n_cnt_free, c.chain_start.get(), c.chain_len.get());
            c.launches++;
        }
        const int n = nodes - reserved;
        sys->nodes = nodes;
        tr.mark(r_flag ? "dea.real.lmm" : "dea.unit.lmm");
        // ---- edges ----
        k_cnt_edge_counts<<<grid_for(NM), 256, 0, s>>>(NM, eb.get(), ee.get(), c.elem_idx.get(), c.lmm.get(), c.cnt_nodes.get());
        exclusive_scan_i32(c.cnt_nodes.get(), c.cnt_node_base.get(), NM, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
        c.launches++;
        const int n_cnt_edges = read_i32(c, c.i32_scalar.get());
        const int n_gnp_edges = in.gnp ? gnp_prepare_edges(c, *in.gnp, r_flag) : 0;
        const int NE = n_cnt_edges + in.n_jlist + n_gnp_edges;
        c.e_n1.ensure(NE + 1); c.e_n2.ensure(NE + 1); c.e_op.ensure(NE + 1); c.e_g.ensure(NE + 1);
        k_cnt_edges<<<grid_for(NM), 256, 0, s>>>(NM, r_flag, p.resistivity_cnt, in.members, eb.get(), ee.get(), c.elem_idx.get(), c.lmm.get(),
                                               c.cnt_node_base.get(), c.radii.get(), c.x.get(), c.y.get(), c.z.get(), c.e_n1.get(),
                                               c.e_n2.get(), c.e_op.get(), c.e_g.get());
        c.launches++;
        if (in.n_jlist > 0) {
            k_junction_edges<<<grid_for(in.n_jlist), 256, 0, s>>>(in.n_jlist, n_cnt_edges, r_flag, reserved, p.junction_type,
                                                                p.junction_resistance, p.C1, p.C2, in.jlist, c.j_p1.get(), c.j_n1.get(),
                                                                c.j_p2.get(), c.j_n2.get(), c.j_d.get(), c.radii.get(), c.lmm.get(),
                                                                c.e_n1.get(), c.e_n2.get(), c.e_op.get(), c.e_g.get());
            c.launches++;
        }
        if (in.gnp) gnp_fill_edges(c, *in.gnp, n_cnt_edges + in.n_jlist, r_flag, reserved, p);
        tr.mark(r_flag ? "dea.real.edges" : "dea.unit.edges");
        // ---- sort-and-reduce assembly ----
        const int bn = bits_for((uint64_t)std::max(nodes, 1));
        const int ND = 2 * NE;
        c.sort_k.ensure(std::max(ND, 2 * NE) + 2);
        c.sort_v.ensure(std::max(ND, 2 * NE) + 2);
        DBuf<uint64_t>& dkey = c.dkey;
        DBuf<uint32_t>& dval = c.dval;
        dkey.ensure(ND + 2);
        dval.ensure(ND + 2);
        k_edge_keys<<<grid_for(NE), 256, 0, s>>>(NE, bn, c.e_n1.get(), c.e_n2.get(), c.e_op.get(), c.sort_k.get(), c.sort_v.get(),
                                               dkey.get(), dval.get());
        c.launches++;
        radix_sort_pairs(c.sort_k.get(), c.sort_v.get(), NE, 2 * bn + 1, c.rs, s, c.launches);
        radix_sort_pairs(dkey.get(), dval.get(), ND, bn + 1, c.rs, s, c.launches);
        tr.mark("asm.sorts");
        c.work_f64a.ensure(std::max(nodes, NE) + 1);  // diag over all nodes
        CICY_CUDA(cudaMemsetAsync(c.work_f64a.get(), 0, sizeof(double) * (nodes + 1), s));
        k_diag_reduce<<<grid_for(ND), 256, 0, s>>>(ND, 1ull << bn, (uint64_t)reserved, dkey.get(), dval.get(), c.e_g.get(),
                                                   c.work_f64a.get());
        c.work_i32a.ensure(NE + 1);
        c.work_i32b.ensure(NE + 1);
        c.work_i32c.ensure(NE + 1);
        c.runval.ensure(NE + 1);
        k_offdiag_reduce<<<grid_for(NE), 256, 0, s>>>(NE, 1ull << (2 * bn), c.sort_k.get(), c.sort_v.get(), c.e_op.get(), c.e_g.get(), c.work_i32a.get(),
                                                    c.runval.get());
        tr.mark("asm.reduce");
        k_sss_flags<<<grid_for(NE), 256, 0, s>>>(NE, bn, reserved, c.sort_k.get(), c.work_i32a.get(), c.work_i32b.get());
        exclusive_scan_i32(c.work_i32b.get(), c.work_i32c.get(), NE, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
        c.launches += 3;
        const int m = read_i32(c, c.i32_scalar.get());
        sys->nnz_lower = m;
        sys->row_ptr.ensure(n + 1); sys->col.ensure(std::max(m, 1)); sys->val.ensure(std::max(m, 1));
        sys->diag.ensure(std::max(n, 1)); sys->b.ensure(std::max(n, 1)); sys->x0.ensure(std::max(n, 1));
        sys->volt.ensure(std::max(nodes, 1));
        c.cnt_nodes.ensure(n + 1);
        CICY_CUDA(cudaMemsetAsync(c.cnt_nodes.get(), 0, sizeof(int32_t) * (n + 1), s));
        k_sss_fill<<<grid_for(NE), 256, 0, s>>>(NE, bn, reserved, c.sort_k.get(), c.work_i32b.get(), c.work_i32c.get(), c.runval.get(),
                                              c.cnt_nodes.get(), sys->col.get(), sys->val.get());
        exclusive_scan_i32(c.cnt_nodes.get(), sys->row_ptr.get(), n + 1, nullptr, c.scan_tmp32, s, c.launches);
        tr.mark("asm.sss");
        // Get_voltage_vector (Direct_Electrifying.cpp:1472-1500)
        std::vector<double> vef(reserved, 0.0);
        const double V = r_flag ? p.applied_voltage : (double)nodes;
        for (int i = 1; i < reserved; i++) vef[i] = vef[i - 1] + V;
        c.vef.ensure(8);
        CICY_CUDA(cudaMemcpyAsync(c.vef.get(), vef.data(), sizeof(double) * reserved, cudaMemcpyHostToDevice, s));
        CICY_CUDA(cudaMemsetAsync(sys->b.get(), 0, sizeof(double) * std::max(n, 1), s));
        k_rhs<<<grid_for(NE), 256, 0, s>>>(NE, bn, reserved, c.sort_k.get(), c.work_i32a.get(), c.runval.get(), c.vef.get(), sys->b.get());
        k_diag_free<<<grid_for(n), 256, 0, s>>>(n, reserved, c.work_f64a.get(), sys->diag.get(), c.status.get());
        c.launches += 3;
        try {
            check_status(c, "Fill_sparse_stiffness_matrix");
        } catch (Fail& f) {
            if (f.status == CICY_E_ZERO_DIAGONAL) {
                // name the nodes and values, as upstream prints them (Direct_Electrifying.cpp:458-484)
                std::vector<double> d(n);
                CICY_CUDA(cudaMemcpy(d.data(), sys->diag.get(), sizeof(double) * n, cudaMemcpyDeviceToHost));
                std::string nodes, vals;
                int shown = 0;
                for (int i = 0; i < n && shown < 8; i++)
                    if (std::fabs(d[i]) < 1.0e-10) {
                        nodes += " " + std::to_string(i + reserved);
                        char buf[32];
                        std::snprintf(buf, sizeof(buf), " %.3e", d[i]);
                        vals += buf;
                        shown++;
                    }
                f.msg += std::string(r_flag ? " (real-resistor pass" : " (unit-resistor pass") + "; nodes:" + nodes + "; values:" + vals + ")";
            }
            throw;
        }
        tr.mark(r_flag ? "dea.real.assembly" : "dea.unit.assembly");
        // ---- full CSR for the CG ----
        const int NF = n + 2 * m;
        const int bnf = bits_for((uint64_t)std::max(n, 1));
        c.sort_k.ensure(NF + 1);
        c.sort_v.ensure(NF + 1);
        c.cg_rp.ensure(n + 1); c.cg_ci.ensure(NF + 1); c.cg_val.ensure(NF + 1); c.cg_minv.ensure(n + 1);
        k_full_keys<<<grid_for(NF), 256, 0, s>>>(n, m, bnf, sys->row_ptr.get(), sys->col.get(), c.sort_k.get(), c.sort_v.get());
        radix_sort_pairs(c.sort_k.get(), c.sort_v.get(), NF, 2 * bnf, c.rs, s, c.launches);
        CICY_CUDA(cudaMemsetAsync(c.cnt_nodes.get(), 0, sizeof(int32_t) * (n + 1), s));
        k_full_fill<<<grid_for(NF), 256, 0, s>>>(n, m, bnf, c.sort_k.get(), c.sort_v.get(), sys->diag.get(), sys->val.get(), c.cnt_nodes.get(),
                                               c.cg_ci.get(), c.cg_val.get(), c.cg_minv.get());
        exclusive_scan_i32(c.cnt_nodes.get(), c.cg_rp.get(), n + 1, nullptr, c.scan_tmp32, s, c.launches);
        c.launches += 2;
        tr.mark(r_flag ? "dea.real.full_csr" : "dea.unit.full_csr");
        // ---- initial guess and r0 ----
        c.cg_x.ensure(n + 1); c.cg_r.ensure(n + 1); c.cg_z.ensure(n + 1); c.cg_p.ensure(n + 1); c.cg_q.ensure(n + 1);
        CICY_CUDA(cudaMemsetAsync(sys->x0.get(), 0, sizeof(double) * std::max(n, 1), s));
        if (r_flag && reserved == 2) {
            const cicy_cuboid& w = c.window;
            const double Lw = in.family == 0 ? w.len_x : in.family == 1 ? w.len_y : w.len_z;
            const double maxc = in.family == 0 ? w.max_x : in.family == 1 ? w.max_y : w.max_z;
            k_initial_guess<<<grid_for(NM), 256, 0, s>>>(NM, reserved, in.family, p.applied_voltage / Lw, maxc, eb.get(), ee.get(),
                                                       c.elem_idx.get(), c.lmm.get(), c.x.get(), c.y.get(), c.z.get(), sys->x0.get());
            c.launches++;
        }
        if (n > 0) {
            k_spmv_residual<<<grid_for(n), 256, 0, s>>>(n, c.cg_rp.get(), c.cg_ci.get(), c.cg_val.get(), sys->x0.get(), sys->b.get(), c.cg_r.get());
            CICY_CUDA(cudaMemcpyAsync(c.cg_x.get(), sys->x0.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
            c.launches++;
        }
        tr.mark(r_flag ? "dea.real.guess" : "dea.unit.guess");
        // ---- CG ----
        SolverSystem ss;
        ss.n = n;
        ss.nnz = NF;
        ss.rp = c.cg_rp.get();
        ss.ci = c.cg_ci.get();
        ss.val = c.cg_val.get();
        ss.diag = sys->diag.get();
        ss.b = sys->b.get();
        ss.x = c.cg_x.get();
        const bool mixed = c.solver.precision == CICY_PRECISION_MIXED;
        int kind = PRECOND_KIND_JACOBI;
        const float* ew = nullptr;
        if (c.solver.preconditioner == CICY_PRECOND_LEARNED && n > 0) {
            kind = PRECOND_KIND_SPAI;
            ew = learned_edge_weights(c, ss, NMc, s);
            tr.mark(r_flag ? "dea.real.gnn" : "dea.unit.gnn");
        } else if (c.solver.preconditioner != CICY_PRECOND_JACOBI && n > 0) {
            kind = PRECOND_KIND_BLOCK;
        }
        // host copy of the chains, for cicy_get_chains
        sys->h_chain_start.resize(NMc);
        sys->h_chain_len.resize(NMc);
        if (NMc > 0) {
            CICY_CUDA(cudaMemcpyAsync(sys->h_chain_start.data(), c.chain_start.get(), sizeof(int32_t) * NMc, cudaMemcpyDeviceToHost, s));
            CICY_CUDA(cudaMemcpyAsync(sys->h_chain_len.data(), c.chain_len.get(), sizeof(int32_t) * NMc, cudaMemcpyDeviceToHost, s));
        }
        PcgStats st;
        const double tol = (r_flag == 0 && p.tolerance_unit > 0) ? p.tolerance_unit : p.tolerance;
        const long long max_iter = (long long)c.solver.max_iter_factor * nodes;
        // small and medium systems: one cluster with everything in shared memory;
        // otherwise (or when disabled) the grid-wide persistent kernel
        bool solved = false;
        if (c.solver.preconditioner == CICY_PRECOND_MG && n > 0) {
            build_block_preconditioner(c.sw, ss, NMc, c.chain_start.get(), c.chain_len.get(), nullptr, nullptr, false, s, c.launches);
            tr.mark(r_flag ? "dea.real.blocks" : "dea.unit.blocks");
            build_mg_hierarchy(c.sw, ss, s, c.launches, mg_fused_path(n, !(c.solver.flags & CICY_SOLVER_NO_CLUSTER)),
                               !(c.solver.flags & CICY_SOLVER_NO_SMOOTHED), c.status.get());
            tr.mark(r_flag ? "dea.real.mg_setup" : "dea.unit.mg_setup");
            pcg_solve_mg(c.sw, ss, tol, max_iter, !(c.solver.flags & CICY_SOLVER_NO_CLUSTER), c.num_sms, c.status.get(), s, c.launches,
                         st);
            solved = true;
        }
        if (!solved && kind != PRECOND_KIND_SPAI && !mixed && !(c.solver.flags & CICY_SOLVER_NO_CLUSTER))
            solved = pcg_solve_cluster(c.sw, ss, kind == PRECOND_KIND_BLOCK, nullptr, nullptr, NMc, c.chain_start.get(), c.chain_len.get(),
                                       tol, max_iter, s, c.launches, st);
        if (!solved) {
            if (kind != PRECOND_KIND_JACOBI)
                build_block_preconditioner(c.sw, ss, NMc, c.chain_start.get(), c.chain_len.get(), nullptr, nullptr, mixed, s, c.launches);
            pcg_solve(c.sw, ss, kind, mixed, tol, max_iter, c.num_sms, c.status.get(), s, c.launches, st, ew);
        }
        check_status(c, "Solve_DEA_equations_CG_SSS");
        tr.mark(r_flag ? "dea.real.cg" : "dea.unit.cg");
        // true FP64 residual |b - A x| / |b|
        auto true_residual = [&]() {
            double rb[2] = {0, 0};
            if (n > 0) {
                c.cg_scal.ensure(4);
                CICY_CUDA(cudaMemsetAsync(c.cg_scal.get(), 0, sizeof(double) * 2, s));
                k_true_residual<<<grid_for(n), 256, 0, s>>>(n, c.cg_rp.get(), c.cg_ci.get(), c.cg_val.get(), c.cg_x.get(), sys->b.get(),
                                                          c.cg_scal.get());
                c.launches++;
                CICY_CUDA(cudaMemcpyAsync(rb, c.cg_scal.get(), sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
                CICY_CUDA(cudaStreamSynchronize(s));
            }
            return rb[1] > 0 ? std::sqrt(rb[0] / rb[1]) : 0.0;
        };
        double rel = true_residual();
        if (kind == PRECOND_KIND_SPAI && !(rel <= 10 * tol && st.iterations < max_iter)) {
            // the learned preconditioner did not reduce the residual: Jacobi-PCG from the initial guess
            const double seconds = st.seconds;
            CICY_CUDA(cudaMemcpyAsync(c.cg_x.get(), sys->x0.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
            pcg_solve(c.sw, ss, PRECOND_KIND_JACOBI, false, tol, max_iter, c.num_sms, c.status.get(), s, c.launches, st);
            check_status(c, "Solve_DEA_equations_CG_SSS (Jacobi fallback)");
            st.seconds += seconds;
            sys->fallback = 1;
            rel = true_residual();
        }
        sys->cluster_solver = st.cluster;
        sys->mg_levels = st.levels;
        sys->seconds = st.seconds;
        sys->iterations = st.iterations;
        sys->restarts = st.restarts;
        k_voltages<<<grid_for(nodes), 256, 0, s>>>(nodes, reserved, c.vef.get(), c.cg_x.get(), sys->volt.get());
        c.launches++;
        CICY_CUDA(cudaStreamSynchronize(s));
        sys->rel_residual = rel;
    } catch (...) {
        c.sys_pool.push_back(sys);
        throw;
    }
    return sys;
}

}  // namespace

// ---------------------------------------------------------------------------
// Electrical_analysis::Perform_analysis_on_clusters (Electrical_analysis.cpp:10-145).
void run_electrical(Ctx& c, const cicy_params& p, cicy_result* out) {
    if (c.stage < 3 || c.have_hybrid) throw Fail{CICY_E_STATE, "cicy_electrical_analysis: run cicy_clusters first"};
    cudaStream_t s = c.stream;
    for (auto* sy : c.systems) c.sys_pool.push_back(sy);
    c.systems.clear();
    const int NC = std::max(c.n_cnts, 1);
    // current elements_cnt state of every CNT: [lo, hi] into elem_idx
    c.bb_lo.ensure(NC);
    c.bb_hi.ensure(NC);
    k_init_ranges<<<grid_for(NC), 256, 0, s>>>(c.n_cnts, c.cstart.get(), c.clen.get(), c.mark_scan.get(), c.bb_lo.get(), c.bb_hi.get());
    c.launches++;
    // working copies of the percolated clusters and their junction lists (backbone shrinks them)
    const int n_clu_idx = c.h_clu_ptr.empty() ? 0 : c.h_clu_ptr.back();
    const int n_cj_idx = c.h_cj_ptr.empty() ? 0 : c.h_cj_ptr.back();
    c.bbclu_idx.ensure(std::max(n_clu_idx, 1));
    c.bbcj_idx.ensure(std::max(n_cj_idx, 1));
    if (n_clu_idx) CICY_CUDA(cudaMemcpyAsync(c.bbclu_idx.get(), c.clu_idx.get(), sizeof(int32_t) * n_clu_idx, cudaMemcpyDeviceToDevice, s));
    if (n_cj_idx) CICY_CUDA(cudaMemcpyAsync(c.bbcj_idx.get(), c.cj_idx.get(), sizeof(int32_t) * n_cj_idx, cudaMemcpyDeviceToDevice, s));
    c.h_bbclu_ptr = c.h_clu_ptr;
    c.h_bbcj_ptr = c.h_cj_ptr;
    std::vector<int32_t> clu_len(c.n_perc), cj_len(c.n_perc);
    for (int k = 0; k < c.n_perc; k++) {
        clu_len[k] = c.h_clu_ptr[k + 1] - c.h_clu_ptr[k];
        cj_len[k] = c.h_cj_ptr[k + 1] - c.h_cj_ptr[k];
    }
    std::vector<std::vector<double> > parallel(3);
    double t_unit = 0, t_bb = 0, t_real = 0;
    DBuf<int32_t>& eb = c.eb;
    DBuf<int32_t>& ee = c.ee;
    c.imax.ensure(1);
    c.alive.ensure(std::max(std::max(n_clu_idx, n_cj_idx), 1) + 1);
    c.alive_scan.ensure(std::max(std::max(n_clu_idx, n_cj_idx), 1) + 1);
    c.tmp_list.ensure(std::max(std::max(n_clu_idx, n_cj_idx), 1) + 1);
    c.cur_out.ensure(4);
    c.vol_acc.ensure(kVolWords);
    CICY_CUDA(cudaStreamWaitEvent(s, c.ev_side, 0));  // the previous step's side-stream volumes are done
    CICY_CUDA(cudaMemsetAsync(c.vol_acc.get(), 0, sizeof(double) * kVolWords, s));
    const int scope = p.simulation_scope;
    // Calculate_percolated_families_fractions' isolated-CNT volumes (Electrical_analysis.cpp:678-756) need
    // only the labels: on the side stream from here, beside the DEA passes
    CICY_CUDA(cudaEventRecord(c.ev_main, s));
    CICY_CUDA(cudaStreamWaitEvent(c.side, c.ev_main, 0));
    const bool fractions = scope < 2 && c.n_inside > 0;
    if (fractions) {
        cudaStream_t ss = c.side;
        c.vol_key.ensure(c.n_inside);
        c.vol_cnt.ensure(c.n_inside);
        k_isolated_keys<<<grid_for(c.n_inside), 256, 0, ss>>>(c.n_inside, c.n_labels, c.inside.get(), c.labels.get(), c.perc_bits.get(),
                                                              c.vol_key.get(), c.vol_cnt.get());
        radix_sort_pairs(c.vol_key.get(), c.vol_cnt.get(), c.n_inside, bits_for((uint64_t)(c.n_labels + 2) * (uint64_t)c.n_inside),
                         c.rs_side, ss, c.launches);
        c.vol_iso.ensure(c.n_inside);
        CICY_CUDA(cudaMemsetAsync(c.i32_scalar.get() + 2, 0, sizeof(int32_t), ss));
        k_isolated_volumes<<<grid_for(c.n_inside), 256, 0, ss>>>(c.n_inside, (uint64_t)(c.n_labels + 1) * (uint64_t)c.n_inside,
                                                                 c.vol_key.get(), c.vol_cnt.get(), c.cstart.get(), c.clen.get(),
                                                                 c.radii.get(), c.x.get(), c.y.get(), c.z.get(), c.vol_iso.get(),
                                                                 c.i32_scalar.get() + 2);
        c.launches += 2;
    }
    CICY_CUDA(cudaEventRecord(c.ev_side, c.side));
    for (int k = 0; k < c.n_perc && scope < 2; k++) {
        int32_t* members = c.bbclu_idx.get() + c.h_clu_ptr[k];
        int32_t* jl = c.bbcj_idx.get() + c.h_cj_ptr[k];
        SolveInput u{k, -1, c.h_family[k], members, clu_len[k], jl, cj_len[k]};
        DeaSystem* su = solve_dea(c, p, u, eb, ee);
        c.systems.push_back(su);
        t_unit += su->seconds;
        TraceSeq trb(s);
        // ---- backbone ----
        cudaEvent_t e0, e1;
        CICY_CUDA(cudaEventCreate(&e0));
        CICY_CUDA(cudaEventCreate(&e1));
        CICY_CUDA(cudaEventRecord(e0, s));
        const int NM = clu_len[k], NJ = cj_len[k];
        CICY_CUDA(cudaMemsetAsync(c.imax.get(), 0, sizeof(unsigned long long), s));
        k_current_max<<<grid_for(NM + NJ), 256, 0, s>>>(NM, eb.get(), ee.get(), c.elem_idx.get(), c.lmm.get(), su->volt.get(), NJ, jl,
                                                      c.j_p1.get(), c.j_p2.get(), c.imax.get());
        c.vol3.ensure(3 * (size_t)std::max(NM, 1));
        c.vol_kind.ensure(std::max(NM, 1));
        c.bb_pts.ensure(5 * (size_t)std::max(NM, 1));
        CICY_CUDA(cudaStreamWaitEvent(s, c.ev_side, 0));  // the side stream's previous volumes have read bb_pts
        k_backbone_scan<<<grid_for(NM), 256, 0, s>>>(NM, members, eb.get(), ee.get(), c.elem_idx.get(), c.lmm.get(), su->volt.get(),
                                                   c.imax.get(), scope == 0 ? 1 : 0, c.bb_lo.get(), c.bb_hi.get(), c.alive.get(),
                                                   c.bb_pts.get());
        // the volumes (read by no later stage of the step) beside the real-resistor pass
        CICY_CUDA(cudaEventRecord(c.ev_main, s));
        CICY_CUDA(cudaStreamWaitEvent(c.side, c.ev_main, 0));
        k_backbone_volumes<<<grid_for(NM), 256, 0, c.side>>>(NM, c.bb_pts.get(), c.radii.get(), c.x.get(), c.y.get(), c.z.get(), c.vol3.get(),
                                                            c.vol_kind.get());
        k_volume_sum<<<1, kSumThreads, 0, c.side>>>(NM, c.h_family[k], c.vol3.get(), c.vol_kind.get(), c.vol_acc.get());
        CICY_CUDA(cudaEventRecord(c.ev_side, c.side));
        c.launches += 3;
        if (scope == 0) {
            exclusive_scan_i32(c.alive.get(), c.alive_scan.get(), NM, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
            k_compact_i32<<<grid_for(NM), 256, 0, s>>>(NM, members, c.alive.get(), c.alive_scan.get(), c.tmp_list.get());
            c.launches++;
            int nm2 = read_i32(c, c.i32_scalar.get());
            if (nm2) CICY_CUDA(cudaMemcpyAsync(members, c.tmp_list.get(), sizeof(int32_t) * nm2, cudaMemcpyDeviceToDevice, s));
            clu_len[k] = nm2;
            if (NJ > 0) {
                k_junction_alive<<<grid_for(NJ), 256, 0, s>>>(NJ, jl, c.j_p1.get(), c.j_n1.get(), c.j_p2.get(), c.j_n2.get(), c.bb_lo.get(),
                                                            c.bb_hi.get(), c.mark_scan.get(), c.alive.get());
                exclusive_scan_i32(c.alive.get(), c.alive_scan.get(), NJ, c.i32_scalar.get(), c.scan_tmp32, s, c.launches);
                k_compact_i32<<<grid_for(NJ), 256, 0, s>>>(NJ, jl, c.alive.get(), c.alive_scan.get(), c.tmp_list.get());
                c.launches += 2;
                int nj2 = read_i32(c, c.i32_scalar.get());
                if (nj2) CICY_CUDA(cudaMemcpyAsync(jl, c.tmp_list.get(), sizeof(int32_t) * nj2, cudaMemcpyDeviceToDevice, s));
                cj_len[k] = nj2;
            }
        }
        CICY_CUDA(cudaEventRecord(e1, s));
        CICY_CUDA(cudaEventSynchronize(e1));
        t_bb += seconds_between(e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (trace_enabled()) {
            unsigned long long bits = 0;
            CICY_CUDA(cudaMemcpy(&bits, c.imax.get(), sizeof(bits), cudaMemcpyDeviceToHost));
            double im;
            std::memcpy(&im, &bits, sizeof(im));
            std::fprintf(stderr, "[cicy] backbone cluster %d: I_max %.17g, zero current %.17g, CNTs %d, junctions %d\n", k, im,
                         std::max(im, kZero) * 1e-9, NM, NJ);
        }
        if (scope != 0) continue;
        trb.mark("backbone");
        // ---- real-resistor passes per percolated direction (Electrical_analysis.cpp:229-289) ----
        std::vector<int> dirs;
        const int fam = c.h_family[k];
        const int dir_bits[7] = {1, 2, 4, 3, 5, 6, 7};
        for (int d = 0; d < 3; d++)
            if ((dir_bits[fam] >> d & 1) && p.resistances[d]) dirs.push_back(d);
        for (int d : dirs) {
            SolveInput r{k, d, d, members, clu_len[k], jl, cj_len[k]};
            DeaSystem* sr = solve_dea(c, p, r, eb, ee);
            c.systems.push_back(sr);
            t_real += sr->seconds;
            // Calculate_parallel_resistor (Electrical_analysis.cpp:355-473)
            const int b1 = d == 0 ? 2 : d == 1 ? 3 : 0;
            const int b2 = d == 0 ? 4 : d == 1 ? 5 : 1;
            if (c.h_bcnt_ptr[b1 + 1] == c.h_bcnt_ptr[b1] || c.h_bcnt_ptr[b2 + 1] == c.h_bcnt_ptr[b2])
                throw Fail{CICY_E_INPUT, "Calculate_parallel_resistor: one boundary vector along the direction is empty"};
            const int nb = (int)(c.h_bcnt_ptr[b1 + 1] - c.h_bcnt_ptr[b1]);
            c.bterm.ensure(2 * (size_t)nb);
            c.bvalid.ensure(2 * (size_t)nb);
            k_boundary_terms<<<grid_for(2 * nb), 128, 0, s>>>((int)c.h_bcnt_ptr[b1], (int)c.h_bcnt_ptr[b1 + 1], c.bcnt_idx.get(),
                                                             c.bb_lo.get(), c.bb_hi.get(), c.elem_idx.get(), c.lmm.get(), sr->volt.get(),
                                                             c.radii.get(), p.resistivity_cnt, c.x.get(), c.y.get(), c.z.get(),
                                                             c.bterm.get(), c.bvalid.get());
            k_boundary_sum<<<1, kSumThreads, 0, s>>>(2 * nb, c.bterm.get(), c.bvalid.get(), c.cur_out.get());
            c.launches += 2;
            double I = 0;
            CICY_CUDA(cudaMemcpyAsync(&I, c.cur_out.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
            CICY_CUDA(cudaStreamSynchronize(s));
            parallel[d].push_back(p.applied_voltage / I);
            trb.mark("boundary_current");
        }
    }
    c.h_bbclu_ptr.assign(c.n_perc + 1, 0);
    c.h_bbcj_ptr.assign(c.n_perc + 1, 0);
    for (int k = 0; k < c.n_perc; k++) {
        c.h_bbclu_ptr[k + 1] = c.h_bbclu_ptr[k] + clu_len[k];
        c.h_bbcj_ptr[k + 1] = c.h_bbcj_ptr[k] + cj_len[k];
    }
    c.bb_clu_len = clu_len;
    c.bb_cj_len = cj_len;
    c.have_backbone = true;
    // Calculate_percolated_families_fractions (Electrical_analysis.cpp:114-119, 678-756)
    if (fractions) {
        k_family_fractions<<<1, kSumThreads, 0, c.side>>>(c.i32_scalar.get() + 2, c.vol_iso.get(), c.vol_acc.get());
        c.launches++;
        c.have_volumes = true;
    }
    // the main stream (and so every later read of the volumes) waits for the side stream's work
    CICY_CUDA(cudaEventRecord(c.ev_side, c.side));
    CICY_CUDA(cudaStreamWaitEvent(s, c.ev_side, 0));
    // Calculate_resistances_and_resistivities (Electrical_analysis.cpp:873-987)
    if (out) {
        const cicy_cuboid& w = c.window;
        const double L[3] = {w.len_x, w.len_y, w.len_z};
        const double A[3] = {w.len_y * w.len_z, w.len_x * w.len_z, w.len_x * w.len_y};
        for (int d = 0; d < 3; d++) {
            double R;
            if (parallel[d].empty()) {
                out->resistivities[d] = p.resistivity_matrix;
                R = p.resistivity_matrix * L[d] / A[d];
                out->resistances[d] = R;
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
        out->n_percolated = c.n_perc;
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

// The GNP branch of the DEA for mixed CNT/GNP networks (same translation unit).
#include "hybrid_dea.cuh"
