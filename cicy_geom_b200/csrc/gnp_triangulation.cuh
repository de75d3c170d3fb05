// Triangulation of one GNP's points, host and device:
// Triangulation::Generate_3d_trangulation (Triangulation.cpp:12-477).  Four
// points or fewer give all pairs; more are projected onto the GNP's mid-plane
// along face 0's normal and triangulated by Bowyer-Watson from a supertriangle
// rotated into the GNP's frame: for each point in list order the triangles
// whose circumcircle holds it (scanned last to first, erased in place) leave
// their edges, the edges that occur once make new triangles with the point,
// and the final edges are those of triangles between real points, first
// occurrences only.  Every branch and FP64 operation follows upstream's order;
// built without FMA contraction, host and device give upstream's edges.
// Fixed capacities replace upstream's vectors: at most MAXP points.
#pragma once

#include <cmath>

#include "gnp_geom.cuh"

namespace cicy {
namespace gnp {

template <int MAXP>
struct TriWork {
    static constexpr int kTris = 2 * MAXP + 1;  // a planar triangulation of n points and the supertriangle
    P3 plane[MAXP];
    P3 sv[3];
    int tri[kTris][3];
    int edge[3 * kTris][2];
    int rep[3 * kTris];
};

// Calculate_circumcenter: ((Q Pn - P Qn) x R) / (2 Rn) + P3, P = P1 - P3, Q = P2 - P3, R = P x Q.
__host__ __device__ inline P3 circumcenter(const P3& P1, const P3& P2, const P3& P3v) {
    const P3 P = sub(P1, P3v), Q = sub(P2, P3v);
    const P3 R = cross(P, Q);
    const double Pn = dot(P, P), Qn = dot(Q, Q), Rn = dot(R, R);
    const P3 a{Q.x * Pn - P.x * Qn, Q.y * Pn - P.y * Qn, Q.z * Pn - P.z * Qn};
    const P3 c = cross(a, R);
    const double den = 2 * Rn;
    return P3{c.x / den + P3v.x, c.y / den + P3v.y, c.z / den + P3v.z};
}

__host__ __device__ inline double sqdist(const P3& a, const P3& b) {
    const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return dx * dx + dy * dy + dz * dz;
}

__host__ __device__ inline bool same_edge(const int a[2], int u, int v) { return (a[0] == u && a[1] == v) || (a[0] == v && a[1] == u); }

// Edges of the GNP whose point numbers are structure[0..n) (coordinates in
// points[3 P]), side l, centre c, row-major rotation M and face-0 normal N0,
// written as global point pairs into out[2 k]; returns the edge count, or -1
// when n exceeds MAXP or the edges exceed `cap`.
template <int MAXP>
__host__ __device__ inline int triangulate(const double* points, const int* structure, int n, double l, const double* c, const double* M, const P3& N0,
                                           TriWork<MAXP>& w, int* out, int cap) {
    if (n <= 4) {  // Generate_trivial_triangulation
        int k = 0;
        for (int i = 0; i < n - 1; i++)
            for (int j = i + 1; j < n; j++) {
                if (k >= cap) return -1;
                out[2 * k] = structure[i];
                out[2 * k + 1] = structure[j];
                k++;
            }
        return k;
    }
    if (n > MAXP) return -1;
    const P3 c0{c[0], c[1], c[2]};
    for (int i = 0; i < n; i++) {  // Points_on_midplane
        const P3 p{points[3 * (size_t)structure[i]], points[3 * (size_t)structure[i] + 1], points[3 * (size_t)structure[i] + 2]};
        const double d = dot(sub(p, c0), N0);
        w.plane[i] = P3{p.x - N0.x * d, p.y - N0.y * d, p.z - N0.z * d};
    }
    const double s3 = sqrt(3.0);  // Generate_supertriangle, then Point_3D::rotation
    const double loc[3][3] = {{0.0, ((0.75 * s3) + 0.5) * l, 0.0}, {(0.75 + (0.5 * s3)) * l, -l, 0.0}, {-((0.75 + (0.5 * s3)) * l), -l, 0.0}};
    for (int v = 0; v < 3; v++) {
        const double* p = loc[v];
        w.sv[v] = P3{M[0] * p[0] + M[1] * p[1] + M[2] * p[2] + c0.x, M[3] * p[0] + M[4] * p[1] + M[5] * p[2] + c0.y,
                     M[6] * p[0] + M[7] * p[1] + M[8] * p[2] + c0.z};
    }
    auto pt = [&](int i) -> const P3& { return i >= 0 ? w.plane[i] : w.sv[-1 - i]; };
    int nt = 1;
    w.tri[0][0] = -1;
    w.tri[0][1] = -2;
    w.tri[0][2] = -3;
    for (int v = 0; v < n; v++) {
        int nb = 0;
        for (int j = nt - 1; j >= 0; j--) {  // Find_bad_triangles
            const int* t = w.tri[j];
            const P3 C = circumcenter(pt(t[0]), pt(t[1]), pt(t[2]));
            if (sqdist(C, w.plane[v]) - sqdist(C, pt(t[0])) <= kZero) {
                if (nb + 3 > 3 * TriWork<MAXP>::kTris) return -1;
                for (int e = 0; e < 3; e++) {
                    w.edge[nb][0] = t[e];
                    w.edge[nb][1] = t[(e + 1) % 3];
                    nb++;
                }
                for (int k = j; k + 1 < nt; k++)
                    for (int e = 0; e < 3; e++) w.tri[k][e] = w.tri[k + 1][e];
                nt--;
            }
        }
        for (int j = 0; j < nb; j++) w.rep[j] = 0;  // Add_new_triangles
        for (int j = 0; j + 1 < nb; j++)
            for (int k = j + 1; k < nb; k++)
                if (same_edge(w.edge[j], w.edge[k][0], w.edge[k][1])) {
                    w.rep[j]++;
                    w.rep[k]++;
                }
        for (int j = 0; j < nb; j++)
            if (!w.rep[j]) {
                if (nt >= TriWork<MAXP>::kTris) return -1;
                w.tri[nt][0] = w.edge[j][0];
                w.tri[nt][1] = w.edge[j][1];
                w.tri[nt][2] = v;
                nt++;
            }
    }
    int ne = 0;  // Final_triangulation_edges
    for (int i = 0; i < nt; i++)
        for (int e = 0; e < 3; e++) {
            const int a = w.tri[i][e], b = w.tri[i][(e + 1) % 3];
            if (a >= 0 && b >= 0) {
                w.edge[ne][0] = a;
                w.edge[ne][1] = b;
                ne++;
            }
        }
    int k = 0;
    for (int i = 0; i < ne; i++) {
        bool seen = false;
        for (int j = 0; j < i && !seen; j++) seen = same_edge(w.edge[j], w.edge[i][0], w.edge[i][1]);
        if (seen) continue;
        if (k >= cap) return -1;
        out[2 * k] = structure[w.edge[i][0]];  // Update_edge_numbers
        out[2 * k + 1] = structure[w.edge[i][1]];
        k++;
    }
    return k;
}

}  // namespace gnp
}  // namespace cicy
