// Junction points of two GNPs in contact, host and device:
// Hoshen_Kopelman::Find_junction_points_for_gnps and the functions it calls
// (Hoshen_Kopelman.cpp:826-1825): the vertices of each GNP on the closest
// features (|Q.N| within 1e-10 of the distance over the 64 vertex
// differences Q), then the vertex / edge / face case analysis that places
// one point on each GNP.  Every branch and FP64 operation follows upstream's
// order; built without FMA contraction, host and device give upstream's
// doubles.  A GNP here is its 8 vertices and the unit normals of its 6 faces.
#pragma once

#include <cmath>

#include "gnp_geom.cuh"

namespace cicy {
namespace gnp {

constexpr int kJuncOk = 0;
constexpr int kJuncBadSimplex = 1;     // closest-feature vertex counts upstream rejects
constexpr int kJuncNoIntersection = 2; // an edge / face-edge intersection outside [0, 1]
constexpr int kJuncNoInsideVertex = 3; // face-face contact with no vertex inside the other face
constexpr int kJuncNoEdge = 4;         // Average_point_with_two_interserctions found no edge
constexpr int kJuncBadFace = 5;        // a vertex sum that names no face

struct Cuboid8 {
    P3 v[8];
    P3 n[6];  // Plane_3D::N of each face
};

__host__ __device__ inline P3 add(const P3& a, const P3& b) { return P3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline P3 divide(const P3& a, double s) { return P3{a.x / s, a.y / s, a.z / s}; }

// A GNP as read: vertices and the normals of its face planes (n = plane coefficients 0..2).
__host__ __device__ inline void load_cuboid(const double* V, const double* F, Cuboid8& g) {
    for (int i = 0; i < 8; i++) g.v[i] = vertex(V, i);
    for (int f = 0; f < 6; f++) g.n[f] = normal(F, f);
}

// Generate_Network::Move_gnp: vertices moved by d, faces rebuilt from them
// (Update_gnp_plane_equations: Plane_3D through three vertices, unit normal).
__host__ __device__ inline void moved_cuboid(const double* V, const P3& d, Cuboid8& g) {
    for (int i = 0; i < 8; i++) g.v[i] = add(vertex(V, i), d);
    const int T[6][3] = {{0, 1, 3}, {4, 7, 5}, {0, 3, 4}, {0, 4, 1}, {1, 5, 2}, {2, 6, 3}};
    for (int f = 0; f < 6; f++) {
        const P3 c = cross(sub(g.v[T[f][1]], g.v[T[f][0]]), sub(g.v[T[f][2]], g.v[T[f][0]]));
        const double l = sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
        g.n[f] = P3{c.x / l, c.y / l, c.z / l};
    }
}

// Lambda_of_two_lines (:1529-1540)
__host__ __device__ inline double lambda_lines(const P3& Pin, const P3& Pout, const P3& e1, const P3& e2) {
    const double detA = (e2.x - e1.x) * (Pin.y - Pout.y) - (Pin.x - Pout.x) * (e2.y - e1.y);
    const double detAP = (e2.x - e1.x) * (e1.y - Pout.y) - (e1.x - Pout.x) * (e2.y - e1.y);
    return detAP / detA;
}

// Get_edges_of_face (:1330-1426): the face named by its vertex sum (vertex 0
// counted as 1), its 4 edges and the face normal bounding each edge.
__host__ __device__ inline bool face_edges(int face_sum, int e[4][2], int nrm[4]) {
    int a[8], b[4];
    switch (face_sum) {
        case 7: { const int t[8] = {0, 3, 0, 1, 1, 2, 2, 3}; const int u[4] = {2, 3, 4, 5}; for (int i = 0; i < 8; i++) a[i] = t[i]; for (int i = 0; i < 4; i++) b[i] = u[i]; break; }
        case 22: { const int t[8] = {4, 7, 4, 5, 5, 6, 6, 7}; const int u[4] = {2, 3, 4, 5}; for (int i = 0; i < 8; i++) a[i] = t[i]; for (int i = 0; i < 4; i++) b[i] = u[i]; break; }
        case 15: { const int t[8] = {0, 3, 3, 7, 7, 4, 0, 4}; const int u[4] = {0, 5, 1, 3}; for (int i = 0; i < 8; i++) a[i] = t[i]; for (int i = 0; i < 4; i++) b[i] = u[i]; break; }
        case 11: { const int t[8] = {1, 0, 0, 4, 4, 5, 5, 1}; const int u[4] = {0, 2, 1, 4}; for (int i = 0; i < 8; i++) a[i] = t[i]; for (int i = 0; i < 4; i++) b[i] = u[i]; break; }
        case 14: { const int t[8] = {1, 2, 2, 6, 6, 5, 5, 1}; const int u[4] = {0, 5, 1, 3}; for (int i = 0; i < 8; i++) a[i] = t[i]; for (int i = 0; i < 4; i++) b[i] = u[i]; break; }
        case 18: { const int t[8] = {2, 3, 3, 7, 7, 6, 6, 2}; const int u[4] = {0, 2, 1, 4}; for (int i = 0; i < 8; i++) a[i] = t[i]; for (int i = 0; i < 4; i++) b[i] = u[i]; break; }
        default: return false;
    }
    for (int i = 0; i < 4; i++) {
        e[i][0] = a[2 * i];
        e[i][1] = a[2 * i + 1];
        nrm[i] = b[i];
    }
    return true;
}

// Get_intersection_with_face_edge (:1428-1527)
__host__ __device__ inline bool face_edge_cut(int count, const int arr[2], const P3& A0, const P3& A1, const int e[4][2], const Cuboid8& B,
                                              P3& P) {
    if (count == 4) {
        P = A0;
        return true;
    }
    double lambda;
    if (count == 3) {
        lambda = lambda_lines(A0, A1, B.v[e[arr[0]][0]], B.v[e[arr[0]][1]]);
        if ((lambda < kZero && fabs(lambda) > kZero) || lambda > 1.0) return false;
    } else if (count == 2) {
        lambda = lambda_lines(A0, A1, B.v[e[arr[0]][0]], B.v[e[arr[0]][1]]);
        if (lambda < kZero && fabs(lambda) > kZero) {
            lambda = lambda_lines(A0, A1, B.v[e[arr[1]][0]], B.v[e[arr[1]][1]]);
            if ((lambda < kZero && fabs(lambda) > kZero) || lambda > 1.0) return false;
        }
    } else {
        return false;
    }
    P = add(A1, scale(sub(A0, A1), lambda));
    return true;
}

// Find_point_for_edge_edge_contact (:1187-1262)
__host__ __device__ inline void edge_edge(const Cuboid8& B, const P3 edgeA[2], const int* sB, const P3& disp, P3& PA, P3& PB) {
    const P3 eA = sub(edgeA[1], edgeA[0]);
    const P3 eB = sub(B.v[sB[1]], B.v[sB[0]]);
    const P3 cr = cross(eA, eB);
    if (fabs(cr.x) < kZero && fabs(cr.y) < kZero && fabs(cr.z) < kZero) {
        const double l0 = (B.v[sB[0]].x - edgeA[0].x) / (edgeA[1].x - edgeA[0].x);
        const double l1 = (B.v[sB[1]].x - edgeA[0].x) / (edgeA[1].x - edgeA[0].x);
        if ((fabs(l0) < kZero && fabs(l1 - 1) < kZero) || (fabs(l1) < kZero && fabs(l0 - 1) < kZero))
            PB = divide(add(B.v[sB[0]], B.v[sB[1]]), 2.0);
        if (l0 >= kZero && l0 - 1 <= kZero) {
            const P3 S0 = add(edgeA[0], scale(eA, l0));
            PB = l1 < kZero ? divide(add(edgeA[0], S0), 2.0) : divide(add(edgeA[1], S0), 2.0);
        } else {
            const P3 S1 = add(edgeA[0], scale(eA, l1));
            PB = l0 < kZero ? divide(add(edgeA[0], S1), 2.0) : divide(add(edgeA[1], S1), 2.0);
        }
    } else {
        const double l = lambda_lines(B.v[sB[1]], B.v[sB[0]], edgeA[0], edgeA[1]);
        PB = add(B.v[sB[0]], scale(eB, l));
    }
    PA = sub(PB, disp);
}

// Find_point_for_edge_face_contact (:1264-1328)
__host__ __device__ inline int edge_face(int face_sum, const Cuboid8& B, const P3 edgeA[2], const P3& disp, P3& PA, P3& PB) {
    int e[4][2], nrm[4];
    if (!face_edges(face_sum, e, nrm)) return kJuncBadFace;
    int c0 = 0, c1 = 0, arr0[2] = {-1, -1}, arr1[2] = {-1, -1};
    for (int i = 0; i < 4; i++) {
        const P3& v1 = B.v[e[i][0]];
        const P3& n = B.n[nrm[i]];
        if (dot(sub(edgeA[0], v1), n) < kZero) c0++;
        else if (arr0[0] == -1) arr0[0] = i;
        else arr0[1] = i;
        if (dot(sub(edgeA[1], v1), n) < kZero) c1++;
        else if (arr1[0] == -1) arr1[0] = i;
        else arr1[1] = i;
    }
    P3 A0, A1;
    if (!face_edge_cut(c0, arr0, edgeA[0], edgeA[1], e, B, A0)) return kJuncNoIntersection;
    if (!face_edge_cut(c1, arr1, edgeA[1], edgeA[0], e, B, A1)) return kJuncNoIntersection;
    PB = scale(add(A0, A1), 0.5);
    PA = sub(PB, disp);
    return kJuncOk;
}

// Get_vertices_inside_face (:1687-1720): vertices of sA on the inner side of all 4 edges of face B.
__host__ __device__ inline int inside_face(const int* sA, int nA, const int eB[4][2], const int nB[4], const Cuboid8& A, const Cuboid8& B,
                                           int* out) {
    int k = 0;
    for (int j = 0; j < nA; j++) {
        int count = 0;
        for (int i = 0; i < 4; i++)
            if (dot(sub(A.v[sA[j]], B.v[eB[i][0]]), B.n[nB[i]]) < kZero) count++;
        if (count == 4) out[k++] = sA[j];
    }
    return k;
}

// Average_point_with_two_interserctions (:1722-1778)
__host__ __device__ inline bool average_two_cuts(const int eA[4][2], const int nA[4], const Cuboid8& A, const int eB[4][2], const Cuboid8& B,
                                                 const P3& disp, int vB, P3& PB) {
    int w[2] = {0, 0}, it = 0;
    for (int i = 0; i < 4; i++) {
        if (eB[i][0] == vB) {
            if (it < 2) w[it] = eB[i][1];
            it++;
        } else if (eB[i][1] == vB) {
            if (it < 2) w[it] = eB[i][0];
            it++;
        }
    }
    int v1 = 0, v2 = -1;
    for (int i = 0; i < 4; i++) {
        v1 = eA[i][0];
        const P3& n = A.n[nA[i]];
        if (dot(sub(B.v[w[0]], A.v[v1]), n) > kZero && dot(sub(B.v[w[1]], A.v[v1]), n) > kZero) {
            v2 = eA[i][1];
            break;
        }
    }
    if (v2 == -1) return false;
    const P3 a1 = sub(A.v[v1], disp), a2 = sub(A.v[v2], disp);
    const double l0 = lambda_lines(PB, B.v[w[0]], a1, a2);
    const double l1 = lambda_lines(PB, B.v[w[1]], a1, a2);
    PB = add(PB, add(B.v[w[0]], scale(sub(PB, B.v[w[0]]), l0)));
    PB = add(PB, add(B.v[w[1]], scale(sub(PB, B.v[w[1]]), l1)));
    PB = divide(PB, 3.0);
    return true;
}

// Find_point_b_for_face_in_simplex_a (:1542-1685)
__host__ __device__ inline int face_face(const int* sA, const int* sB, int nB, int sumA, int sumB, const Cuboid8& A, const Cuboid8& B, const P3& N,
                                         double distance, P3& PA, P3& PB) {
    if (nB != 4) return kJuncBadSimplex;
    int eB[4][2], nrmB[4];
    if (!face_edges(sumB, eB, nrmB)) return kJuncBadFace;
    int inA[4];
    const int kA = inside_face(sA, 4, eB, nrmB, A, B, inA);
    if (kA == 0) return kJuncNoInsideVertex;
    if (kA == 4) {
        PA = P3{0.0, 0.0, 0.0};
        PB = P3{0.0, 0.0, 0.0};
        for (int k = 0; k < nB; k++) {
            PA = add(PA, A.v[sA[k]]);
            PB = add(PB, B.v[sB[k]]);
        }
        PA = divide(PA, 4.0);
        PB = divide(PB, 4.0);
        return kJuncOk;
    }
    int eA[4][2], nrmA[4];
    if (!face_edges(sumA, eA, nrmA)) return kJuncBadFace;
    int inB[4];
    const int kB = inside_face(sB, 4, eA, nrmA, B, A, inB);
    if (kB == 0) return kJuncNoInsideVertex;
    const P3 disp = scale(N, distance);
    if (kA == 0 && kB == 1) {  // not reached: kA > 0 here, as upstream's checks leave it
        PB = B.v[inB[0]];
        if (!average_two_cuts(eA, nrmA, A, eB, B, disp, inB[0], PB)) return kJuncNoEdge;
        PA = sub(PB, disp);
    } else if (kA == 1 && kB == 0) {  // not reached either; upstream passes face B's edges twice here
        PA = A.v[inA[0]];
        if (!average_two_cuts(eB, nrmB, B, eB, B, scale(disp, -1.0), inA[0], PA)) return kJuncNoEdge;
        PB = add(PA, disp);
    } else {
        PB = P3{0.0, 0.0, 0.0};
        for (int k = 0; k < kA; k++) PB = add(add(PB, A.v[inA[k]]), disp);
        for (int k = 0; k < kB; k++) PB = add(PB, B.v[inB[k]]);
        PB = divide(PB, (double)(kA + kB));
        PA = sub(PB, disp);
    }
    return kJuncOk;
}

// Find_junction_points_in_gnps (:1049-1111) for simplex sizes nA <= nB.
__host__ __device__ inline int junction_in(const int* sA, int nA, const int* sB, int nB, const Cuboid8& A, const Cuboid8& B, const P3& N,
                                           double distance, int sumA, int sumB, P3& PA, P3& PB) {
    if (nA == 1) {
        PA = A.v[sA[0]];
        if (nB == 1) PB = B.v[sB[0]];
        else if (nB == 2 || nB == 4) PB = add(PA, scale(N, distance));
        else return kJuncBadSimplex;
        return kJuncOk;
    }
    if (nA == 2) {
        const P3 disp = scale(N, distance);
        const P3 edgeA[2] = {add(A.v[sA[0]], disp), add(A.v[sA[1]], disp)};
        if (nB == 2) {
            edge_edge(B, edgeA, sB, disp, PA, PB);
            return kJuncOk;
        }
        if (nB == 4) return edge_face(sumB, B, edgeA, disp, PA, PB);
        return kJuncBadSimplex;
    }
    if (nA == 4) return face_face(sA, sB, nB, sumA, sumB, A, B, N, distance, PA, PB);
    return kJuncBadSimplex;
}

// Complete_simplex_of_size_three (:968-1047): the fourth vertex of the face
// through three vertices i < j < k, or -1.
__host__ __device__ inline int fourth_vertex(int i, int j, int k) {
    const int key = 100 * i + 10 * j + k;
    const int T[24][2] = {{12, 3},  {13, 2},  {23, 1},  {123, 0}, {456, 7}, {457, 6}, {467, 5}, {567, 4},
                          {14, 5},  {15, 4},  {45, 1},  {145, 0}, {125, 6}, {126, 5}, {156, 2}, {256, 1},
                          {236, 7}, {237, 6}, {267, 3}, {367, 2}, {34, 7},  {37, 4},  {47, 3},  {347, 0}};
    for (int t = 0; t < 24; t++)
        if (T[t][0] == key) return T[t][1];
    return -1;
}

// A face's three closest vertices completed to its four (allow_simplex3); false
// when the three name no face.
__host__ __device__ inline bool complete_three(bool in[8]) {
    int t[3], c = 0;
    for (int i = 0; i < 8; i++)
        if (in[i]) {
            if (c < 3) t[c] = i;
            c++;
        }
    if (c != 3) return true;
    const int v = fourth_vertex(t[0], t[1], t[2]);
    if (v < 0) return false;
    in[v] = true;
    return true;
}

// Find_junction_points_for_gnps (:826-857) with Find_closest_simplices_of_gnps_in_contact
// (:860-966): A and B as placed (B already moved apart when they interpenetrated),
// N and distance from the GNP-GNP distance step.
__host__ __device__ inline int junction_points(const Cuboid8& A, const Cuboid8& B, const P3& N, double distance, bool allow_simplex3, P3& PA,
                                               P3& PB) {
    bool inA[8] = {false, false, false, false, false, false, false, false};
    bool inB[8] = {false, false, false, false, false, false, false, false};
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) {
            const P3 Q = sub(A.v[i], B.v[j]);
            if (fabs(fabs(dot(Q, N)) - distance) <= kZero) {
                inA[i] = true;
                inB[j] = true;
            }
        }
    if (allow_simplex3 && (!complete_three(inA) || !complete_three(inB))) return kJuncBadSimplex;
    int sA[4], sB[4], nA = 0, nB = 0, cA = 0, cB = 0;
    for (int i = 0; i < 8; i++) {
        cA += inA[i];
        cB += inB[i];
    }
    if (cA > 4 || cB > 4) return kJuncBadSimplex;  // upstream rejects every size but 1, 2 and 4
    int sumA = 0, sumB = 0;
    for (int i = 0; i < 8; i++) {
        if (inA[i]) {
            sA[nA++] = i;
            sumA += i > 1 ? i : 1;
        }
        if (inB[i]) {
            sB[nB++] = i;
            sumB += i > 1 ? i : 1;
        }
    }
    if (nA <= nB) return junction_in(sA, nA, sB, nB, A, B, N, distance, sumA, sumB, PA, PB);
    return junction_in(sB, nB, sA, nA, B, A, scale(N, -1.0), distance, sumB, sumA, PB, PA);
}

// Point_3D::is_outside_cuboid (Geometry_3D.cpp:227-235) for a cuboid given by its min and max corners.
__host__ __device__ inline bool outside_box(const P3& p, const double lo[3], const double hi[3]) {
    return (p.x - lo[0] < kZero) || (p.x - hi[0] > kZero) || (p.y - lo[1] < kZero) || (p.y - hi[1] > kZero) || (p.z - lo[2] < kZero) ||
           (p.z - hi[2] > kZero);
}

}  // namespace gnp
}  // namespace cicy
