// Distance between two GNPs (cuboids given by their 8 vertices), host and
// device: the GJK distance of Collision_detection::GJK_distance with its
// simplex bookkeeping (Direction_from_simplex_to_origin,
// Is_point_contained_in_simplex, Distance_from_simplex_to_origin,
// Find_voroni_region and its 3- and 4-vertex cases, Collision_detection.cpp:
// 751-1703) and, when the GNPs interpenetrate, the penetration depth and
// direction of the expanding polytope, Collision_detection::EPA
// (:1704-1946), as Hoshen_Kopelman::Get_distance_between_GNPs combines them
// (Hoshen_Kopelman.cpp:770-823).  Every branch and FP64 operation follows
// upstream's order; built without FMA contraction, host and device give
// upstream's doubles.
//
// Fixed capacities replace upstream's growing vectors: the polytope holds at
// most kEpaVerts vertices, kEpaFaces faces and kEpaEdges horizon edges, and a
// pair that would need more reports kGjkCapacity instead of growing.
#pragma once

#include <cmath>

#include "gnp_geom.cuh"

namespace cicy {
namespace gnp {

constexpr int kGjkOk = 0;
constexpr int kGjkNoConvergence = 1;   // 50 GJK iterations without meeting the stop test
constexpr int kGjkBadSimplex = 2;      // a simplex size upstream reports as an error
constexpr int kGjkCapacity = 3;        // EPA polytope beyond the fixed capacity
constexpr int kGjkNoHorizon = 4;       // EPA support point sees no face (upstream reads past its list)
constexpr int kEpaVerts = 72;
constexpr int kEpaFaces = 160;
constexpr int kEpaEdges = 160;

__host__ __device__ inline P3 scale(const P3& a, double s) { return P3{a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline double len2(const P3& a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
__host__ __device__ inline P3 unit(const P3& a) {
    const double l = sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    return P3{a.x / l, a.y / l, a.z / l};
}

// Support point of the Minkowski difference A - B in direction D (Support_AB, Support_map).
__host__ __device__ inline P3 support_vertex(const P3& D, const double* V) {
    double best = dot(D, vertex(V, 0));
    int k = 0;
    for (int i = 1; i < 8; i++) {
        const double d = dot(D, vertex(V, i));
        if (d - best > 0.0) {
            best = d;
            k = i;
        }
    }
    return vertex(V, k);
}
__host__ __device__ inline P3 support(const P3& D, const double* VA, const double* VB) {
    return sub(support_vertex(D, VA), support_vertex(scale(D, -1.0), VB));
}

struct Simplex {
    P3 s[4];
    int n = 0;
};

// Direction_from_simplex_to_origin; false for a simplex of 0 or 4 vertices.
__host__ __device__ inline bool direction_to_origin(const Simplex& S, P3& N) {
    if (S.n == 1) {
        N = unit(scale(S.s[0], -1.0));
    } else if (S.n == 2) {
        const P3 AO = scale(S.s[0], -1.0), AB = sub(S.s[1], S.s[0]);
        N = unit(cross(cross(AB, AO), AB));
    } else if (S.n == 3) {
        N = unit(cross(sub(S.s[1], S.s[0]), sub(S.s[2], S.s[0])));
        if (dot(N, S.s[0]) > 0.0) N = scale(N, -1.0);
    } else {
        return false;
    }
    return true;
}

// Is_point_contained_in_simplex: 1 contained, 0 not, -1 invalid simplex size.
__host__ __device__ inline int contains(const Simplex& S, const P3& A) {
    if (S.n == 1) {
        if (dist(S.s[0], A) < kZero) return 1;
    } else if (S.n == 2) {
        const P3 S0A = sub(A, S.s[0]), S0S1 = sub(S.s[1], S.s[0]);
        const P3 N = cross(cross(S0S1, S0A), S0S1);
        if (dot(N, S0A) < kZero) return 1;
    } else if (S.n == 3) {
        const P3 N = cross(sub(S.s[1], S.s[0]), sub(S.s[2], S.s[0]));
        if (fabs(dot(N, sub(A, S.s[0]))) < kZero) return 1;
    } else {
        return -1;
    }
    return 0;
}

// Distance_from_simplex_to_origin; false for a simplex of 0 or 4 vertices.
__host__ __device__ inline bool distance_to_origin(const Simplex& S, double& d) {
    if (S.n == 1) {
        d = sqrt(len2(S.s[0]));
    } else if (S.n == 2) {
        const P3 AO = scale(S.s[0], -1.0), AB = sub(S.s[1], S.s[0]);
        const double t = dot(AO, AB);
        const double dp2 = t * t / len2(AB);
        d = sqrt(len2(AO) - dp2);
    } else if (S.n == 3) {
        const P3 N = unit(cross(sub(S.s[1], S.s[0]), sub(S.s[2], S.s[0])));
        d = fabs(dot(N, S.s[0]));
    } else {
        return false;
    }
    return true;
}

__host__ __device__ inline void keep1(Simplex& S, int i) {
    const P3 a = S.s[i];
    S.s[0] = a;
    S.n = 1;
}
__host__ __device__ inline void keep2(Simplex& S, int i, int j) {
    const P3 a = S.s[i], b = S.s[j];
    S.s[0] = a;
    S.s[1] = b;
    S.n = 2;
}

// Normal_to_face_ouside_tetrahedron: normal of face ABC pointing away from D.
__host__ __device__ inline P3 outer_normal(const P3& A, const P3& B, const P3& C, const P3& D) {
    P3 n = cross(sub(B, A), sub(C, A));
    if (dot(n, sub(D, A)) > 0.0) n = scale(n, -1.0);
    return n;
}

// In-plane normal of an edge, pointing away from the face's third vertex side
// given by `away` (flip when dot(n, ref) has the sign `flip_if_positive` names).
__host__ __device__ inline P3 edge_normal(const P3& edge, const P3& face_n, const P3& ref, bool flip_if_positive) {
    P3 n = cross(edge, face_n);
    const double t = dot(n, ref);
    if (flip_if_positive ? t > 0.0 : t < 0.0) n = scale(n, -1.0);
    return n;
}

// Voroni_region_case3 (Collision_detection.cpp:1068-1206): reduce a triangle
// to its feature closest to the origin.
__host__ __device__ inline void reduce_triangle(Simplex& S) {
    const P3 S0S1 = sub(S.s[1], S.s[0]), S0S2 = sub(S.s[2], S.s[0]);
    const double s0_01 = -dot(S.s[0], S0S1), s0_02 = -dot(S.s[0], S0S2);
    if (s0_02 < 0.0 && s0_01 < 0.0) return keep1(S, 0);
    const P3 S1S2 = sub(S.s[2], S.s[1]);
    const double s1_10 = dot(S.s[1], S0S1), s1_12 = -dot(S.s[1], S1S2);
    if (s1_10 < 0.0 && s1_12 < 0.0) return keep1(S, 1);
    const double s2_20 = dot(S.s[2], S0S2), s2_21 = dot(S.s[2], S1S2);
    if (s2_20 < 0.0 && s2_21 < 0.0) return keep1(S, 2);
    const P3 NT = cross(S0S1, S0S2);
    const P3 N01 = edge_normal(S0S1, NT, S1S2, true);
    if (-dot(S.s[0], N01) > 0.0 && s0_01 > 0.0 && s1_10 > 0.0) return keep2(S, 0, 1);
    const P3 N02 = edge_normal(S0S2, NT, S0S1, true);
    if (-dot(S.s[0], N02) > 0.0 && s0_02 > 0.0 && s2_20 > 0.0) return keep2(S, 0, 2);
    const P3 N12 = edge_normal(S1S2, NT, S0S1, false);
    if (-dot(S.s[1], N12) > 0.0 && s1_12 > 0.0 && s2_21 > 0.0) return keep2(S, 1, 2);
}

// Voroni_region_case4 (:1211-1654): reduce a tetrahedron to its feature
// closest to the origin; false when the origin is inside (interpenetration).
__host__ __device__ inline bool reduce_tetrahedron(Simplex& S) {
    const P3 s0 = S.s[0], s1 = S.s[1], s2 = S.s[2], s3 = S.s[3];
    const P3 S0S1 = sub(s1, s0), S0S2 = sub(s2, s0), S0S3 = sub(s3, s0);
    const double s0_01 = -dot(s0, S0S1), s0_02 = -dot(s0, S0S2), s0_03 = -dot(s0, S0S3);
    if (s0_02 < 0.0 && s0_01 < 0.0 && s0_03 < 0.0) return keep1(S, 0), true;
    const P3 S1S2 = sub(s2, s1), S1S3 = sub(s3, s1);
    const double s1_10 = dot(s1, S0S1), s1_12 = -dot(s1, S1S2), s1_13 = -dot(s1, S1S3);
    if (s1_10 < 0.0 && s1_12 < 0.0 && s1_13 < 0.0) return keep1(S, 1), true;
    const P3 S2S3 = sub(s3, s2);
    const double s2_20 = dot(s2, S0S2), s2_21 = dot(s2, S1S2), s2_23 = -dot(s2, S2S3);
    if (s2_20 < 0.0 && s2_21 < 0.0 && s2_23 < 0.0) return keep1(S, 2), true;
    const double s3_30 = dot(s3, S0S3), s3_31 = dot(s3, S1S3), s3_32 = dot(s3, S2S3);
    if (s3_30 < 0.0 && s3_31 < 0.0 && s3_32 < 0.0) return keep1(S, 3), true;

    // edges: each edge's two in-face normals, pointing away from the face's other vertex
    const P3 N013 = outer_normal(s0, s1, s3, s2), N012 = outer_normal(s0, s1, s2, s3);
    const P3 N01_012 = edge_normal(S0S1, N012, S0S2, true), N01_013 = edge_normal(S0S1, N013, S0S3, true);
    const double e01a = -dot(s0, N01_012), e01b = -dot(s0, N01_013);
    if (s0_01 > 0.0 && s1_10 > 0.0 && e01a > 0.0 && e01b > 0.0) return keep2(S, 0, 1), true;
    const P3 N023 = outer_normal(s0, s2, s3, s1);
    const P3 N02_012 = edge_normal(S0S2, N012, S0S1, true), N02_023 = edge_normal(S0S2, N023, S0S3, true);
    const double e02a = -dot(s0, N02_012), e02b = -dot(s0, N02_023);
    if (s0_02 > 0.0 && s2_20 > 0.0 && e02a > 0.0 && e02b > 0.0) return keep2(S, 0, 2), true;
    const P3 N03_013 = edge_normal(S0S3, N013, S0S1, true), N03_023 = edge_normal(S0S3, N023, S0S2, true);
    const double e03a = -dot(s0, N03_013), e03b = -dot(s0, N03_023);
    if (s0_03 > 0.0 && s3_30 > 0.0 && e03a > 0.0 && e03b > 0.0) return keep2(S, 0, 3), true;
    const P3 N123 = outer_normal(s1, s2, s3, s0);
    const P3 N12_012 = edge_normal(S1S2, N012, S0S1, false), N12_123 = edge_normal(S1S2, N123, S1S3, true);
    const double e12a = -dot(s1, N12_012), e12b = -dot(s1, N12_123);
    if (s1_12 > 0.0 && s2_21 > 0.0 && e12a > 0.0 && e12b > 0.0) return keep2(S, 1, 2), true;
    const P3 N13_013 = edge_normal(S1S3, N013, S0S1, false), N13_123 = edge_normal(S1S3, N123, S1S2, true);
    const double e13a = -dot(s1, N13_013), e13b = -dot(s1, N13_123);
    if (s1_13 > 0.0 && s3_31 > 0.0 && e13a > 0.0 && e13b > 0.0) return keep2(S, 1, 3), true;
    const P3 N23_023 = edge_normal(S2S3, N023, S0S2, false), N23_123 = edge_normal(S2S3, N123, S1S2, false);
    const double e23a = -dot(s2, N23_023), e23b = -dot(s2, N23_123);
    if (s2_23 > 0.0 && s3_32 > 0.0 && e23a > 0.0 && e23b > 0.0) return keep2(S, 2, 3), true;

    // faces
    if (-dot(s0, N012) > 0.0 && e01a < 0.0 && e02a < 0.0 && e12a < 0.0) {
        S.n = 3;
        return true;
    }
    if (-dot(s0, N023) > 0.0 && e02b < 0.0 && e03b < 0.0 && e23a < 0.0) {
        S.s[1] = s3;
        S.n = 3;
        return true;
    }
    if (-dot(s0, N013) > 0.0 && e01b < 0.0 && e13a < 0.0 && e03a < 0.0) {
        S.s[2] = s3;
        S.n = 3;
        return true;
    }
    if (-dot(s1, N123) > 0.0 && e12b < 0.0 && e13b < 0.0 && e23b < 0.0) {
        S.s[0] = s3;
        S.n = 3;
        return true;
    }
    return false;  // origin inside the tetrahedron
}

// Find_voroni_region (:1012-1063): reduce the simplex to the feature closest to
// the origin; 1 reduced, 0 origin inside a tetrahedron, -1 invalid size.
__host__ __device__ inline int reduce_simplex(Simplex& S) {
    if (S.n == 2) {
        const P3 S0S1 = sub(S.s[1], S.s[0]);
        const double d0 = -dot(S.s[0], S0S1), d1 = dot(S.s[1], S0S1);
        if (d0 > 0.0 && d1 > 0.0) return 1;
        if (d1 < 0.0) S.s[0] = S.s[1];
        S.n = 1;
    } else if (S.n == 3) {
        reduce_triangle(S);
    } else if (S.n == 4) {
        return reduce_tetrahedron(S) ? 1 : 0;
    } else if (S.n != 1) {
        return -1;
    }
    return 1;
}

// GJK_distance (:751-870) from an empty simplex.  On interpenetration
// `penetrating` is set and S is the tetrahedron that encloses the origin.
__host__ __device__ inline int gjk_distance(const double* VA, const double* VB, Simplex& S, double& d, P3& N, bool& penetrating) {
    S.n = 1;
    S.s[0] = sub(vertex(VA, 0), vertex(VB, 0));
    penetrating = false;
    if (!distance_to_origin(S, d)) return kGjkBadSimplex;
    for (int it = 1; it <= 50; it++) {
        P3 D;
        if (!direction_to_origin(S, D)) return kGjkBadSimplex;
        const P3 A = support(D, VA, VB);
        const int c = contains(S, A);
        if (c == 1) {
            N = D;
            return kGjkOk;
        }
        if (c == -1) return kGjkBadSimplex;
        S.s[S.n++] = A;
        const int r = reduce_simplex(S);
        if (r == 0) {
            penetrating = true;
            return kGjkOk;
        }
        if (r == -1) return kGjkBadSimplex;
        if (!distance_to_origin(S, d)) return kGjkBadSimplex;
        if (fabs(d - fabs(dot(A, D))) < kZero) {
            N = D;
            return kGjkOk;
        }
    }
    return kGjkNoConvergence;
}

// The expanding polytope of EPA: vertices, triangular faces with their outward
// unit normals and distances to the origin.
struct Polytope {
    P3 v[kEpaVerts];
    int nv = 0;
    int f[kEpaFaces][3];
    P3 fn[kEpaFaces];
    double fd[kEpaFaces];
    int nf = 0;
    int e[kEpaEdges][2];
};

// Normal_and_distance_to_origin (:1785-1812)
__host__ __device__ inline void face_plane(const Polytope& T, int a, int b, int c, P3& n, double& d) {
    const P3 N = unit(cross(sub(T.v[b], T.v[a]), sub(T.v[c], T.v[a])));
    const double signed_dist = dot(N, scale(T.v[a], -1.0));
    n = signed_dist > 0.0 ? scale(N, -1.0) : N;
    d = fabs(signed_dist);
}

__host__ __device__ inline void push_face(Polytope& T, int a, int b, int c) {
    T.f[T.nf][0] = a;
    T.f[T.nf][1] = b;
    T.f[T.nf][2] = c;
    face_plane(T, a, b, c, T.fn[T.nf], T.fd[T.nf]);
    T.nf++;
}

// EPA (:1704-1780) on the tetrahedron S from gjk_distance: penetration depth
// and direction (unit normal of the closest face of the expanded polytope).
__host__ __device__ inline int epa_depth(const double* VA, const double* VB, const Simplex& S, Polytope& T, P3& normal, double& depth) {
    T.nv = 4;
    for (int i = 0; i < 4; i++) T.v[i] = S.s[i];
    T.nf = 0;
    push_face(T, 0, 1, 2);
    push_face(T, 0, 1, 3);
    push_face(T, 0, 2, 3);
    push_face(T, 1, 2, 3);
    for (;;) {
        // Find_closest_face: the first face of least distance
        int k = 0;
        for (int i = 1; i < T.nf; i++)
            if (T.fd[i] < T.fd[k]) k = i;
        const P3 N = T.fn[k];
        const double pd = T.fd[k];
        const P3 P = support(N, VA, VB);
        if (dot(P, N) - pd < kZero) {
            normal = N;
            depth = pd;
            return kGjkOk;
        }
        if (T.nv == kEpaVerts) return kGjkCapacity;
        const int s = T.nv++;
        T.v[s] = P;
        // Reconstruct_simplex (:1849-1945): drop the faces the new vertex sees and
        // close the hole with faces from it to the horizon edges, which are the
        // seen faces' edges not shared by two seen faces, in upstream's list order
        int ne = 0, first = -1;
        for (int i = 0; i < T.nf; i++) {
            if (!(dot(T.fn[i], sub(T.v[s], T.v[T.f[i][0]])) > 0.0)) continue;
            if (first < 0) {
                first = i;
                for (int j = 0; j < 3; j++) {
                    T.e[ne][0] = T.f[i][j];
                    T.e[ne][1] = T.f[i][(j + 1) % 3];
                    ne++;
                }
                continue;
            }
            for (int j = 0; j < 3; j++) {
                const int a = T.f[i][j], b = T.f[i][(j + 1) % 3];
                int hit = -1;
                for (int m = 0; m < ne; m++)
                    if ((T.e[m][0] == a && T.e[m][1] == b) || (T.e[m][0] == b && T.e[m][1] == a)) {
                        hit = m;
                        break;
                    }
                if (hit < 0) {
                    if (ne == kEpaEdges) return kGjkCapacity;
                    T.e[ne][0] = a;
                    T.e[ne][1] = b;
                    ne++;
                } else {
                    for (int m = hit; m + 1 < ne; m++) {
                        T.e[m][0] = T.e[m + 1][0];
                        T.e[m][1] = T.e[m + 1][1];
                    }
                    ne--;
                }
            }
        }
        if (first < 0) return kGjkNoHorizon;
        // keep the unseen faces in order (the seen test reads the old normals)
        int w = 0;
        for (int i = 0; i < T.nf; i++) {
            if (dot(T.fn[i], sub(T.v[s], T.v[T.f[i][0]])) > 0.0) continue;
            if (w != i) {
                T.f[w][0] = T.f[i][0];
                T.f[w][1] = T.f[i][1];
                T.f[w][2] = T.f[i][2];
                T.fn[w] = T.fn[i];
                T.fd[w] = T.fd[i];
            }
            w++;
        }
        T.nf = w;
        if (T.nf + ne > kEpaFaces) return kGjkCapacity;
        for (int m = 0; m < ne; m++) push_face(T, s, T.e[m][0], T.e[m][1]);
    }
}

// Get_distance_between_GNPs (Hoshen_Kopelman.cpp:770-823): the separation of
// GNPs a and b with the direction of GJK, or, when they interpenetrate, the
// EPA direction, the move of b by N (depth + vdW) and the distance vdW.
__host__ __device__ inline int pair_distance(const double* VA, const double* VB, double vdw, Polytope& T, double& d, P3& N, P3& disp,
                                             bool& penetrating) {
    Simplex S;
    disp = P3{0.0, 0.0, 0.0};
    int st = gjk_distance(VA, VB, S, d, N, penetrating);
    if (st != kGjkOk || !penetrating) return st;
    st = epa_depth(VA, VB, S, T, N, d);
    if (st != kGjkOk) return st;
    disp = scale(N, d + vdw);
    d = vdw;
    return kGjkOk;
}

}  // namespace gnp
}  // namespace cicy
