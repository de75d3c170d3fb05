// Closest point of a GNP (graphene nanoplatelet cuboid) to a point, host and
// device: Generate_Network::Get_gnp_point_closest_to_point,
// Get_point_closest_to_large_gnp_face and Distance_from_point_to_edge
// (Generate_Network.cpp:5577-5856), with Point_3D::distance_to,
// Point_3D::distance_to(P0, P1), Point_3D::cross, make_unit and
// Plane_3D::distance_to (Geometry_3D.cpp) — the CNT-GNP distance of the mixed
// contact search (Hoshen_Kopelman::Find_adjacent_labels).  The decision tree
// and every arithmetic step follow upstream's order; built without FMA
// contraction on both sides, host and device give upstream's doubles.
//
// A GNP is its 8 vertices V[24] (x, y, z each) and 6 face planes F[24]
// (normal x, y, z, offset d; n.p + d = 0 on the face), as cicy_read_gnps builds
// them.  Returns 0 with the distance and closest point, or -1 (distance 0) when
// the point is inside the GNP.
#pragma once

#include <cmath>

namespace cicy {
namespace gnp {

constexpr double kZero = 1.0e-10;  // MathMatrix.h:18

struct P3 {
    double x, y, z;
};

__host__ __device__ inline P3 sub(const P3& a, const P3& b) { return P3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline double dot(const P3& a, const P3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline P3 cross(const P3& a, const P3& b) {
    return P3{a.y * b.z - b.y * a.z, -(a.x * b.z - b.x * a.z), a.x * b.y - b.x * a.y};
}
__host__ __device__ inline P3 vertex(const double* V, int k) { return P3{V[3 * k], V[3 * k + 1], V[3 * k + 2]}; }
__host__ __device__ inline P3 normal(const double* F, int f) { return P3{F[4 * f], F[4 * f + 1], F[4 * f + 2]}; }
__host__ __device__ inline double dist(const P3& a, const P3& b) {
    const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return sqrt(dx * dx + dy * dy + dz * dz);
}
// Plane_3D::distance_to: |n.p + d| / |n|
__host__ __device__ inline double plane_dist(const double* F, int f, const P3& p) {
    const double* c = F + 4 * f;
    const double num = c[0] * p.x + c[1] * p.y + c[2] * p.z + c[3];
    const double den = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    return fabs(num / den);
}
// Distance_from_point_to_edge: distance to the line A B and the point at that distance along the in-plane normal
__host__ __device__ inline void to_edge(const P3& p, const P3& a, const P3& b, P3& q, double& d) {
    const P3 v = sub(b, a);
    const P3 c = cross(v, sub(p, a));
    const double num = c.x * c.x + c.y * c.y + c.z * c.z;
    const double den = v.x * v.x + v.y * v.y + v.z * v.z;
    d = sqrt(num / den);
    P3 n = cross(cross(v, sub(p, a)), v);
    const double len = sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
    n = P3{n.x / len, n.y / len, n.z / len};
    q = P3{p.x - n.x * d, p.y - n.y * d, p.z - n.z * d};
}
__host__ __device__ inline void project(const double* F, int f, const P3& p, P3& q, double& d) {
    d = plane_dist(F, f, p);
    const P3 n = normal(F, f);
    q = P3{p.x - n.x * d, p.y - n.y * d, p.z - n.z * d};
}
// Get_point_closest_to_large_gnp_face (vertices v0..v3 of face f)
__host__ __device__ inline void large_face(const double* V, const double* F, int i0, int i1, int i2, int i3, int f, const P3& p, P3& q,
                                           double& d) {
    const P3 v0 = vertex(V, i0), v1 = vertex(V, i1), v2 = vertex(V, i2), v3 = vertex(V, i3);
    const P3 v0p = sub(p, v0), v1p = sub(p, v1);
    if (dot(normal(F, 2), v0p) > kZero) {
        if (dot(normal(F, 3), v0p) > kZero) {
            d = dist(p, v0);
            q = v0;
        } else if (dot(normal(F, 5), sub(p, v3)) > kZero) {
            d = dist(p, v3);
            q = v3;
        } else {
            to_edge(p, v0, v3, q, d);
        }
    } else if (dot(normal(F, 4), v1p) > kZero) {
        if (dot(normal(F, 3), v1p) > kZero) {
            d = dist(p, v1);
            q = v1;
        } else if (dot(normal(F, 5), sub(p, v2)) > kZero) {
            d = dist(p, v2);
            q = v2;
        } else {
            to_edge(p, v1, v2, q, d);
        }
    } else if (dot(normal(F, 3), v0p) > kZero) {
        to_edge(p, v0, v1, q, d);
    } else if (dot(normal(F, 5), sub(p, v3)) > kZero) {
        to_edge(p, v2, v3, q, d);
    } else {
        project(F, f, p, q, d);
    }
}

// Get_gnp_point_closest_to_point
__host__ __device__ inline int closest_point(const double* V, const double* F, const P3& p, P3& q, double& d) {
    const P3 v0p = sub(p, vertex(V, 0)), v1p = sub(p, vertex(V, 1));
    if (dot(normal(F, 0), v0p) > kZero) {
        large_face(V, F, 0, 1, 2, 3, 0, p, q, d);
    } else if (dot(normal(F, 1), sub(p, vertex(V, 4))) > kZero) {
        large_face(V, F, 4, 5, 6, 7, 1, p, q, d);
    } else if (dot(normal(F, 2), v0p) > kZero) {
        if (dot(normal(F, 3), v0p) > kZero) to_edge(p, vertex(V, 0), vertex(V, 4), q, d);
        else if (dot(normal(F, 5), sub(p, vertex(V, 3))) > kZero) to_edge(p, vertex(V, 3), vertex(V, 7), q, d);
        else project(F, 2, p, q, d);
    } else if (dot(normal(F, 4), v1p) > kZero) {
        if (dot(normal(F, 3), v1p) > kZero) to_edge(p, vertex(V, 1), vertex(V, 5), q, d);
        else if (dot(normal(F, 5), sub(p, vertex(V, 2))) > kZero) to_edge(p, vertex(V, 2), vertex(V, 6), q, d);
        else project(F, 4, p, q, d);
    } else if (dot(normal(F, 3), v0p) > kZero) {
        project(F, 3, p, q, d);
    } else if (dot(normal(F, 5), sub(p, vertex(V, 2))) > kZero) {
        project(F, 5, p, q, d);
    } else {
        q = P3{0.0, 0.0, 0.0};
        d = 0.0;
        return -1;
    }
    return 0;
}

}  // namespace gnp
}  // namespace cicy
