"""CPU restatement of the GNP part of the contact grid and of the CNT-GNP
contact pass (TEST ORACLE: only tests/ call it, never the product).

Contact_grid::Fill_sectioned_domain_gnps / Fill_sectioned_domain_single_gnp /
Assign_point_to_regions_gnps (Contact_grid.cpp:297-512): every GNP in
`gnps_inside` order is sampled on a regular grid of its volume (at least
40 x 40 x 2 points, bilinear between its vertices), and every sample point
strictly inside the window adds the GNP to its region and to the neighbour
regions its overlap flags name (Calculate_region_coordinates :163-184,
Calculate_overlapping_flags :186-212); a region lists each GNP once, in
`gnps_inside` order.  numpy's element-wise +, -, *, / are the same IEEE
operations as upstream's scalar code, in the same order, so the points and the
region lists are identical.

Generate_Network::Get_gnp_point_closest_to_point (Generate_Network.cpp:5577-
5856) and Hoshen_Kopelman::Find_adjacent_labels (Hoshen_Kopelman.cpp:1989-2142)
are restated with Python floats, which are IEEE doubles evaluated left to right
without contraction, as upstream's code is compiled.
"""
from __future__ import annotations

import math

import numpy as np

ZERO = 1.0e-10  # MathMatrix.h:18


def region_grid(window, gs_min, overlap_cnt: float, overlap_gnp: float):
    """(n_regions, l_regions) of Contact_grid::Generate_contact_grid + Adjust_regions_if_needed
    (Contact_grid.cpp:18-102); window = (min xyz, len xyz, max xyz)."""
    n = [max(1, int(window[3 + a] / gs_min[a])) for a in range(3)]
    l = [float(g) for g in gs_min]
    ov = max(overlap_cnt, overlap_gnp)
    for a in range(3):
        if gs_min[a] < 2 * ov:
            l[a] = 2.0 * (ov + ZERO)
            n[a] = 1 + int(window[3 + a] / l[a])
    return n, l


def sample_points(V, l_side: float, t: float, l_regions):
    """Sample points of one GNP (vertices V[8, 3]) in upstream's k, j, i order."""
    nx = max(40, 1 + int(l_side / l_regions[0]))
    ny = max(40, 1 + int(l_side / l_regions[1]))
    nz = max(2, 1 + int(t / l_regions[2]))
    lz = (np.arange(nz, dtype=np.float64) / (nz - 1))[:, None]
    start1 = V[7] + (V[3] - V[7]) * lz
    end1 = V[4] + (V[0] - V[4]) * lz
    diff1 = end1 - start1
    start2 = V[6] + (V[2] - V[6]) * lz
    end2 = V[5] + (V[1] - V[5]) * lz
    diff2 = end2 - start2
    ly = (np.arange(ny, dtype=np.float64) / (ny - 1))[None, :, None]
    start_x = start1[:, None, :] + diff1[:, None, :] * ly
    end_x = start2[:, None, :] + diff2[:, None, :] * ly
    diff_x = end_x - start_x
    lx = (np.arange(nx, dtype=np.float64) / (nx - 1))[None, None, :, None]
    pts = start_x[:, :, None, :] + diff_x[:, :, None, :] * lx
    return pts.reshape(-1, 3)


def fill_sectioned_domain_gnps(window, vertices, l_side, thickness, gnps_inside, n, l, overlap: float):
    """Region lists (list of GNP index lists, region t = a + b sx + c sx sy)."""
    w = np.asarray(window, dtype=np.float64)
    lo, hi = w[0:3], w[6:9]
    n_arr = np.asarray(n)
    l_arr = np.asarray(l, dtype=np.float64)
    regions = [[] for _ in range(n[0] * n[1] * n[2])]
    for g in gnps_inside:
        P = sample_points(vertices[g], l_side[g], thickness[g], l)
        inside = ~np.any((P <= lo) | (P >= hi), axis=1)
        P = P[inside]
        if len(P) == 0:
            continue
        abc = np.trunc((P - lo) / l_arr).astype(np.int64)
        abc = np.where(abc < 0, 0, np.where(abc >= n_arr, n_arr - 1, abc))
        x1 = abc.astype(np.float64) * l_arr + lo
        x2 = x1 + l_arr
        low = (abc > 0) & (P >= x1) & (P <= x1 + overlap)
        high = ~low & (abc < n_arr - 1) & (P >= x2 - overlap) & (P <= x2)
        f = np.where(low, -1, np.where(high, 1, 0))
        touched = set()
        t = abc[:, 0] + abc[:, 1] * n[0] + abc[:, 2] * n[0] * n[1]
        touched.update(t.tolist())
        for a in range(3):
            m = f[:, a] != 0
            if m.any():
                q = abc[m].copy()
                q[:, a] += f[m, a]
                touched.update((q[:, 0] + q[:, 1] * n[0] + q[:, 2] * n[0] * n[1]).tolist())
        for r in touched:
            regions[r].append(int(g))
    return regions


# ---------------------------------------------------------------------------
# Closest GNP point to a point (Generate_Network.cpp:5577-5856)


def _sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _cross(a, b):
    return (a[1] * b[2] - b[1] * a[2], -(a[0] * b[2] - b[0] * a[2]), a[0] * b[1] - b[0] * a[1])


def _dist(a, b):
    dx, dy, dz = a[0] - b[0], a[1] - b[1], a[2] - b[2]
    return math.sqrt(dx * dx + dy * dy + dz * dz)


def _to_edge(p, a, b):
    """Distance_from_point_to_edge: distance from p to the line a b, and the point
    reached from p along the unit normal of the line in the plane of p, a, b."""
    v = _sub(b, a)
    c = _cross(v, _sub(p, a))
    d = math.sqrt((c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) / (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]))
    n = _cross(_cross(v, _sub(p, a)), v)
    ln = math.sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2])
    n = (n[0] / ln, n[1] / ln, n[2] / ln)
    return (p[0] - n[0] * d, p[1] - n[1] * d, p[2] - n[2] * d), d


def _project(F, f, p):
    """Plane_3D::distance_to (|n.p + d| / |n|) and the foot along the face normal."""
    c = F[f]
    d = abs((c[0] * p[0] + c[1] * p[1] + c[2] * p[2] + c[3]) / math.sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]))
    return (p[0] - c[0] * d, p[1] - c[1] * d, p[2] - c[2] * d), d


def _large_face(V, F, i, f, p):
    """Get_point_closest_to_large_gnp_face for the face f with vertices i[0..3]."""
    v0, v1, v2, v3 = V[i[0]], V[i[1]], V[i[2]], V[i[3]]
    v0p, v1p = _sub(p, v0), _sub(p, v1)
    if _dot(F[2][:3], v0p) > ZERO:
        if _dot(F[3][:3], v0p) > ZERO:
            return v0, _dist(p, v0)
        if _dot(F[5][:3], _sub(p, v3)) > ZERO:
            return v3, _dist(p, v3)
        return _to_edge(p, v0, v3)
    if _dot(F[4][:3], v1p) > ZERO:
        if _dot(F[3][:3], v1p) > ZERO:
            return v1, _dist(p, v1)
        if _dot(F[5][:3], _sub(p, v2)) > ZERO:
            return v2, _dist(p, v2)
        return _to_edge(p, v1, v2)
    if _dot(F[3][:3], v0p) > ZERO:
        return _to_edge(p, v0, v1)
    if _dot(F[5][:3], _sub(p, v3)) > ZERO:
        return _to_edge(p, v2, v3)
    return _project(F, f, p)


def closest_point(V, F, p):
    """(point, distance, flag) of Get_gnp_point_closest_to_point for the GNP with
    vertices V[8][3] and face planes F[6][4] (normal, offset); flag -1 with
    distance 0 when p is inside the GNP."""
    V = [tuple(float(c) for c in v) for v in V]
    F = [tuple(float(c) for c in f) for f in F]
    p = tuple(float(c) for c in p)
    v0p, v1p = _sub(p, V[0]), _sub(p, V[1])
    if _dot(F[0][:3], v0p) > ZERO:
        q, d = _large_face(V, F, (0, 1, 2, 3), 0, p)
    elif _dot(F[1][:3], _sub(p, V[4])) > ZERO:
        q, d = _large_face(V, F, (4, 5, 6, 7), 1, p)
    elif _dot(F[2][:3], v0p) > ZERO:
        if _dot(F[3][:3], v0p) > ZERO:
            q, d = _to_edge(p, V[0], V[4])
        elif _dot(F[5][:3], _sub(p, V[3])) > ZERO:
            q, d = _to_edge(p, V[3], V[7])
        else:
            q, d = _project(F, 2, p)
    elif _dot(F[4][:3], v1p) > ZERO:
        if _dot(F[3][:3], v1p) > ZERO:
            q, d = _to_edge(p, V[1], V[5])
        elif _dot(F[5][:3], _sub(p, V[2])) > ZERO:
            q, d = _to_edge(p, V[2], V[6])
        else:
            q, d = _project(F, 4, p)
    elif _dot(F[3][:3], v0p) > ZERO:
        q, d = _project(F, 3, p)
    elif _dot(F[5][:3], _sub(p, V[2])) > ZERO:
        q, d = _project(F, 5, p)
    else:
        return (0.0, 0.0, 0.0), 0.0, -1
    return q, d, 0


# ---------------------------------------------------------------------------
# CNT-GNP contacts (Hoshen_Kopelman.cpp:1989-2142)


def find_adjacent_labels(xyz, flag, radii, sd_cnt, sd_gnp, vertices, planes, vdw: float, tunnel: float):
    """CNT-GNP contacts of Find_adjacent_labels with inside points ignored
    (ignore_eror_cnt_inside_gnp = 1: distance r + 3 tunnel, no contact).

    Regions in order, the GNPs of a region in list order, the CNT points of the
    region in list order; a (point, GNP) pair not yet in contact is a contact
    when its junction distance (closest distance minus the CNT radius, raised to
    `vdw`) is within `tunnel`, and takes the next contact-point number.
    Returns {(P, GNP): (number, junction distance, closest point)}."""
    out = {}
    memo = {}
    for pts, gs in zip(sd_cnt, sd_gnp):
        for g in gs:
            for P in pts:
                if (P, g) in out:
                    continue
                key = (P, g)
                if key not in memo:
                    cnt = int(flag[P])
                    q, d, f = closest_point(vertices[g], planes[g], xyz[P])
                    if f == -1:
                        d = float(radii[cnt]) + 3.0 * tunnel
                    dj = d - float(radii[cnt])
                    if dj < vdw:
                        dj = vdw
                    memo[key] = (dj - tunnel <= ZERO, dj, q)
                hit, dj, q = memo[key]
                if hit:
                    out[key] = (len(out), dj, q)
    return out


# ---------------------------------------------------------------------------
# GNP-GNP distance: GJK, EPA (Collision_detection.cpp:751-1946) as
# Hoshen_Kopelman::Get_distance_between_GNPs combines them (Hoshen_Kopelman.cpp:770-823)


def _scale(a, s):
    return (a[0] * s, a[1] * s, a[2] * s)


def _len2(a):
    return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]


def _unit(a):
    ln = math.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
    return (a[0] / ln, a[1] / ln, a[2] / ln)


def _support_map(D, V):
    """Support_map: the first vertex of largest D.v (strictly larger replaces)."""
    best, k = _dot(D, V[0]), 0
    for i in range(1, 8):
        d = _dot(D, V[i])
        if d - best > 0.0:
            best, k = d, i
    return V[k]


def _support(D, VA, VB):
    return _sub(_support_map(D, VA), _support_map(_scale(D, -1.0), VB))


def _direction(S):
    """Direction_from_simplex_to_origin (:872-914)."""
    if len(S) == 1:
        return _unit(_scale(S[0], -1.0))
    if len(S) == 2:
        AO, AB = _scale(S[0], -1.0), _sub(S[1], S[0])
        return _unit(_cross(_cross(AB, AO), AB))
    if len(S) == 3:
        N = _unit(_cross(_sub(S[1], S[0]), _sub(S[2], S[0])))
        return _scale(N, -1.0) if _dot(N, S[0]) > 0.0 else N
    raise ValueError("Direction_from_simplex_to_origin: invalid simplex size")


def _contained(S, A):
    """Is_point_contained_in_simplex (:916-967)."""
    if len(S) == 1:
        return _dist(S[0], A) < ZERO
    if len(S) == 2:
        S0A, S0S1 = _sub(A, S[0]), _sub(S[1], S[0])
        return _dot(_cross(_cross(S0S1, S0A), S0S1), S0A) < ZERO
    if len(S) == 3:
        N = _cross(_sub(S[1], S[0]), _sub(S[2], S[0]))
        return abs(_dot(N, _sub(A, S[0]))) < ZERO
    raise ValueError("Is_point_contained_in_simplex: invalid simplex size")


def _distance(S):
    """Distance_from_simplex_to_origin (:969-1010)."""
    if len(S) == 1:
        return math.sqrt(_len2(S[0]))
    if len(S) == 2:
        AO, AB = _scale(S[0], -1.0), _sub(S[1], S[0])
        t = _dot(AO, AB)
        return math.sqrt(_len2(AO) - t * t / _len2(AB))
    if len(S) == 3:
        return abs(_dot(_unit(_cross(_sub(S[1], S[0]), _sub(S[2], S[0]))), S[0]))
    raise ValueError("Distance_from_simplex_to_origin: invalid simplex size")


def _outer_normal(A, B, C, D):
    """Normal_to_face_ouside_tetrahedron (:484-503)."""
    n = _cross(_sub(B, A), _sub(C, A))
    return _scale(n, -1.0) if _dot(n, _sub(D, A)) > 0.0 else n


def _edge_normal(edge, face_n, ref, flip_if_positive):
    n = _cross(edge, face_n)
    t = _dot(n, ref)
    return _scale(n, -1.0) if (t > 0.0 if flip_if_positive else t < 0.0) else n


def _triangle(S):
    """Voroni_region_case3 (:1068-1206): the triangle's feature closest to the origin."""
    s0, s1, s2 = S
    S0S1, S0S2 = _sub(s1, s0), _sub(s2, s0)
    a01, a02 = -_dot(s0, S0S1), -_dot(s0, S0S2)
    if a02 < 0.0 and a01 < 0.0:
        return [s0]
    S1S2 = _sub(s2, s1)
    b10, b12 = _dot(s1, S0S1), -_dot(s1, S1S2)
    if b10 < 0.0 and b12 < 0.0:
        return [s1]
    c20, c21 = _dot(s2, S0S2), _dot(s2, S1S2)
    if c20 < 0.0 and c21 < 0.0:
        return [s2]
    NT = _cross(S0S1, S0S2)
    if -_dot(s0, _edge_normal(S0S1, NT, S1S2, True)) > 0.0 and a01 > 0.0 and b10 > 0.0:
        return [s0, s1]
    if -_dot(s0, _edge_normal(S0S2, NT, S0S1, True)) > 0.0 and a02 > 0.0 and c20 > 0.0:
        return [s0, s2]
    if -_dot(s1, _edge_normal(S1S2, NT, S0S1, False)) > 0.0 and b12 > 0.0 and c21 > 0.0:
        return [s1, s2]
    return S


def _tetrahedron(S):
    """Voroni_region_case4 (:1211-1654): the tetrahedron's feature closest to the
    origin, or None when the origin is inside it."""
    s0, s1, s2, s3 = S
    S0S1, S0S2, S0S3 = _sub(s1, s0), _sub(s2, s0), _sub(s3, s0)
    a01, a02, a03 = -_dot(s0, S0S1), -_dot(s0, S0S2), -_dot(s0, S0S3)
    if a02 < 0.0 and a01 < 0.0 and a03 < 0.0:
        return [s0]
    S1S2, S1S3 = _sub(s2, s1), _sub(s3, s1)
    b10, b12, b13 = _dot(s1, S0S1), -_dot(s1, S1S2), -_dot(s1, S1S3)
    if b10 < 0.0 and b12 < 0.0 and b13 < 0.0:
        return [s1]
    S2S3 = _sub(s3, s2)
    c20, c21, c23 = _dot(s2, S0S2), _dot(s2, S1S2), -_dot(s2, S2S3)
    if c20 < 0.0 and c21 < 0.0 and c23 < 0.0:
        return [s2]
    d30, d31, d32 = _dot(s3, S0S3), _dot(s3, S1S3), _dot(s3, S2S3)
    if d30 < 0.0 and d31 < 0.0 and d32 < 0.0:
        return [s3]
    N013, N012 = _outer_normal(s0, s1, s3, s2), _outer_normal(s0, s1, s2, s3)
    e01a = -_dot(s0, _edge_normal(S0S1, N012, S0S2, True))
    e01b = -_dot(s0, _edge_normal(S0S1, N013, S0S3, True))
    if a01 > 0.0 and b10 > 0.0 and e01a > 0.0 and e01b > 0.0:
        return [s0, s1]
    N023 = _outer_normal(s0, s2, s3, s1)
    e02a = -_dot(s0, _edge_normal(S0S2, N012, S0S1, True))
    e02b = -_dot(s0, _edge_normal(S0S2, N023, S0S3, True))
    if a02 > 0.0 and c20 > 0.0 and e02a > 0.0 and e02b > 0.0:
        return [s0, s2]
    e03a = -_dot(s0, _edge_normal(S0S3, N013, S0S1, True))
    e03b = -_dot(s0, _edge_normal(S0S3, N023, S0S2, True))
    if a03 > 0.0 and d30 > 0.0 and e03a > 0.0 and e03b > 0.0:
        return [s0, s3]
    N123 = _outer_normal(s1, s2, s3, s0)
    e12a = -_dot(s1, _edge_normal(S1S2, N012, S0S1, False))
    e12b = -_dot(s1, _edge_normal(S1S2, N123, S1S3, True))
    if b12 > 0.0 and c21 > 0.0 and e12a > 0.0 and e12b > 0.0:
        return [s1, s2]
    e13a = -_dot(s1, _edge_normal(S1S3, N013, S0S1, False))
    e13b = -_dot(s1, _edge_normal(S1S3, N123, S1S2, True))
    if b13 > 0.0 and d31 > 0.0 and e13a > 0.0 and e13b > 0.0:
        return [s1, s3]
    e23a = -_dot(s2, _edge_normal(S2S3, N023, S0S2, False))
    e23b = -_dot(s2, _edge_normal(S2S3, N123, S1S2, False))
    if c23 > 0.0 and d32 > 0.0 and e23a > 0.0 and e23b > 0.0:
        return [s2, s3]
    if -_dot(s0, N012) > 0.0 and e01a < 0.0 and e02a < 0.0 and e12a < 0.0:
        return [s0, s1, s2]
    if -_dot(s0, N023) > 0.0 and e02b < 0.0 and e03b < 0.0 and e23a < 0.0:
        return [s0, s3, s2]
    if -_dot(s0, N013) > 0.0 and e01b < 0.0 and e13a < 0.0 and e03a < 0.0:
        return [s0, s1, s3]
    if -_dot(s1, N123) > 0.0 and e12b < 0.0 and e13b < 0.0 and e23b < 0.0:
        return [s3, s1, s2]
    return None


def _reduce(S):
    """Find_voroni_region (:1012-1063); None when the origin is inside."""
    if len(S) == 2:
        S0S1 = _sub(S[1], S[0])
        d0, d1 = -_dot(S[0], S0S1), _dot(S[1], S0S1)
        if d0 > 0.0 and d1 > 0.0:
            return S
        return [S[1]] if d1 < 0.0 else [S[0]]
    if len(S) == 3:
        return _triangle(S)
    if len(S) == 4:
        return _tetrahedron(S)
    return S


def gjk_distance(VA, VB):
    """GJK_distance (:751-870) from an empty simplex: (distance, direction,
    penetrating, simplex); on interpenetration the simplex is the tetrahedron
    that encloses the origin."""
    S = [_sub(VA[0], VB[0])]
    d = _distance(S)
    for _ in range(50):
        D = _direction(S)
        A = _support(D, VA, VB)
        if _contained(S, A):
            return d, D, False, S
        T = S + [A]
        S = _reduce(T)
        if S is None:
            return None, None, True, T
        d = _distance(S)
        if abs(d - abs(_dot(A, D))) < ZERO:
            return d, D, False, S
    raise RuntimeError("GJK_distance: maximum number of iterations reached")


def _face_plane(P, f):
    """Normal_and_distance_to_origin (:1785-1812)."""
    N = _unit(_cross(_sub(P[f[1]], P[f[0]]), _sub(P[f[2]], P[f[0]])))
    sd = _dot(N, _scale(P[f[0]], -1.0))
    return (_scale(N, -1.0) if sd > 0.0 else N), abs(sd)


def epa(VA, VB, tetra):
    """EPA (:1704-1780) with Reconstruct_simplex (:1849-1945): (depth, direction)."""
    P = list(tetra)
    faces = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]
    planes = [_face_plane(P, f) for f in faces]
    while True:
        k = 0
        for i in range(1, len(faces)):
            if planes[i][1] < planes[k][1]:
                k = i
        N, pd = planes[k]
        s = _support(N, VA, VB)
        if _dot(s, N) - pd < ZERO:
            return pd, N
        P.append(s)
        S = len(P) - 1
        seen = [i for i in range(len(faces)) if _dot(planes[i][0], _sub(P[S], P[faces[i][0]])) > 0.0]
        f0 = faces[seen[0]]
        edges = [(f0[0], f0[1]), (f0[1], f0[2]), (f0[2], f0[0])]
        for i in seen[1:]:
            f = faces[i]
            for e in ((f[0], f[1]), (f[1], f[2]), (f[2], f[0])):
                hit = next((m for m, g in enumerate(edges) if g == e or g == (e[1], e[0])), -1)
                if hit < 0:
                    edges.append(e)
                else:
                    del edges[hit]
        keep = [i for i in range(len(faces)) if i not in set(seen)]
        faces = [faces[i] for i in keep]
        planes = [planes[i] for i in keep]
        for e in edges:
            faces.append((S, e[0], e[1]))
            planes.append(_face_plane(P, faces[-1]))


def pair_distance(VA, VB, vdw: float):
    """Get_distance_between_GNPs: (dist, direction, displacement of B, penetrating)."""
    VA = [tuple(float(c) for c in v) for v in VA]
    VB = [tuple(float(c) for c in v) for v in VB]
    d, N, pen, S = gjk_distance(VA, VB)
    if not pen:
        return d, N, (0.0, 0.0, 0.0), False
    depth, N = epa(VA, VB, S)
    return vdw, N, _scale(N, depth + vdw), True


def contact_pairs(sd_gnp, vertices, vdw: float, tunnel: float):
    """GNP-GNP pairs of Label_gnps_in_window (Hoshen_Kopelman.cpp:626-767) within the
    tunnelling cutoff, in upstream's visiting order (regions, then j < k in the
    region; a pair measured at its first visit): list of (a, b, dist, direction,
    displacement, penetrating), a pair ordered (min, max)."""
    visited = set()
    out = []
    for gs in sd_gnp:
        for j in range(len(gs) - 1):
            for k in range(j + 1, len(gs)):
                a, b = min(gs[j], gs[k]), max(gs[j], gs[k])
                if (a, b) in visited:
                    continue
                visited.add((a, b))
                d, N, m, pen = pair_distance(vertices[a], vertices[b], vdw)
                if d <= tunnel:
                    out.append((a, b, d, N, m, pen))
    return out


# ---------------------------------------------------------------------------
# Junction points of two GNPs in contact (Hoshen_Kopelman.cpp:826-1825)

_FACE_EDGES = {  # Get_edges_of_face (:1330-1426): vertex sum -> 4 edges, the face normal bounding each
    7: (((0, 3), (0, 1), (1, 2), (2, 3)), (2, 3, 4, 5)),
    22: (((4, 7), (4, 5), (5, 6), (6, 7)), (2, 3, 4, 5)),
    15: (((0, 3), (3, 7), (7, 4), (0, 4)), (0, 5, 1, 3)),
    11: (((1, 0), (0, 4), (4, 5), (5, 1)), (0, 2, 1, 4)),
    14: (((1, 2), (2, 6), (6, 5), (5, 1)), (0, 5, 1, 3)),
    18: (((2, 3), (3, 7), (7, 6), (6, 2)), (0, 2, 1, 4)),
}
_FOURTH = {(0, 1, 2): 3, (0, 1, 3): 2, (0, 2, 3): 1, (1, 2, 3): 0, (4, 5, 6): 7, (4, 5, 7): 6, (4, 6, 7): 5, (5, 6, 7): 4,
           (0, 1, 4): 5, (0, 1, 5): 4, (0, 4, 5): 1, (1, 4, 5): 0, (1, 2, 5): 6, (1, 2, 6): 5, (1, 5, 6): 2, (2, 5, 6): 1,
           (2, 3, 6): 7, (2, 3, 7): 6, (2, 6, 7): 3, (3, 6, 7): 2, (0, 3, 4): 7, (0, 3, 7): 4, (0, 4, 7): 3, (3, 4, 7): 0}
_PLANE_VERTS = ((0, 1, 3), (4, 7, 5), (0, 3, 4), (0, 4, 1), (1, 5, 2), (2, 6, 3))  # Update_gnp_plane_equations


class JunctionError(Exception):
    """A step upstream's junction search fails in (it returns 0 there)."""


def _add(a, b):
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def _div(a, s):
    return (a[0] / s, a[1] / s, a[2] / s)


def moved_gnp(V, d):
    """Generate_Network::Move_gnp: vertices + d and the face normals rebuilt from them."""
    v = [_add(tuple(float(c) for c in p), d) for p in V]
    return v, [_unit(_cross(_sub(v[b], v[a]), _sub(v[c], v[a]))) for a, b, c in _PLANE_VERTS]


def _lambda(Pin, Pout, e1, e2):
    """Lambda_of_two_lines (:1529-1540)."""
    detA = (e2[0] - e1[0]) * (Pin[1] - Pout[1]) - (Pin[0] - Pout[0]) * (e2[1] - e1[1])
    detAP = (e2[0] - e1[0]) * (e1[1] - Pout[1]) - (e1[0] - Pout[0]) * (e2[1] - e1[1])
    return detAP / detA


def _face(face_sum):
    if face_sum not in _FACE_EDGES:
        raise JunctionError("Get_edges_of_face: invalid face")
    return _FACE_EDGES[face_sum]


def _edge_cut(count, arr, A0, A1, edges, BV):
    """Get_intersection_with_face_edge (:1428-1527)."""
    if count == 4:
        return A0
    if count == 3:
        e = edges[arr[0]]
        lam = _lambda(A0, A1, BV[e[0]], BV[e[1]])
        if (lam < ZERO and abs(lam) > ZERO) or lam > 1.0:
            raise JunctionError("Get_intersection_with_face_edge (1)")
    elif count == 2:
        e = edges[arr[0]]
        lam = _lambda(A0, A1, BV[e[0]], BV[e[1]])
        if lam < ZERO and abs(lam) > ZERO:
            e = edges[arr[1]]
            lam = _lambda(A0, A1, BV[e[0]], BV[e[1]])
            if (lam < ZERO and abs(lam) > ZERO) or lam > 1.0:
                raise JunctionError("Get_intersection_with_face_edge (2)")
    else:
        raise JunctionError("Get_intersection_with_face_edge: invalid count")
    return _add(A1, _scale(_sub(A0, A1), lam))


def _inside_face(sA, edges, normals, AV, BV, BN):
    """Get_vertices_inside_face (:1687-1720)."""
    out = [v for v in sA if sum(_dot(_sub(AV[v], BV[e[0]]), BN[n]) < ZERO for e, n in zip(edges, normals)) == 4]
    if not out:
        raise JunctionError("Get_vertices_inside_face: no vertices inside face")
    return out


def _average_two_cuts(edgesA, normalsA, AV, AN, edgesB, BV, disp, vB, PB):
    """Average_point_with_two_interserctions (:1722-1778)."""
    w = []
    for e in edgesB:
        if e[0] == vB:
            w.append(e[1])
        elif e[1] == vB:
            w.append(e[0])
    w = (w + [0, 0])[:2]
    v1, v2 = 0, -1
    for e, n in zip(edgesA, normalsA):
        v1 = e[0]
        if _dot(_sub(BV[w[0]], AV[v1]), AN[n]) > ZERO and _dot(_sub(BV[w[1]], AV[v1]), AN[n]) > ZERO:
            v2 = e[1]
            break
    if v2 == -1:
        raise JunctionError("Average_point_with_two_interserctions: no edge")
    a1, a2 = _sub(AV[v1], disp), _sub(AV[v2], disp)
    l0 = _lambda(PB, BV[w[0]], a1, a2)
    l1 = _lambda(PB, BV[w[1]], a1, a2)
    PB = _add(PB, _add(BV[w[0]], _scale(_sub(PB, BV[w[0]]), l0)))
    PB = _add(PB, _add(BV[w[1]], _scale(_sub(PB, BV[w[1]]), l1)))
    return _div(PB, 3.0)


def _junction_in(sA, sB, A, B, N, distance, sumA, sumB):
    """Find_junction_points_in_gnps (:1049-1111) and the point-B cases it calls."""
    (AV, AN), (BV, BN) = A, B
    if len(sA) == 1:
        PA = AV[sA[0]]
        if len(sB) == 1:
            return PA, BV[sB[0]]
        if len(sB) in (2, 4):
            return PA, _add(PA, _scale(N, distance))
        raise JunctionError("Find_point_b_for_vertex_in_simplex_a: simplex size")
    if len(sA) == 2:
        disp = _scale(N, distance)
        eA = (_add(AV[sA[0]], disp), _add(AV[sA[1]], disp))
        if len(sB) == 2:  # Find_point_for_edge_edge_contact (:1187-1262)
            dA, dB = _sub(eA[1], eA[0]), _sub(BV[sB[1]], BV[sB[0]])
            cr = _cross(dA, dB)
            if abs(cr[0]) < ZERO and abs(cr[1]) < ZERO and abs(cr[2]) < ZERO:
                with np.errstate(divide="ignore", invalid="ignore"):
                    x1, x2 = np.float64(eA[0][0]), np.float64(eA[1][0])
                    l0 = float((np.float64(BV[sB[0]][0]) - x1) / (x2 - x1))
                    l1 = float((np.float64(BV[sB[1]][0]) - x1) / (x2 - x1))
                PB = None
                if (abs(l0) < ZERO and abs(l1 - 1) < ZERO) or (abs(l1) < ZERO and abs(l0 - 1) < ZERO):
                    PB = _div(_add(BV[sB[0]], BV[sB[1]]), 2.0)
                if l0 >= ZERO and l0 - 1 <= ZERO:
                    S0 = _add(eA[0], _scale(dA, l0))
                    PB = _div(_add(eA[0], S0), 2.0) if l1 < ZERO else _div(_add(eA[1], S0), 2.0)
                else:
                    S1 = _add(eA[0], _scale(dA, l1))
                    PB = _div(_add(eA[0], S1), 2.0) if l0 < ZERO else _div(_add(eA[1], S1), 2.0)
            else:
                lam = _lambda(BV[sB[1]], BV[sB[0]], eA[0], eA[1])
                PB = _add(BV[sB[0]], _scale(dB, lam))
            return _sub(PB, disp), PB
        if len(sB) == 4:  # Find_point_for_edge_face_contact (:1264-1328)
            edges, normals = _face(sumB)
            c, arr = [0, 0], [[-1, -1], [-1, -1]]
            for i, (e, n) in enumerate(zip(edges, normals)):
                for k in range(2):
                    if _dot(_sub(eA[k], BV[e[0]]), BN[n]) < ZERO:
                        c[k] += 1
                    elif arr[k][0] == -1:
                        arr[k][0] = i
                    else:
                        arr[k][1] = i
            A0 = _edge_cut(c[0], arr[0], eA[0], eA[1], edges, BV)
            A1 = _edge_cut(c[1], arr[1], eA[1], eA[0], edges, BV)
            PB = _scale(_add(A0, A1), 0.5)
            return _sub(PB, disp), PB
        raise JunctionError("Find_point_b_for_edge_in_simplex_a: simplex size")
    if len(sA) == 4:  # Find_point_b_for_face_in_simplex_a (:1542-1685)
        if len(sB) != 4:
            raise JunctionError("Find_point_b_for_face_in_simplex_a: simplex size")
        edgesB, normalsB = _face(sumB)
        inA = _inside_face(sA, edgesB, normalsB, AV, BV, BN)
        if len(inA) == 4:
            PA, PB = (0.0, 0.0, 0.0), (0.0, 0.0, 0.0)
            for k in range(4):
                PA, PB = _add(PA, AV[sA[k]]), _add(PB, BV[sB[k]])
            return _div(PA, 4.0), _div(PB, 4.0)
        edgesA, normalsA = _face(sumA)
        inB = _inside_face(sB, edgesA, normalsA, BV, AV, AN)
        disp = _scale(N, distance)
        if len(inA) == 0 and len(inB) == 1:
            PB = _average_two_cuts(edgesA, normalsA, AV, AN, edgesB, BV, disp, inB[0], BV[inB[0]])
            return _sub(PB, disp), PB
        if len(inA) == 1 and len(inB) == 0:  # upstream passes face B's edges for both faces here
            PA = _average_two_cuts(edgesB, normalsB, BV, BN, edgesB, BV, _scale(disp, -1.0), inA[0], AV[inA[0]])
            return PA, _add(PA, disp)
        PB = (0.0, 0.0, 0.0)
        for v in inA:
            PB = _add(_add(PB, AV[v]), disp)
        for v in inB:
            PB = _add(PB, BV[v])
        PB = _div(PB, float(len(inA) + len(inB)))
        return _sub(PB, disp), PB
    raise JunctionError("Find_junction_points_in_gnps: simplex size")


def junction_points(A, B, N, distance: float, allow_simplex3: bool = False):
    """Find_junction_points_for_gnps (:826-857) with
    Find_closest_simplices_of_gnps_in_contact (:860-966).  A and B are (vertices,
    face normals), B already moved apart when the pair interpenetrates.
    Returns (point on A, point on B); raises JunctionError where upstream fails."""
    AV, BV = A[0], B[0]
    setA, setB = set(), set()
    for i in range(8):
        for j in range(8):
            if abs(abs(_dot(_sub(AV[i], BV[j]), N)) - distance) <= ZERO:
                setA.add(i)
                setB.add(j)
    if allow_simplex3:
        for s in (setA, setB):
            if len(s) == 3:
                key = tuple(sorted(s))
                if key not in _FOURTH:
                    raise JunctionError("Complete_simplex_of_size_three: no face")
                s.add(_FOURTH[key])
    sA, sB = sorted(setA), sorted(setB)
    sumA, sumB = sum(max(1, v) for v in sA), sum(max(1, v) for v in sB)
    if len(sA) <= len(sB):
        return _junction_in(sA, sB, A, B, N, distance, sumA, sumB)
    PB, PA = _junction_in(sB, sA, B, A, _scale(N, -1.0), distance, sumB, sumA)
    return PA, PB


def outside_box(p, lo, hi) -> bool:
    """Point_3D::is_outside_cuboid (Geometry_3D.cpp:227-235)."""
    return any(p[k] - lo[k] < ZERO or p[k] - hi[k] > ZERO for k in range(3))


def pair_junction(VA, FA, VB, FB, vdw: float, lo, hi, allow_simplex3: bool = False):
    """The junction step of Label_gnps_in_window for a pair within the cutoff
    (Hoshen_Kopelman.cpp:712-746): (point on a, point on b moved back, outside
    code 1 a / 2 b), or None where upstream fails."""
    d, N, m, pen = pair_distance(VA, VB, vdw)
    A = ([tuple(float(c) for c in v) for v in VA], [tuple(float(c) for c in f[:3]) for f in FA])
    B = moved_gnp(VB, m) if pen else ([tuple(float(c) for c in v) for v in VB], [tuple(float(c) for c in f[:3]) for f in FB])
    try:
        PA, PB = junction_points(A, B, N, d, allow_simplex3)
    except JunctionError:
        return None
    if pen:
        PB = _sub(PB, m)
    return PA, PB, (1 if outside_box(PA, lo, hi) else 0) + (2 if outside_box(PB, lo, hi) else 0)


# ---------------------------------------------------------------------------
# Labels: HK76, Find_root, Merge_labels, Cleanup_labels (Hoshen_Kopelman.cpp:2908-2989, 374-425)


def hk_labels(labels, labels_labels, contacts):
    """Upstream's HK76 over `contacts` (pairs of particle indices, in order) on the
    label state (labels per particle, labels_labels per raw label), then
    Cleanup_labels: returns (proper labels, number of labels)."""
    labels, LL = list(labels), list(labels_labels)

    def root(L):
        while LL[L] <= 0:
            L = -LL[L]
            if LL[L] == 0:
                return 0
        return L

    new_label = len(LL)
    for p1, p2 in contacts:
        if labels[p1] == -1 and labels[p2] == -1:
            labels[p1] = labels[p2] = new_label
            new_label += 1
            LL.append(2)
        elif labels[p1] == -1 or labels[p2] == -1:
            q, other = (p1, p2) if labels[p1] == -1 else (p2, p1)
            L = labels[other]
            if LL[L] <= 0:
                L = root(L)
            labels[q] = L
            LL[L] += 1
        elif labels[p1] != labels[p2]:
            r1, r2 = root(labels[p1]), root(labels[p2])
            if LL[r1] <= 0 or LL[r2] <= 0:
                raise RuntimeError("Merge_labels: a root is not a root")
            if r1 < r2:
                LL[r1] += LL[r2]
                LL[r2] = -r1
            elif r2 < r1:
                LL[r2] += LL[r1]
                LL[r1] = -r2
    proper = {}
    for i, c in enumerate(LL):
        if c > 0:
            proper[i] = len(proper)
    return [proper[root(L)] if L != -1 else -1 for L in labels], len(proper)


def gnp_labels(n_gnps: int, pairs, outside, n_labels_cnt: int):
    """Make_gnp_clusters' labels (:575-616): HK76 over the GNP-GNP contacts whose
    junction points are inside the sample, Cleanup_labels, Renumber_gnp_labels."""
    lab, n = hk_labels([-1] * n_gnps, [], [(a, b) for (a, b), o in zip(pairs, outside) if o == 0])
    return [l + n_labels_cnt if l >= 0 else -1 for l in lab], n_labels_cnt + n


def mixed_labels(labels_cnt, labels_gnp, n_total: int, cnt_gnp_contacts):
    """Make_mixed_clusters' labels (:1925-1987): labels_labels starts at -1 for the
    n_total earlier labels plus one per labelled particle (Initialize_mixed_labels),
    HK76 over (CNT, n_cnts + GNP) in contact-number order, Cleanup_labels."""
    n_cnts = len(labels_cnt)
    labels = list(labels_cnt) + list(labels_gnp)
    LL = [-1] * n_total
    for L in labels:
        if L != -1:
            LL[L] += 1
    lab, n = hk_labels(labels, LL, [(c, n_cnts + g) for c, g in cnt_gnp_contacts])
    return lab[:n_cnts], lab[n_cnts:], n


# ---------------------------------------------------------------------------
# GNP point structures: Add_gnp_junction (Hoshen_Kopelman.cpp:1837-1923) and
# Compress_mixed_contacts / Add_mixed_junction (:2181-2306)


def add_gnp_junctions(contacts, n_gnps: int, tol_gnp2: float, points=None, structure=None):
    """Add_gnp_junction for every GNP-GNP contact with both junction points inside
    the sample, in contact order.  `contacts`: (a, b, dist, penetrating, point_a,
    point_b, outside).  A point of an interpenetrating pair reuses the first point
    of its GNP's structure within squared distance tol_gnp2
    (Add_gnp_point_to_vectors_if_not_repeated), else it is appended.  Returns
    (points, structure, junctions (Pa, a, Pb, b, dist), boundary-point flags)."""
    points = [tuple(p) for p in (points or [])]
    structure = [list(s) for s in (structure or [[] for _ in range(n_gnps)])]
    bp = [False] * len(points)
    n_bdd = len(points)
    junctions = []

    def add(P, g, pen):
        if pen:
            for q in structure[g]:
                dx, dy, dz = P[0] - points[q][0], P[1] - points[q][1], P[2] - points[q][2]
                if dx * dx + dy * dy + dz * dz < tol_gnp2:
                    return q
        points.append(tuple(P))
        structure[g].append(len(points) - 1)
        return len(points) - 1

    for a, b, d, pen, PA, PB, out in contacts:
        if out != 0:
            continue
        Pa, Pb = add(PA, a, pen), add(PB, b, pen)
        junctions.append((Pa, a, Pb, b, d))
        for P in (Pa, Pb):
            if P < n_bdd:
                bp[P] = True
    return points, structure, junctions, bp


def compress_mixed_contacts(contacts: dict, cnt_of_point, min_points: int, points, structure):
    """Compress_mixed_contacts: for each GNP ascending, each CNT in contact with it
    ascending, the CNT's contact points ascending are cut into runs (a new run
    when a point is min_points or more past the run's first point); each run
    keeps its first point of least junction distance, whose closest GNP point is
    appended to the GNP's structure (Add_mixed_junction).  `contacts`:
    {(P, GNP): (contact number, junction distance, closest point)}.  Returns
    (points, structure, junctions (P_cnt, CNT, P_gnp, GNP, dist), CNT element
    points added)."""
    points = [tuple(p) for p in points]
    structure = [list(s) for s in structure]
    by_gnp = {}
    for (P, g) in contacts:
        by_gnp.setdefault(g, {}).setdefault(int(cnt_of_point[P]), []).append(P)
    closest = {v[0]: v[2] for v in contacts.values()}
    junctions, elements = [], []

    def emit(Pi, Pj, c, g, d):
        points.append(tuple(closest[Pi]))
        structure[g].append(len(points) - 1)
        junctions.append((Pj, c, len(points) - 1, g, d))
        elements.append((c, Pj))

    for g in sorted(by_gnp):
        for c in sorted(by_gnp[g]):
            Ps = sorted(by_gnp[g][c])
            Pj0 = Ps[0]
            Pi_j, Pj_j, dmin = contacts[(Pj0, g)][0], Pj0, contacts[(Pj0, g)][1]
            for Pj1 in Ps[1:]:
                Pi1, d = contacts[(Pj1, g)][0], contacts[(Pj1, g)][1]
                if Pj1 - Pj0 >= min_points:
                    emit(Pi_j, Pj_j, c, g, dmin)
                    dmin, Pi_j, Pj_j, Pj0 = d, Pi1, Pj1, Pj1
                elif d < dmin:
                    dmin, Pi_j, Pj_j = d, Pi1, Pj1
            emit(Pi_j, Pj_j, c, g, dmin)
    return points, structure, junctions, elements


# ---------------------------------------------------------------------------
# Triangulation of a GNP's points (Triangulation.cpp:12-477): Bowyer-Watson on
# the points projected onto the GNP's mid-plane, from a supertriangle


def _rotate(M, p, d):
    """Point_3D::rotation (Geometry_3D.cpp:147-164): M p + d, row by row."""
    return tuple(M[r][0] * p[0] + M[r][1] * p[1] + M[r][2] * p[2] + d[r] for r in range(3))


def _circumcenter(P1, P2, P3):
    """Calculate_circumcenter: C = ((Q Pn - P Qn) x R) / (2 Rn) + P3."""
    P, Q = _sub(P1, P3), _sub(P2, P3)
    R = _cross(P, Q)
    Pn, Qn, Rn = _dot(P, P), _dot(Q, Q), _dot(R, R)
    C = _div(_cross(_sub(_scale(Q, Pn), _scale(P, Qn)), R), 2 * Rn)
    return _add(C, P3)


def _sqdist(a, b):
    dx, dy, dz = a[0] - b[0], a[1] - b[1], a[2] - b[2]
    return dx * dx + dy * dy + dz * dz


def triangulate_gnp(points, structure, l_side: float, center, rotation, face0_normal):
    """Triangulation::Generate_3d_trangulation for one GNP: its point numbers
    `structure` (into `points`), side l, centre, rotation matrix (3x3) and the
    unit normal of face 0.  Returns the edges (global point numbers) in
    upstream's order: all pairs for four points or fewer, else the edges of the
    Bowyer-Watson triangles not touching the supertriangle, first occurrences."""
    structure = [int(v) for v in structure]
    if len(structure) <= 4:  # Generate_trivial_triangulation
        return [(structure[i], structure[j]) for i in range(len(structure) - 1) for j in range(i + 1, len(structure))]
    N = tuple(float(c) for c in face0_normal)
    c0 = tuple(float(c) for c in center)
    plane = []
    for P in structure:  # Points_on_midplane
        p = tuple(float(c) for c in points[P])
        d = _dot(_sub(p, c0), N)
        plane.append(_sub(p, _scale(N, d)))
    s3 = math.sqrt(3.0)  # Generate_supertriangle
    l = float(l_side)
    sv = [(0.0, ((0.75 * s3) + 0.5) * l, 0.0), ((0.75 + (0.5 * s3)) * l, -l, 0.0)]
    sv.append((-sv[1][0], sv[1][1], 0.0))
    M = [[float(x) for x in row] for row in rotation]
    sv = [_rotate(M, v, c0) for v in sv]

    def pt(i):
        return plane[i] if i >= 0 else sv[-1 - i]

    triangles = [(-1, -2, -3)]
    for v in range(len(plane)):  # Bowyer_watson
        bad = []
        for j in range(len(triangles) - 1, -1, -1):  # Find_bad_triangles
            t = triangles[j]
            C = _circumcenter(pt(t[0]), pt(t[1]), pt(t[2]))
            if _sqdist(C, plane[v]) - _sqdist(C, pt(t[0])) <= ZERO:
                bad += [(t[0], t[1]), (t[1], t[2]), (t[2], t[0])]
                del triangles[j]
        rep = [0] * len(bad)  # Add_new_triangles
        for j in range(len(bad) - 1):
            for k in range(j + 1, len(bad)):
                if bad[j] == bad[k] or bad[j] == (bad[k][1], bad[k][0]):
                    rep[j] += 1
                    rep[k] += 1
        triangles += [(e[0], e[1], v) for e, r in zip(bad, rep) if not r]
    edges = []  # Final_triangulation_edges
    for t in triangles:
        for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            if a >= 0 and b >= 0:
                edges.append((a, b))
    keep = [not any(edges[i] == edges[j] or edges[i] == (edges[j][1], edges[j][0]) for j in range(i)) for i in range(len(edges))]
    return [(structure[a], structure[b]) for (a, b), k in zip(edges, keep) if k]  # Update_edge_numbers


# ---------------------------------------------------------------------------
# Clusters and percolation of a mixed network (Hoshen_Kopelman.cpp:2331-2738)

FAMILY = {1: 0, 11: 1, 21: 2, 12: 3, 22: 4, 32: 5, 33: 6}  # Family_map


def mixed_percolation(n_clusters, cnts_inside, gnps_inside, labels_cnt, labels_gnp, boundary_cnt, boundary_gnp, junctions_cnt, junctions_gnp,
                      junctions_mixed):
    """Make_particle_clusters (CNTs, then GNPs), Find_percolated_clusters (a
    cluster percolates along x, y, z when a particle of face 2/3/0 and one of
    face 4/5/1 carry its label; direction code 10 d + 1), the families, and
    Group_junctions (CNT-CNT and GNP-GNP junctions by the label of their
    particles, mixed ones by the CNT's).  Junctions: lists of (N1, N2) particle
    pairs.  Returns a dict of the public members upstream fills."""
    def make(inside, labels):
        clusters, iso = [[] for _ in range(n_clusters)], []
        for p in inside:
            (clusters[labels[p]] if labels[p] != -1 else iso).append(int(p))
        return clusters, iso

    cc, iso_c = make(cnts_inside, labels_cnt) if len(labels_cnt) else ([], None)
    cg, iso_g = make(gnps_inside, labels_gnp) if len(labels_gnp) else ([], None)
    dirs = [set() for _ in range(n_clusters)]
    for d, (b1, b2) in enumerate(((2, 4), (3, 5), (0, 1))):
        first = set()
        for parts, labels in ((boundary_cnt, labels_cnt), (boundary_gnp, labels_gnp)):
            if len(parts):
                first |= {labels[p] for p in parts[b1] if labels[p] != -1}
        if first:
            for parts, labels in ((boundary_cnt, labels_cnt), (boundary_gnp, labels_gnp)):
                if len(parts):
                    for p in parts[b2]:
                        if labels[p] in first:
                            dirs[labels[p]].add(10 * d + 1)
    out = {"clusters_cnt": [], "clusters_gnp": [], "isolated_cnt": [iso_c] if iso_c is not None else [],
           "isolated_gnp": [iso_g] if iso_g is not None else [], "family": []}
    perc = {}
    for i in range(n_clusters):
        if not dirs[i]:
            if cc:
                out["isolated_cnt"].append(cc[i])
            if cg:
                out["isolated_gnp"].append(cg[i])
        else:
            perc[i] = len(out["family"])
            out["family"].append(FAMILY[sum(dirs[i])])
            if cc:
                out["clusters_cnt"].append(cc[i])
            if cg:
                out["clusters_gnp"].append(cg[i])

    def group(junctions, l1, l2, n):
        groups = [[] for _ in range(n)]
        for k, (a, b) in enumerate(junctions):
            if l1[a] != l2[b]:
                raise RuntimeError("Group_junctions: the particles of a junction have different labels")
            if l1[a] in perc:
                groups[perc[l1[a]]].append(k)
        return groups

    if out["clusters_cnt"] or out["clusters_gnp"]:
        out["cluster_cnt_junctions"] = group(junctions_cnt, labels_cnt, labels_cnt, len(out["clusters_cnt"])) if junctions_cnt else []
        out["cluster_gnp_junctions"] = group(junctions_gnp, labels_gnp, labels_gnp, len(out["clusters_gnp"])) if junctions_gnp else []
        out["cluster_mix_junctions"] = group(junctions_mixed, labels_cnt, labels_gnp, len(out["clusters_cnt"])) if junctions_mixed else []
    return out


RELEVANT = {0: (2, 4), 1: (3, 5), 2: (0, 1), 3: (2, 4, 3, 5), 4: (2, 4, 0, 1), 5: (3, 5, 0, 1)}  # Get_vector_with_relevant_boundaries


def remove_nonrelevant_boundary_points(clusters_gnp, family, pts_boundary, structure, bp_flags):
    """Remove_gnp_points_in_non_relevant_boundaries (Hoshen_Kopelman.cpp:2740-2903): in a
    cluster of family 0-5, a GNP's boundary point on a face the family does not use, and not
    a junction point (bp_flags), leaves the GNP's point list and its boundary points.  Lists
    are changed in place."""
    for i, cl in enumerate(clusters_gnp):
        if family[i] == 6:
            continue
        rb = RELEVANT[family[i]]
        for g in cl:
            relevant = []
            for P, b in pts_boundary[g]:
                if b in rb or bp_flags[P]:
                    relevant.append((P, b))
                elif P in structure[g]:
                    structure[g].remove(P)
            if len(relevant) < len(pts_boundary[g]):
                pts_boundary[g] = relevant


def gnp_resistance(P1, P2, rad1: float, rad2: float, rho_surf: float, rho_t: float):
    """Direct_Electrifying::Calculate_resistance_gnp (Direct_Electrifying.cpp:1198-1232):
    R = rho L / (pi r1 r2) with rho = u . (u_x rho_surf, u_y rho_surf, u_z rho_t),
    u the unit vector from P1 to P2 (the global z axis as the through-plane
    direction, as upstream has it); None when the points coincide (L < 1e-10)."""
    P1 = tuple(float(c) for c in P1)
    P2 = tuple(float(c) for c in P2)
    L = _dist(P1, P2)
    if L < ZERO:
        return None
    u = _div(_sub(P2, P1), L)
    rho = _dot((u[0] * rho_surf, u[1] * rho_surf, u[2] * rho_t), u)
    return rho * L / (3.1415926535897932384626433832795 * rad1 * rad2)
