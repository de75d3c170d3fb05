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
