"""CPU restatement of the GNP part of the contact grid (TEST ORACLE: only tests/
call it, never the product).

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
"""
from __future__ import annotations

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
