"""CPU restatement of the CICY_geom network-to-conductance hot path — TEST ORACLE.

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker, never by the product path.  It
restates, in plain Python/numpy with the upstream operation order, the
algorithm of the upstream sources (file:line cited per function) for a
window-trimmed CNT network, and is pinned against outputs of the upstream
program itself (tests/golden/, written by tests/golden/make_golden.py from
oracle/_ref/ref_dump).

Input: the dict of arrays of a window network (x, y, z, flag, structure_ptr,
structure_idx, radii, cnts_inside, boundary_cnt_ptr/idx, boundary_pts_ptr/idx,
window) and a parameter dict (see `params_from_config`).
"""
from __future__ import annotations

import math
from collections import defaultdict

import numpy as np

ZERO = 1.0e-10                                # MathMatrix.h:18
PI = 3.1415926535897932384626433832795        # Input_Reader.h:23


def params_from_config(cfg) -> dict:
    c1, c2 = cfg.c1_c2()
    return {"gs_min": (cfg.gs_min,) * 3, "gs_overlap_cnt": 2 * cfg.radius + cfg.tunnel, "gs_overlap_gnp": 0.0, "vdw": cfg.vdw,
            "tunnel": cfg.tunnel, "min_points": cfg.min_points, "tolerance": cfg.tolerance, "V": cfg.applied_voltage,
            "rho_cnt": cfg.resistivity_cnt, "rho_matrix": cfg.resistivity_matrix, "junction": cfg.junction,
            "junction_resistance": cfg.junction_resistance, "C1": c1, "C2": c2, "resistances": tuple(cfg.resistances),
            "scope": cfg.simulation_scope}


# ---------------------------------------------------------------------------
def contact_grid(net: dict, p: dict):
    """Contact_grid::Generate_contact_grid + Fill_sectioned_domain_cnts (Contact_grid.cpp:18-295).
    Returns (n_regions[3], l_regions[3], list of region point lists)."""
    w = net["window"]  # min xyz, len xyz, max xyz
    n = [max(1, int(w[3 + a] / p["gs_min"][a])) for a in range(3)]
    l = list(p["gs_min"])
    ov_max = max(p["gs_overlap_cnt"], p["gs_overlap_gnp"])
    for a in range(3):  # Adjust_regions_if_needed (:82-102)
        if p["gs_min"][a] < 2 * ov_max:
            l[a] = 2.0 * (ov_max + ZERO)
            n[a] = 1 + int(w[3 + a] / l[a])
    ov = p["gs_overlap_cnt"]
    regions = [[] for _ in range(n[0] * n[1] * n[2])]
    sp, si = net["structure_ptr"], net["structure_idx"]
    X, Y, Z = net["x"], net["y"], net["z"]
    for cnt in net["cnts_inside"]:
        for P in si[sp[cnt]:sp[cnt + 1]]:
            P = int(P)
            pt = (X[P], Y[P], Z[P])
            abc = []
            for a in range(3):  # Calculate_region_coordinates (:163-184)
                k = int((pt[a] - w[a]) / l[a])
                k = 0 if k < 0 else (n[a] - 1 if k >= n[a] else k)
                abc.append(k)
            f = [0, 0, 0]
            for a in range(3):  # Calculate_overlapping_flags (:186-212)
                x1 = float(abc[a]) * l[a] + w[a]
                x2 = x1 + l[a]
                if abc[a] > 0 and pt[a] >= x1 and pt[a] <= x1 + ov:
                    f[a] = -1
                elif abc[a] < n[a] - 1 and pt[a] >= x2 - ov and pt[a] <= x2:
                    f[a] = 1
            t = abc[0] + abc[1] * n[0] + abc[2] * n[0] * n[1]  # Assign_point_to_regions_cnts (:214-290)
            regions[t].append(P)
            for a in range(3):
                if f[a]:
                    q = list(abc)
                    q[a] += f[a]
                    regions[q[0] + q[1] * n[0] + q[2] * n[0] * n[1]].append(P)
    return n, l, regions


def label_cnts(net: dict, p: dict, regions):
    """Hoshen_Kopelman::Label_cnts_in_window + HK76 + Cleanup_labels (Hoshen_Kopelman.cpp:249-425, 2908-2989).
    Returns labels, n_labels, point_contacts {(Pa, CNTb): (Pb, d)}, contact_elements {(CNTa, CNTb): set(Pa)}."""
    X, Y, Z, F, R = net["x"], net["y"], net["z"], net["flag"], net["radii"]
    n_cnts = len(R)
    labels = [-1] * n_cnts
    ll = []  # labels_labels

    def find_root(L):
        r = L
        while ll[r] <= 0:
            r = -ll[r]
            if ll[r] == 0:
                return 0
        return r

    def hk76(c1, c2):
        if labels[c1] == -1 and labels[c2] == -1:
            labels[c1] = labels[c2] = len(ll)
            ll.append(2)
        elif labels[c1] == -1:
            L = labels[c2]
            if ll[L] <= 0:
                L = find_root(L)
            labels[c1] = L
            ll[L] += 1
        elif labels[c2] == -1:
            L = labels[c1]
            if ll[L] <= 0:
                L = find_root(L)
            labels[c2] = L
            ll[L] += 1
        elif labels[c1] != labels[c2]:
            r1, r2 = find_root(labels[c1]), find_root(labels[c2])
            if r1 < r2:
                ll[r1] += ll[r2]
                ll[r2] = -r1
            elif r2 < r1:
                ll[r2] += ll[r1]
                ll[r1] = -r2

    pc, pcd = {}, {}
    ce = defaultdict(set)
    vdw, tun = p["vdw"], p["tunnel"]
    for reg in regions:
        k = len(reg)
        if k < 2:
            continue
        idx = np.asarray(reg, dtype=np.int64)
        cn = F[idx]
        for j in range(k - 1):
            P1 = int(idx[j]); c1 = int(cn[j])
            rest = idx[j + 1:]
            c2s = cn[j + 1:]
            dx = X[P1] - X[rest]; dy = Y[P1] - Y[rest]; dz = Z[P1] - Z[rest]
            d = np.sqrt(dx * dx + dy * dy + dz * dz) - R[c1] - R[c2s]  # Point_3D::distance_to (Geometry_3D.cpp:64-70)
            d = np.where(d < vdw, vdw, d)
            hit = np.nonzero((c2s != c1) & (d <= tun))[0]
            for h in hit:
                P2, c2, dj = int(rest[h]), int(c2s[h]), float(d[h])
                hk76(c1, c2)
                ca, cb = min(c1, c2), max(c1, c2)
                pa, pb = (P1, P2) if c1 < c2 else (P2, P1)
                ce[(ca, cb)].add(pa)
                key = (pa, cb)
                if key not in pc or pcd[key] > dj:
                    pcd[key] = dj
                    pc[key] = pb
    proper, n_labels = {}, 0  # Cleanup_labels
    for i, v in enumerate(ll):
        if v > 0:
            proper[i] = n_labels
            n_labels += 1
    labels = [proper[find_root(L)] if L != -1 else -1 for L in labels]
    return np.array(labels, dtype=np.int32), n_labels, {k: (pc[k], pcd[k]) for k in pc}, ce


def compress_junctions(net: dict, p: dict, point_contacts: dict, ce: dict):
    """Compress_cnt_cnt_contact_segments + Complete_cnt_elements (Hoshen_Kopelman.cpp:443-572).
    Returns junctions [(P1, N1, P2, N2, d)], elements {cnt: sorted list}."""
    mp = p["min_points"]
    junctions = []
    elements = defaultdict(set)
    for (ci, cj) in sorted(ce):
        pts = sorted(ce[(ci, cj)])
        Pi0 = pts[0]
        Pj0, d = point_contacts[(Pi0, cj)]
        Pi_j, Pj_j, dmin = Pi0, Pj0, d
        for Pi1 in pts[1:]:
            Pj1, d = point_contacts[(Pi1, cj)]
            if Pi1 - Pi0 >= mp or abs(Pj1 - Pj0) >= mp:
                junctions.append((Pi_j, ci, Pj_j, cj, dmin))
                elements[ci].add(Pi_j)
                elements[cj].add(Pj_j)
                dmin, Pi_j, Pj_j = d, Pi1, Pj1
            elif d < dmin:
                dmin, Pi_j, Pj_j = d, Pi1, Pj1
            Pi0, Pj0 = Pi1, Pj1
        junctions.append((Pi_j, ci, Pj_j, cj, dmin))
        elements[ci].add(Pi_j)
        elements[cj].add(Pj_j)
    sp, si = net["structure_ptr"], net["structure_idx"]
    out = {}
    for c, s in elements.items():
        s.add(int(si[sp[c]]))
        s.add(int(si[sp[c + 1] - 1]))
        out[c] = sorted(s)
    return junctions, out


def isolated_lists(net: dict, labels, n_labels, clusters_all_labels=None):
    """HoKo->isolated_cnt (Hoshen_Kopelman.cpp:2331-2363, 2527-2539): the CNTs with label -1 in
    cnts_inside order, then every non-percolated cluster in label order (its CNTs in cnts_inside order)."""
    tmp = [[] for _ in range(n_labels)]
    iso0 = []
    for c in net["cnts_inside"]:
        if labels[c] != -1:
            tmp[labels[c]].append(int(c))
        else:
            iso0.append(int(c))
    perc = set(clusters_all_labels or ())
    return [iso0] + [tmp[L] for L in range(n_labels) if L not in perc]


def percolation(net: dict, labels, n_labels, junctions, with_isolated: bool = False):
    """Make_particle_clusters, Find_percolated_clusters, Family_map, Group_junctions
    (Hoshen_Kopelman.cpp:2331-2710).  Returns clusters (CNT lists), families, cluster junction lists
    (and, with_isolated, HoKo->isolated_cnt)."""
    bptr, bidx = net["boundary_cnt_ptr"], net["boundary_cnt_idx"]
    face = lambda f: [int(c) for c in bidx[bptr[f]:bptr[f + 1]]]
    tmp = [[] for _ in range(n_labels)]
    for c in net["cnts_inside"]:
        if labels[c] != -1:
            tmp[labels[c]].append(int(c))
    dirs = [set() for _ in range(n_labels)]
    for d, (b1, b2) in enumerate([(2, 4), (3, 5), (0, 1)]):
        s1 = {labels[c] for c in face(b1) if labels[c] != -1}
        if s1:
            for c in face(b2):
                if labels[c] in s1:
                    dirs[labels[c]].add(10 * d + 1)
    fam_of = {1: 0, 11: 1, 21: 2, 12: 3, 22: 4, 32: 5, 33: 6}
    clusters, families, perc = [], [], {}
    for L in range(n_labels):
        if dirs[L]:
            perc[L] = len(clusters)
            clusters.append(tmp[L])
            families.append(fam_of[sum(dirs[L])])
    cj = [[] for _ in clusters]
    for i, (P1, N1, P2, N2, d) in enumerate(junctions):
        assert labels[N1] == labels[N2]
        if labels[N1] in perc:
            cj[perc[labels[N1]]].append(i)
    if with_isolated:
        return clusters, families, cj, isolated_lists(net, labels, n_labels, perc)
    return clusters, families, cj


BOUNDARIES = {0: [2, 4], 1: [3, 5], 2: [0, 1], 3: [2, 4, 3, 5], 4: [2, 4, 0, 1], 5: [3, 5, 0, 1], 6: [2, 4, 3, 5, 0, 1]}


def cnt_resistance(net, P1, P2, radius, rho):
    """Calculate_resistance_cnt (Direct_Electrifying.cpp:611-646)."""
    X, Y, Z = net["x"], net["y"], net["z"]
    length = 0.0
    for i in range(P1, P2):
        dx, dy, dz = X[i] - X[i + 1], Y[i] - Y[i + 1], Z[i] - Z[i + 1]
        length = length + math.sqrt(dx * dx + dy * dy + dz * dz)
    return rho * length / (PI * radius * radius)


def assemble(net: dict, p: dict, cluster, family, r_flag, elements, junctions, cj):
    """Get_global_nodes, LM_matrix_for_cnts, Fill_sparse_stiffness_matrix, From_2d_to_1d_vectors,
    Initial_guess_for_CG (Direct_Electrifying.cpp:11-1470).  Returns a dict with the SSS system."""
    bnd = BOUNDARIES[family]
    reserved = len(bnd)
    lmm = {}
    bpp, bpi = net["boundary_pts_ptr"], net["boundary_pts_idx"]
    for k, b in enumerate(bnd):  # Map_points_at_boundaries (:217-246)
        for P in bpi[bpp[b]:bpp[b + 1]]:
            lmm[int(P)] = k
    nodes = reserved
    for c in cluster:  # LM_matrix_for_cnts (:139-215)
        e = elements[c]
        assert len(e) > 1
        if e[0] not in lmm:
            lmm[e[0]] = nodes; nodes += 1
        for P in e[1:-1]:
            lmm[P] = nodes; nodes += 1
        if e[-1] not in lmm:
            lmm[e[-1]] = nodes; nodes += 1
    col = [dict() for _ in range(nodes)]
    diag = [0.0] * nodes
    R = net["radii"]
    for c in cluster:  # Fill_2d_matrices_cnts + Three_points_in_element (:489-608)
        e = elements[c]
        if len(e) == 3 and lmm[e[0]] == lmm[e[2]]:
            g = 1.0 + 1.0 if not r_flag else 1 / cnt_resistance(net, e[0], e[1], R[c], p["rho_cnt"]) + \
                1 / cnt_resistance(net, e[1], e[2], R[c], p["rho_cnt"])
            n1, n2 = lmm[e[0]], lmm[e[1]]
            diag[n1] += g; diag[n2] += g
            col[n2][n1] = -g
            continue
        for P1, P2 in zip(e[:-1], e[1:]):
            g = 1 / cnt_resistance(net, P1, P2, R[c], p["rho_cnt"]) if r_flag else 1.0
            n1, n2 = lmm[P1], lmm[P2]
            diag[n1] += g; diag[n2] += g
            col[max(n1, n2)][min(n1, n2)] = -g
    for j in cj:  # Fill_2d_matrices_cnt_junctions + Calculate_junction_resistance (:737-901)
        P1, N1, P2, N2, d = junctions[j]
        if P1 not in lmm or P2 not in lmm:
            continue
        n1, n2 = lmm[P1], lmm[P2]
        g = 1.0
        if r_flag:
            if p["junction"] == "constant":
                Re = p["junction_resistance"]
            else:
                jl1, jl2 = R[N1] + R[N1], R[N2] + R[N2]
                A = jl1 * jl1 if jl1 - jl2 < ZERO else jl2 * jl2
                Re = p["C1"] * d * math.exp(p["C2"] * d) / A
            g = 1 / Re
        hi, lo = max(n1, n2), min(n1, n2)
        if n1 >= reserved and n2 >= reserved:
            diag[n1] += g; diag[n2] += g
            col[hi][lo] = -g
        elif reserved > 2:
            diag[n1] += g; diag[n2] += g
            col[hi][lo] = col[hi].get(lo, 0.0) - g
    V = p["V"] if r_flag else float(nodes)  # Get_voltage_vector (:1472-1500)
    vef = [0.0] * reserved
    for i in range(1, reserved):
        vef[i] = vef[i - 1] + V
    n = nodes - reserved
    rp, ci, val, b = [0], [], [], [0.0] * n
    for i in range(reserved, nodes):  # From_2d_to_1d_vectors (:1329-1394)
        for cc in sorted(col[i]):
            if cc >= reserved:
                val.append(col[i][cc]); ci.append(cc - reserved)
            else:
                b[i - reserved] = b[i - reserved] - col[i][cc] * vef[cc]
        rp.append(len(val))
    dg = np.array(diag[reserved:])
    assert np.all(np.abs(dg) >= ZERO), "zero on the diagonal (Direct_Electrifying.cpp:458-484)"
    x0 = np.zeros(n)
    if r_flag and reserved == 2:  # Initial_guess_for_cnt_nodes (:1434-1470)
        w = net["window"]
        Lw, mx = w[3 + family], w[6 + family]
        coord = [net["x"], net["y"], net["z"]][family]
        for c in cluster:
            for P in elements[c]:
                nd = lmm[P]
                if nd >= 2:
                    x0[nd - reserved] = (p["V"] / Lw) * (mx - coord[P])
    return {"nodes": nodes, "reserved": reserved, "row_ptr": np.array(rp, np.int64), "col_ind": np.array(ci, np.int64),
            "values": np.array(val), "diag": dg, "b": np.array(b), "x0": x0, "vef": np.array(vef), "lmm": lmm}


def full_matrix(S):
    import scipy.sparse as sp

    n = len(S["diag"])
    L = sp.csr_matrix((S["values"], S["col_ind"], S["row_ptr"]), shape=(n, n))
    return (L + L.T + sp.diags(S["diag"])).tocsr()


def solve_cg(S, tol):
    """Solve_DEA_equations_CG_SSS (Direct_Electrifying.cpp:1538-1659): Jacobi-PCG, stop at |r| <= tol |r0|."""
    A = full_matrix(S)
    n = len(S["diag"])
    x = S["x0"].copy()
    r = S["b"] - A @ x
    minv = 1 / S["diag"]
    y = minv * r
    pvec = y.copy()
    R0 = tol * math.sqrt(r @ r)
    k = 0
    for k in range(1, 300 * S["nodes"] + 1):
        ap = A @ pvec
        rr0 = y @ r
        with np.errstate(invalid="ignore", divide="ignore"):  # upstream's 0/0 on a zero initial residual gives NaN
            alpha = rr0 / (pvec @ ap)
        x += alpha * pvec
        r -= alpha * ap
        if math.sqrt(r @ r) <= R0:
            break
        y = minv * r
        beta = (y @ r) / rr0
        pvec = y + beta * pvec
    volt = np.concatenate([S["vef"], x]) if n else S["vef"].copy()
    return volt, k


def grounded_mask(S):
    """Free nodes whose connected component touches a prescribed-voltage node.

    After the backbone of a multi-direction cluster, a single-direction pass can
    hold islands that carried current only between the other faces; their
    Laplacian block is singular (zero row sums) and their voltages are not
    determined by the system, so accuracy checks exclude them."""
    from scipy.sparse.csgraph import connected_components

    A = full_matrix(S)
    n = A.shape[0]
    if n == 0:
        return np.zeros(0, bool)
    nc, lab = connected_components(A, directed=False)
    rs = np.abs(np.asarray(A.sum(1)).ravel())
    grounded = np.zeros(nc, bool)
    np.logical_or.at(grounded, lab, rs > 1e-12 * np.abs(S["diag"]))
    return grounded[lab]


def solve_direct(S):
    """FP64 direct solve of the same system (the accuracy reference for voltages)."""
    import scipy.sparse.linalg as spl

    A = full_matrix(S)
    m = grounded_mask(S)
    x = np.full(len(S["b"]), np.nan)
    if m.any():
        x[m] = spl.spsolve(A[m][:, m].tocsc(), S["b"][m])
    return np.concatenate([S["vef"], x])


def cnt_volume(net, P1, P2, radius):
    """CNT_volume_between_two_points (Backbone_Network.cpp:558-574): the polyline length from
    P1 to P2 times PI r^2, as (length * PI * r) * r."""
    X, Y, Z = net["x"], net["y"], net["z"]
    length = 0.0
    for i in range(P1, P2):
        dx, dy, dz = X[i] - X[i + 1], Y[i] - Y[i + 1], Z[i] - Z[i + 1]
        length = length + math.sqrt(dx * dx + dy * dy + dz * dz)
    return length * PI * radius * radius


def new_volumes() -> dict:
    """Backbone_Network's volume members as its constructor sets them (Backbone_Network.h:37-48)."""
    return {"volumes_cnt": [0.0] * 8, "volumes_gnp": [0.0] * 8, "dead_branches": [0.0] * 7, "dead_gnps": [0.0] * 7}


def backbone(cluster, cj, elements, junctions, lmm, volt, trim=True, net=None, family=None, vols=None):
    """Find_zero_current, Find_backbone_cnts, Calculate_cnt_volumes,
    Remove_junctions_with_dead_particles_cnts (Backbone_Network.cpp:64-409, 412-556, 950-992).
    With `vols` (see new_volumes) the backbone and dead-branch volumes of the cluster's CNTs are
    added to its `family`, CNTs visited last to first as upstream does (Backbone_Network.cpp:325)."""
    imax = ZERO
    cur = []
    for c in cluster:
        e = elements[c]
        I = [abs(volt[lmm[a]] - volt[lmm[b]]) for a, b in zip(e[:-1], e[1:])]
        cur.append(I)
        imax = max([imax] + I)
    for j in cj:
        P1, _, P2, _, _ = junctions[j]
        imax = max(imax, abs(volt[lmm[P1]] - volt[lmm[P2]]))
    zero = imax * 1e-9
    idx = []
    for I in cur:
        i1 = i2 = -1
        for j, v in enumerate(I):
            if v - zero > ZERO:
                if i1 == -1:
                    i1 = j
            elif i1 != -1 and i2 == -1:
                i2 = j
                break
        idx.append((i1, i2))
    if vols is not None:
        R = net["radii"]
        for c, (i1, i2) in reversed(list(zip(cluster, idx))):
            e = elements[c]
            if i1 == -1:
                vols["dead_branches"][family] = vols["dead_branches"][family] + cnt_volume(net, e[0], e[-1], R[c])
                continue
            vols["dead_branches"][family] = vols["dead_branches"][family] + cnt_volume(net, e[0], e[i1], R[c])
            if i2 == -1:
                vb = cnt_volume(net, e[i1], e[-1], R[c])
            else:
                vb = cnt_volume(net, e[i1], e[i2], R[c])
                vols["dead_branches"][family] = vols["dead_branches"][family] + cnt_volume(net, e[i2], e[-1], R[c])
            vols["volumes_cnt"][family] = vols["volumes_cnt"][family] + vb
    new_cluster = []
    for c, (i1, i2) in zip(cluster, idx):
        if not trim:
            new_cluster.append(c)
            continue
        if i1 == -1:
            elements[c] = []
        else:
            e = elements[c]
            elements[c] = e[i1:(i2 + 1 if i2 != -1 else len(e))]
            new_cluster.append(c)
    new_cj = []
    for j in cj:
        P1, N1, P2, N2, _ = junctions[j]
        if elements.get(N1) and elements.get(N2) and P1 in elements[N1] and P2 in elements[N2]:
            new_cj.append(j)
    return new_cluster, new_cj, zero


def family_fractions(net, isolated, vols):
    """Calculate_percolated_families_fractions with Calculate_volume_of_non_percolated_cnts
    (Electrical_analysis.cpp:678-786) for a CNT network: volumes_cnt[7] becomes the dead-branch
    plus non-percolated volume; returns total_volumes and fractions (8 each)."""
    total_dead, total_dead_gnps = 0.0, 0.0
    for i in range(7):
        total_dead = total_dead + vols["dead_branches"][i]
        total_dead_gnps = total_dead_gnps + vols["dead_gnps"][i]
    sp, si = net["structure_ptr"], net["structure_idx"]
    np_cnts = 0.0
    for lst in isolated:
        for c in lst:
            np_cnts = np_cnts + cnt_volume(net, int(si[sp[c]]), int(si[sp[c + 1] - 1]), net["radii"][c])
    vols["volumes_cnt"][7] = total_dead + np_cnts
    vols["volumes_gnp"][7] = total_dead_gnps + 0.0
    vc, vg = vols["volumes_cnt"], vols["volumes_gnp"]
    total = [0.0] * 8
    tv = 0.0
    for i in range(8):
        total[i] = total[i] + vc[i] + vg[i]
        tv = tv + vc[i] + vg[i]
    with np.errstate(divide="ignore", invalid="ignore"):
        fr = [float(np.float64(total[i]) / np.float64(tv)) for i in range(8)]
    return total, fr


def boundary_current(net, p, bcnt, elements, lmm, volt):
    """Currents_through_boundary_cnts / Current_of_element_in_boundary (Electrical_analysis.cpp:499-605)."""
    I = 0.0
    R = net["radii"]
    for c in bcnt:
        e = elements.get(c) or []
        if not e:
            continue
        for P1, P2 in ((e[0], e[1]), (e[-1], e[-2])):
            if P1 not in lmm or lmm[P1] > 1 or P2 not in lmm:
                continue
            V = volt[lmm[P2]] - volt[lmm[P1]]
            Re = cnt_resistance(net, min(P1, P2), max(P1, P2), R[c], p["rho_cnt"])
            I = I + V / Re
    return I


def network_to_conductance(net: dict, p: dict, solver: str = "cg") -> dict:
    """The whole hot path for one window (App_Network_3D.cpp:140-179, Electrical_analysis.cpp:10-145,
    :229-473, :873-987).  solver "cg" follows upstream; "direct" uses the FP64 direct solve."""
    n, l, regions = contact_grid(net, p)
    labels, n_labels, pc, ce = label_cnts(net, p, regions)
    junctions, elements = compress_junctions(net, p, pc, ce)
    clusters, families, cj, isolated = percolation(net, labels, n_labels, junctions, with_isolated=True)
    vols = new_volumes()
    out = {"regions": regions, "labels": labels, "n_labels": n_labels, "point_contacts": pc, "junctions": junctions,
           "elements": {k: list(v) for k, v in elements.items()}, "clusters": [list(c) for c in clusters], "families": families,
           "cluster_junctions": [list(c) for c in cj], "systems": [], "backbone": []}
    parallel = [[], [], []]
    bptr, bidx = net["boundary_cnt_ptr"], net["boundary_cnt_idx"]
    elems = {k: list(v) for k, v in elements.items()}
    for k, (cl, fam) in enumerate(zip(clusters, families)):
        if p["scope"] >= 2:
            break
        S = assemble(net, p, cl, fam, 0, elems, junctions, cj[k])
        volt, it = solve_cg(S, p["tolerance"]) if solver == "cg" else (solve_direct(S), 0)
        S["voltages"], S["iterations"] = volt, it
        out["systems"].append(("unit", k, S))
        cl2, cj2, zero = backbone(cl, cj[k], elems, junctions, S["lmm"], volt, trim=p["scope"] == 0, net=net, family=fam, vols=vols)
        clusters[k], cj[k] = cl2, cj2
        out["backbone"].append({"cluster": list(cl2), "junctions": list(cj2), "zero_current": zero})
        if p["scope"] != 0:
            continue
        dir_bits = {0: 1, 1: 2, 2: 4, 3: 3, 4: 5, 5: 6, 6: 7}[fam]
        for d in range(3):
            if not (dir_bits >> d & 1) or not p["resistances"][d]:
                continue
            S2 = assemble(net, p, cl2, d, 1, elems, junctions, cj2)
            v2, it2 = solve_cg(S2, p["tolerance"]) if solver == "cg" else (solve_direct(S2), 0)
            S2["voltages"], S2["iterations"] = v2, it2
            out["systems"].append((d, k, S2))
            b1 = [2, 3, 0][d]
            I = boundary_current(net, p, [int(c) for c in bidx[bptr[b1]:bptr[b1 + 1]]], elems, S2["lmm"], v2)
            with np.errstate(divide="ignore", invalid="ignore"):  # a zero current gives upstream's inf / nan R
                parallel[d].append(p["V"] / I)
    w = net["window"]
    L = [w[3], w[4], w[5]]
    A = [w[4] * w[5], w[3] * w[5], w[3] * w[4]]
    res = []
    for d in range(3):
        if not parallel[d]:
            res.append(p["rho_matrix"] * L[d] / A[d])
        elif len(parallel[d]) == 1:
            res.append(parallel[d][0])
        else:
            s = 0.0
            for r in parallel[d]:
                s = s + 1 / r
            res.append(1 / s)
    out["elements_backbone"] = elems
    out["resistances"] = res
    if p["scope"] < 2:
        out["volumes_before_fractions"] = {k: list(v) for k, v in vols.items()}
        out["total_volumes"], out["fractions"] = family_fractions(net, isolated, vols)
        out["volumes"] = vols
    return out
