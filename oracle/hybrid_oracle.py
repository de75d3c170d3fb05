"""CPU restatement of the electrical stage of a mixed CNT/GNP network — TEST ORACLE.

Test infrastructure only (imported by tests/ as the checker, never by the
product path).  It restates, in plain Python with upstream's operation order,
Electrical_analysis::Perform_analysis_on_clusters for GNP_CNT_mix
(Electrical_analysis.cpp:10-145, 229-675): the node maps of CNT and GNP points,
the stiffness matrix with CNT resistors, CNT-CNT, CNT-GNP and GNP-GNP
junctions and the resistors of every GNP's triangulation, the unit-resistor
solve, the backbone of CNTs and GNPs with its cascade of removals, the
real-resistor solve per percolated direction and the boundary currents of CNTs
and GNPs.  Pinned against upstream's own stage-by-stage dumps
(tests/golden/gnp_hybrid_electrical.npz, oracle/gnp_dump.cpp "electrical").

State: a dict `h` holding upstream's public members as plain lists
  clusters_cnt, clusters_gnp     percolated clusters (lists of particles)
  family                         family of each cluster
  cluster_cnt_junctions, cluster_gnp_junctions, cluster_mix_junctions
  junctions_cnt/gnp/mixed        (P1, N1, P2, N2, distance) tuples
  elements                       CNT -> sorted list of element points
  structure_gnp                  GNP -> list of GNP point numbers
  pts_boundary                   GNP -> list of (point, face) boundary points
and the inputs
  net                            CNT window network arrays (cicy_oracle layout)
  points_gnp                     GNP points (x, y, z)
  gnp_t, gnp_volume, gnp_geom    per GNP: thickness, volume, (l, centre, rotation, face-0 normal)
  boundary_cnt, boundary_gnp     particles on each face; boundary_cnt_pts, boundary_gnp_pts their points
"""
from __future__ import annotations

import math

import numpy as np

from . import cicy_oracle as O
from . import gnp_oracle as G

ZERO = O.ZERO


def lm_matrices(h, j, family):
    """Get_global_nodes, LM_matrix_for_cnts, LM_matrix_for_gnps with Map_points_at_boundaries
    (Direct_Electrifying.cpp:123-348): reserved node per prescribed face, then CNT element
    points, then GNP points in cluster and point-list order."""
    bnd = O.BOUNDARIES[family]
    reserved = len(bnd)
    nodes = reserved
    lmm_c, lmm_g = {}, {}
    if h["clusters_cnt"] and h["clusters_cnt"][j]:
        for k, b in enumerate(bnd):
            for P in h["boundary_cnt_pts"][b]:
                lmm_c[int(P)] = k
        for c in h["clusters_cnt"][j]:
            e = h["elements"][c]
            if e[0] not in lmm_c:
                lmm_c[e[0]] = nodes
                nodes += 1
            for P in e[1:-1]:
                lmm_c[P] = nodes
                nodes += 1
            if e[-1] not in lmm_c:
                lmm_c[e[-1]] = nodes
                nodes += 1
    if h["clusters_gnp"] and h["clusters_gnp"][j]:
        for k, b in enumerate(bnd):
            for P in h["boundary_gnp_pts"][b]:
                lmm_g[int(P)] = k
        for g in h["clusters_gnp"][j]:
            for P in h["structure_gnp"][g]:
                if P not in lmm_g:
                    lmm_g[P] = nodes
                    nodes += 1
    return reserved, nodes, lmm_c, lmm_g


def junction_resistance(p, d, jl1, jl2):
    """Calculate_junction_resistance (Direct_Electrifying.cpp:854-901); jl: diameter of a CNT
    (its radius doubled by the caller's type test), thickness of a GNP."""
    if p["junction"] == "constant":
        return p["junction_resistance"]
    A = jl1 * jl1 if jl1 - jl2 < ZERO else jl2 * jl2
    return p["C1"] * d * math.exp(p["C2"] * d) / A


def triangulate(h, g):
    l, cen, rot, n0 = h["gnp_geom"][g]
    return G.triangulate_gnp(h["points_gnp"], h["structure_gnp"][g], l, cen, rot, n0)


def assemble(h, p, j, family, r_flag):
    """Compute_voltage_field's assembly (Direct_Electrifying.cpp:11-113, 351-1394): the SSS system
    of cluster j, the node maps, the GNP points with a CNT radius and the GNP triangulations
    (h["tri"], kept between passes as upstream keeps gnps[].triangulation)."""
    net = h["net"]
    R = net["radii"]
    reserved, nodes, lmm_c, lmm_g = lm_matrices(h, j, family)
    col = [dict() for _ in range(nodes)]
    diag = [0.0] * nodes

    def add_new(n1, n2, g):
        diag[n1] += g
        diag[n2] += g
        col[max(n1, n2)][min(n1, n2)] = -g

    def add_existing(n1, n2, g):
        diag[n1] += g
        diag[n2] += g
        hi, lo = max(n1, n2), min(n1, n2)
        col[hi][lo] = col[hi].get(lo, 0.0) - g

    if h["clusters_cnt"] and h["clusters_cnt"][j]:
        for c in h["clusters_cnt"][j]:  # Fill_2d_matrices_cnts, Three_points_in_element (:489-608)
            e = h["elements"][c]
            if len(e) == 3 and lmm_c[e[0]] == lmm_c[e[2]]:
                g = 1.0 + 1.0 if not r_flag else 1 / O.cnt_resistance(net, e[0], e[1], R[c], p["rho_cnt"]) + \
                    1 / O.cnt_resistance(net, e[1], e[2], R[c], p["rho_cnt"])
                n1, n2 = lmm_c[e[0]], lmm_c[e[1]]
                diag[n1] += g
                diag[n2] += g
                col[n2][n1] = -g
                continue
            for P1, P2 in zip(e[:-1], e[1:]):
                g = 1 / O.cnt_resistance(net, P1, P2, R[c], p["rho_cnt"]) if r_flag else 1.0
                add_new(lmm_c[P1], lmm_c[P2], g)
        for jj in h["cluster_cnt_junctions"][j] if h["cluster_cnt_junctions"] else []:  # :737-852
            P1, N1, P2, N2, d = h["junctions_cnt"][jj]
            if P1 not in lmm_c or P2 not in lmm_c:
                continue
            n1, n2 = lmm_c[P1], lmm_c[P2]
            g = 1 / junction_resistance(p, d, R[N1] + R[N1], R[N2] + R[N2]) if r_flag else 1.0
            if n1 >= reserved and n2 >= reserved:
                add_new(n1, n2, g)
            elif reserved > 2:
                add_existing(n1, n2, g)
    cnt_rad = {}
    for jj in h["cluster_mix_junctions"][j] if h["cluster_mix_junctions"] else []:  # Fill_2d_matrices_mixed_junctions (:903-1019)
        Pc, Nc, Pg, Ng, d = h["junctions_mixed"][jj]
        n1, n2 = lmm_c.get(Pc, -1), lmm_g.get(Pg, -1)
        if n1 == -1 or n2 == -1:
            continue
        g = 1 / junction_resistance(p, d, R[Nc] + R[Nc], h["gnp_t"][Ng]) if r_flag else 1.0
        if n1 >= reserved and n2 >= reserved:
            add_new(n1, n2, g)
        elif reserved > 2:
            add_existing(n1, n2, g)
        cnt_rad[Pg] = R[Nc]
    if h["clusters_gnp"] and h["clusters_gnp"][j]:
        for g_i in h["clusters_gnp"][j]:  # Fill_2d_matrices_gnp (:1021-1190)
            if not r_flag or not h["tri"].get(g_i):
                h["tri"][g_i] = triangulate(h, g_i)
                if len(h["structure_gnp"][g_i]) > 4 and not h["tri"][g_i]:
                    raise RuntimeError("Bowyer-Watson gave no triangulation for more than 4 points")
            t = h["gnp_t"][g_i]
            for v1, v2 in reversed(h["tri"][g_i]):
                n1, n2 = lmm_g[v1], lmm_g[v2]
                g = 1.0
                if r_flag:
                    r1 = cnt_rad.get(v1, t / 2)
                    r2 = cnt_rad.get(v2, t / 2)
                    Re = G.gnp_resistance(h["points_gnp"][v1], h["points_gnp"][v2], r1, r2, p["rho_gnp_surf"], p["rho_gnp_t"])
                    if Re is None:
                        raise RuntimeError("Calculate_resistance_gnp: coincident points")
                    g = 1 / Re
                add_new(n1, n2, g)
        for jj in h["cluster_gnp_junctions"][j] if h["cluster_gnp_junctions"] else []:  # Fill_2d_matrices_gnp_junctions (:1234-1319)
            P1, N1, P2, N2, d = h["junctions_gnp"][jj]
            n1, n2 = lmm_g.get(P1, -1), lmm_g.get(P2, -1)
            if n1 == -1 or n2 == -1:
                continue
            g = 1 / junction_resistance(p, d, h["gnp_t"][N1], h["gnp_t"][N2]) if r_flag else 1.0
            add_new(n1, n2, g)
    V = p["V"] if r_flag else float(nodes)  # Get_voltage_vector (:1472-1500)
    vef = [0.0] * reserved
    for i in range(1, reserved):
        vef[i] = vef[i - 1] + V
    n = nodes - reserved
    rp, ci, val, b = [0], [], [], [0.0] * n
    for i in range(reserved, nodes):  # From_2d_to_1d_vectors (:1329-1394)
        for cc in sorted(col[i]):
            if cc >= reserved:
                val.append(col[i][cc])
                ci.append(cc - reserved)
            else:
                b[i - reserved] = b[i - reserved] - col[i][cc] * vef[cc]
        rp.append(len(val))
    dg = np.array(diag[reserved:])
    if not np.all(np.abs(dg) >= ZERO):
        raise RuntimeError("zero on the diagonal (Direct_Electrifying.cpp:458-484)")
    x0 = np.zeros(n)
    if r_flag and reserved == 2 and h["clusters_cnt"] and h["clusters_cnt"][j]:  # Initial_guess_for_cnt_nodes (:1434-1470)
        w = net["window"]
        Lw, mx = w[3 + family], w[6 + family]
        coord = [net["x"], net["y"], net["z"]][family]
        for c in h["clusters_cnt"][j]:
            for P in h["elements"][c]:
                nd = lmm_c[P]
                if nd >= 2:
                    x0[nd - reserved] = (p["V"] / Lw) * (mx - coord[P])
    return {"nodes": nodes, "reserved": reserved, "row_ptr": np.array(rp, np.int64), "col_ind": np.array(ci, np.int64),
            "values": np.array(val), "diag": dg, "b": np.array(b), "x0": x0, "vef": np.array(vef), "lmm_cnt": lmm_c, "lmm_gnp": lmm_g,
            "cnt_rad": cnt_rad}


def remove_point(P, lst):
    """Remove_point_from_vector (Backbone_Network.cpp:1041-1055): the first occurrence."""
    for k, q in enumerate(lst):
        if q == P:
            del lst[k]
            return


def backbone(h, j, S, volt, vols):
    """Determine_backbone_network for a mixed cluster (Backbone_Network.cpp:11-1127):
    zero current over CNT elements, all junction kinds and the GNP triangulations;
    the CNT backbone (with volumes); the GNP backbone (junctions below the zero
    current, dead GNPs and their junctions until none is left, CNTs left without
    elements, GNP volumes); CNT junctions with dead particles.  Returns the zero current."""
    lc, lg = S["lmm_cnt"], S["lmm_gnp"]
    fam = h["family"][j]
    imax = ZERO
    cur = []
    cc = h["clusters_cnt"][j] if h["clusters_cnt"] else []
    for c in cc:
        e = h["elements"][c]
        I = [abs(volt[lc[a]] - volt[lc[b]]) for a, b in zip(e[:-1], e[1:])]
        cur.append(I)
        for v in I:
            if v > imax:
                imax = v
    for jj in h["cluster_cnt_junctions"][j] if h["cluster_cnt_junctions"] else []:
        P1, _, P2, _, _ = h["junctions_cnt"][jj]
        v = abs(volt[lc[P1]] - volt[lc[P2]])
        if v > imax:
            imax = v
    cg = h["clusters_gnp"][j] if h["clusters_gnp"] else []
    for g in cg:
        for v1, v2 in h["tri"].get(g, []):
            v = abs(volt[lg[v1]] - volt[lg[v2]])
            if v > imax:
                imax = v
    for jj in h["cluster_gnp_junctions"][j] if h["cluster_gnp_junctions"] else []:
        P1, _, P2, _, _ = h["junctions_gnp"][jj]
        v = abs(volt[lg[P1]] - volt[lg[P2]])
        if v > imax:
            imax = v
    for jj in h["cluster_mix_junctions"][j] if h["cluster_mix_junctions"] else []:
        P1, _, P2, _, _ = h["junctions_mixed"][jj]
        v = abs(volt[lc[P1]] - volt[lg[P2]])
        if v > imax:
            imax = v
    zero = imax * 1e-9
    net = h["net"]
    if cc:  # Find_backbone_cnts, Calculate_cnt_volumes (:313-556), CNTs last to first
        for i in range(len(cc) - 1, -1, -1):
            c = cc[i]
            i1 = i2 = -1
            for k, v in enumerate(cur[i]):
                if v - zero > ZERO:
                    if i1 == -1:
                        i1 = k
                elif i1 != -1 and i2 == -1:
                    i2 = k
                    break
            e = h["elements"][c]
            r = net["radii"][c]
            if i1 == -1:
                vols["dead_branches"][fam] = vols["dead_branches"][fam] + O.cnt_volume(net, e[0], e[-1], r)
                h["elements"][c] = []
            else:
                vols["dead_branches"][fam] = vols["dead_branches"][fam] + O.cnt_volume(net, e[0], e[i1], r)
                if i2 == -1:
                    vb = O.cnt_volume(net, e[i1], e[-1], r)
                    h["elements"][c] = e[i1:]
                else:
                    vb = O.cnt_volume(net, e[i1], e[i2], r)
                    vols["dead_branches"][fam] = vols["dead_branches"][fam] + O.cnt_volume(net, e[i2], e[-1], r)
                    h["elements"][c] = e[i1:i2 + 1]
                vols["volumes_cnt"][fam] = vols["volumes_cnt"][fam] + vb
            if not h["elements"][c]:
                del cc[i]
    if cg:  # Find_backbone_gnps (:577-660)
        sg = h["structure_gnp"]
        mix = h["cluster_mix_junctions"][j] if h["cluster_mix_junctions"] else []
        for i in range(len(mix) - 1, -1, -1):  # Find_and_remove_gnp_and_mixed_junctions_below_zero_current (:662-790)
            P1, N1, P2, N2, _ = h["junctions_mixed"][mix[i]]
            Ij = abs(volt[lc[P1]] - volt[lg[P2]])
            e = h["elements"][N1]
            if Ij - zero < ZERO or not e or P1 not in e:
                remove_point(P2, sg[N2])
                del mix[i]
                if P1 in e:
                    e.remove(P1)
                    if len(e) < 2:
                        e.clear()
        gj = h["cluster_gnp_junctions"][j] if h["cluster_gnp_junctions"] else []
        for i in range(len(gj) - 1, -1, -1):
            P1, N1, P2, N2, _ = h["junctions_gnp"][gj[i]]
            if abs(volt[lg[P1]] - volt[lg[P2]]) - zero < ZERO:
                remove_point(P1, sg[N1])
                remove_point(P2, sg[N2])
                del gj[i]

        def clear_dead():  # Clear_structure_of_dead_gnps (:792-853)
            to_remove = 0
            for g in cg:
                NT, NB = len(sg[g]), len(h["pts_boundary"][g])
                NJ = NT - NB
                if NT == 0 or (NB == 0 and NJ == 1) or NB == NT:
                    if sg[g]:
                        sg[g].clear()
                        to_remove += 1
                    if NJ == 1:
                        to_remove += 1
                elif len(sg[g]) < 2:
                    raise RuntimeError("Clear_structure_of_dead_gnps: fewer than two points")
            return to_remove

        to_remove = clear_dead()
        while to_remove:
            for i in range(len(gj) - 1, -1, -1):  # Remove_junctions_with_dead_particles_gnps (:994-1040)
                P1, N1, P2, N2, _ = h["junctions_gnp"][gj[i]]
                if not sg[N1] or not sg[N2]:
                    del gj[i]
                    if sg[N1]:
                        remove_point(P1, sg[N1])
                    if sg[N2]:
                        remove_point(P2, sg[N2])
            for i in range(len(mix) - 1, -1, -1):  # Remove_junctions_with_dead_particles_mixed (:1057-1127)
                P1, N1, P2, N2, _ = h["junctions_mixed"][mix[i]]
                if not h["elements"][N1] or not sg[N2]:
                    del mix[i]
                    if sg[N2]:
                        remove_point(P2, sg[N2])
                elif P1 not in h["elements"][N1]:
                    del mix[i]
                    remove_point(P2, sg[N2])
            to_remove = clear_dead()
        if h["clusters_cnt"]:  # Remove_additional_cnts_from_cluster (:855-880)
            for i in range(len(cc) - 1, -1, -1):
                if not h["elements"][cc[i]]:
                    del cc[i]
        for g in cg:  # Calculate_gnp_backbone_volume (:882-948)
            if sg[g]:
                vols["volumes_gnp"][fam] = vols["volumes_gnp"][fam] + h["gnp_volume"][g]
            else:
                vols["dead_gnps"][fam] = vols["dead_gnps"][fam] + h["gnp_volume"][g]
            h["tri"][g] = []
    cj = h["cluster_cnt_junctions"][j] if h["cluster_cnt_junctions"] else []
    for i in range(len(cj) - 1, -1, -1):  # Remove_junctions_with_dead_particles_cnts (:950-992)
        P1, N1, P2, N2, _ = h["junctions_cnt"][cj[i]]
        e1, e2 = h["elements"][N1], h["elements"][N2]
        if not e1 or not e2 or P1 not in e1 or P2 not in e2:
            del cj[i]
    return zero


def boundary_current_gnps(h, p, S, volt, node, gnps_on_face):
    """Currents_through_boundary_gnps (Electrical_analysis.cpp:607-675)."""
    I = 0.0
    lg = S["lmm_gnp"]
    for g in gnps_on_face:
        tri = h["tri"].get(g) or []
        t = h["gnp_t"][g]
        for v1, v2 in tri:
            nA, nB = lg[v1], lg[v2]
            if nA <= 1 or nB <= 1:
                if nA == nB:
                    raise RuntimeError("Currents_through_boundary_gnps: both nodes at the same boundary")
                n1 = nA if nA == node else nB
                n2 = nB if nA == node else nA
                r1 = S["cnt_rad"].get(v1, t / 2)
                r2 = S["cnt_rad"].get(v2, t / 2)
                V = volt[n2] - volt[n1]
                Re = G.gnp_resistance(h["points_gnp"][v1], h["points_gnp"][v2], r1, r2, p["rho_gnp_surf"], p["rho_gnp_t"])
                I = I + V / Re
    return I


def boundary_current_cnts(h, p, S, volt, cnts_on_face):
    """Currents_through_boundary_cnts / Current_of_element_in_boundary (Electrical_analysis.cpp:499-605)
    on the node map of a mixed system."""
    return O.boundary_current(h["net"], p, cnts_on_face, {c: e for c, e in enumerate(h["elements"]) if e}, S["lmm_cnt"], volt)


def electrical(h, p, solver: str = "cg", log=None):
    """Perform_analysis_on_clusters for a mixed network (Electrical_analysis.cpp:10-145):
    returns the resistances along x, y, z and a record per stage."""
    vols = O.new_volumes()
    h["tri"] = {}
    parallel = [[], [], []]
    rec = []
    n_clusters = len(h["clusters_cnt"]) if h["clusters_cnt"] else len(h["clusters_gnp"])
    for j in range(n_clusters):
        fam = h["family"][j]
        S = assemble(h, p, j, fam, 0)
        volt, it = O.solve_cg(S, p["tolerance"]) if solver == "cg" else (O.solve_direct(S), 0)
        r = {"unit": S, "unit_voltages": volt, "unit_tri": {g: list(h["tri"].get(g, [])) for g in (h["clusters_gnp"][j] if h["clusters_gnp"] else [])}}
        r["zero_current"] = backbone(h, j, S, volt, vols)
        r["bb"] = {"clusters_cnt": list(h["clusters_cnt"][j]) if h["clusters_cnt"] else [],
                   "clusters_gnp": list(h["clusters_gnp"][j]) if h["clusters_gnp"] else [],
                   "elements": [list(e) for e in h["elements"]], "structure_gnp": [list(s) for s in h["structure_gnp"]],
                   "cnt_junctions": list(h["cluster_cnt_junctions"][j]) if h["cluster_cnt_junctions"] else [],
                   "gnp_junctions": list(h["cluster_gnp_junctions"][j]) if h["cluster_gnp_junctions"] else [],
                   "mix_junctions": list(h["cluster_mix_junctions"][j]) if h["cluster_mix_junctions"] else []}
        if p["scope"] != 0:
            rec.append(r)
            continue
        if h["clusters_gnp"] and j:  # Clear_triangulations_of_cluster (:183-193)
            for g in h["clusters_gnp"][j - 1]:
                h["tri"][g] = []
        dir_bits = {0: 1, 1: 2, 2: 4, 3: 3, 4: 5, 5: 6, 6: 7}[fam]
        for d in range(3):
            if not (dir_bits >> d & 1) or not p["resistances"][d]:
                continue
            S2 = assemble(h, p, j, d, 1)
            v2, _ = O.solve_cg(S2, p["tolerance"]) if solver == "cg" else (O.solve_direct(S2), 0)
            b1 = [2, 3, 0][d]
            I_c = boundary_current_cnts(h, p, S2, v2, h["boundary_cnt"][b1]) if h["clusters_cnt"] and h["clusters_cnt"][j] else 0.0
            I_g = boundary_current_gnps(h, p, S2, v2, 0, h["boundary_gnp"][b1]) if h["clusters_gnp"] and h["clusters_gnp"][j] else 0.0
            with np.errstate(divide="ignore", invalid="ignore"):
                Rd = p["V"] / (I_c + I_g)
            parallel[d].append(Rd)
            r[f"d{d}"] = S2
            r[f"d{d}_voltages"] = v2
            r[f"d{d}_R"] = Rd
        rec.append(r)
    w = h["net"]["window"]
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
            for x in parallel[d]:
                s = s + 1 / x
            res.append(1 / s)
    return res, rec, vols
