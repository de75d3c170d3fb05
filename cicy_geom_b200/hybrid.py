"""The whole network-to-conductance path of a mixed CNT/GNP network (GNP_CNT_mix)
through the C ABI, window 0 = the sample, in App_Network_3D's order
(App_Network_3D.cpp:85-180):

  window extraction   CNTs (cicy_extract_window) and GNPs (cicy_gnp_extract_window)
  contact grid        cicy_contact_grid with the GNP overlap (Generate_contact_grid)
  clusters            CNT contacts and labels (cicy_clusters), the GNP-GNP contact pass,
                      labels and point lists (cicy_gnp_contact_pairs, cicy_gnp_labels,
                      cicy_gnp_junction_structures), the CNT-GNP contacts, mixed junctions
                      and labels (cicy_gnp_cnt_contacts, cicy_mixed_junctions,
                      cicy_mixed_labels), then clusters and percolation
                      (cicy_mixed_percolation)
  electrical          cicy_hybrid_electrical

Every stage runs on the device; this module moves upstream's public members from one
entry point to the next (the C ABI's host arrays), as App_Network_3D passes them
between its objects.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import check, lib


def _fill(struct_cls, arrays: dict):
    """A ctypes struct of `struct_cls` from numpy arrays (and ints) named as its fields;
    returns (struct, keep-alive list)."""
    s, keep = struct_cls(), []
    for f, t in struct_cls._fields_:
        if t in (C.c_int32, C.c_int64):
            setattr(s, f, int(arrays[f]))
            continue
        dt = {C.c_int64: np.int64, C.c_int32: np.int32, C.c_double: np.float64}[t._type_]
        a = np.ascontiguousarray(arrays[f], dtype=dt)
        if a.size == 0:
            a = np.zeros(1, dt)
        keep.append(a)
        setattr(s, f, a.ctypes.data_as(t))
    return s, keep


def _merge_csr(ptr, idx, row, val, n):
    """CSR (ptr, idx) over n rows with the pairs (row[k], val[k]) appended to their rows in
    k order, after the row's own entries."""
    rows = np.concatenate([np.repeat(np.arange(n, dtype=np.int64), np.diff(ptr)), row])
    vals = np.concatenate([np.asarray(idx, np.int64), val])
    order = np.argsort(rows, kind="stable")
    return np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int64), vals[order]


def _csr(lists, dt=np.int32):
    ptr = np.concatenate([[0], np.cumsum([len(x) for x in lists])]).astype(np.int64)
    return ptr, np.array([v for x in lists for v in x], dtype=dt)


def mixed_percolation(ctx, st: dict) -> dict:
    """cicy_mixed_percolation on the fields of cicy_mixed_state; returns the lists of
    cicy_mixed_clusters_list as numpy arrays."""
    s, keep = _fill(_abi.MixedState, st)
    h = C.c_void_p()
    ctx._check(lib().cicy_mixed_percolation(ctx.handle, C.byref(s), C.byref(h)), "cicy_mixed_percolation")
    try:
        v = _abi.MixedClustersList()
        check(lib().cicy_mixed_clusters_view(h, C.byref(v)), "cicy_mixed_clusters_view")
        K, NG = int(v.n_percolated), int(st["n_gnps"])

        def arr(ptr, n):
            return np.ctypeslib.as_array(ptr, shape=(max(n, 1),))[:n].copy() if n > 0 else np.zeros(0)

        out = {"n_percolated": K, "family": arr(v.family, K).astype(np.int32)}
        for name, rows in (("clusters_cnt", K), ("clusters_gnp", K), ("cnt_junctions", K), ("gnp_junctions", K), ("mix_junctions", K),
                           ("isolated_cnt", int(v.n_isolated_cnt)), ("isolated_gnp", int(v.n_isolated_gnp)), ("structure_gnp", NG)):
            ptr = arr(getattr(v, name + "_ptr"), rows + 1).astype(np.int64)
            out[name + "_ptr"] = ptr
            out[name + "_idx"] = arr(getattr(v, name + "_idx"), int(ptr[-1]) if len(ptr) else 0)
        pbp = arr(v.pts_boundary_ptr, NG + 1).astype(np.int64)
        out["pts_boundary_ptr"] = pbp
        out["pts_boundary_point"] = arr(v.pts_boundary_point, int(pbp[-1])).astype(np.int64)
        out["pts_boundary_face"] = arr(v.pts_boundary_face, int(pbp[-1])).astype(np.int32)
        return out
    finally:
        lib().cicy_mixed_clusters_free(h)


def hybrid_network_to_conductance(directory: str, cfg, overlap_gnp: float, device: int = 0, rho_gnp_surf: float = 1e-4,
                                  rho_gnp_t: float = 1.0, min_points: int = 5, ctx=None, timings=None):
    """Resistances of the mixed network whose Read_Network files (CNTs, gnp_data.dat,
    sample_geom.csv) are in `directory`; `cfg` a NetworkConfig (sample side, cutoffs,
    electrical parameters).  Returns (cicy_result, context, state) with the context
    holding the systems and the backbone; `timings`, when a dict, gets the host wall
    time of each stage."""
    import time

    from .device import Context
    from .network import gnp_contact_pairs, gnp_extract_window, read_gnps, read_network_files

    t = [time.perf_counter()]
    side = cfg.side
    win = [0.0, 0.0, 0.0, side, side, side, side, side, side]
    net = read_network_files(directory).extract_window(cfg)
    a = net.arrays()
    gw = gnp_extract_window(directory, side)
    gv = read_gnps(directory)
    t.append(time.perf_counter())
    p = cfg.params()
    p.gs_overlap_gnp = overlap_gnp
    ctx = ctx or Context(device)
    ctx.upload(net)
    ctx.contact_grid(p)
    ctx.clusters(p)
    lab_cnt, n_cnt = ctx.labels()
    p1, n1, p2, n2, jd = ctx.junctions()
    ep, ei = ctx.elements(0)
    t.append(time.perf_counter())
    tol = 1.5 * float(np.max(gv["t"]))  # Cutoff_dist::tol_gnp (Input_Reader.cpp:1161)
    gp = gnp_contact_pairs(directory, gw["gnps_inside"], win, list(p.gs_min), p.gs_overlap_cnt, overlap_gnp, p.van_der_waals_dist,
                           p.tunneling_dist, n_labels_cnt=n_cnt, tol_gnp2=tol * tol, device=device,
                           init=(gw["points"], gw["structure_ptr"], gw["structure_idx"]))
    t.append(time.perf_counter())
    ctx.gnp_cnt_contacts(directory, p, gnps_inside=gw["gnps_inside"])
    mj = ctx.mixed_junctions(len(gp["gnp_points"]), min_points)
    lc, lg, nm = ctx.mixed_labels(gp["labels_gnp"], gp["n_total_labels"])
    t.append(time.perf_counter())
    NG = len(gv["t"])
    # points_gnp and structure_gnp after Compress_mixed_contacts appends the mixed points
    # (each GNP's list, then its mixed-junction points in junction order)
    pts = np.concatenate([gp["gnp_points"], mj["points"].reshape(-1, 3)]) if len(mj["points"]) else gp["gnp_points"]
    sp, si = gp["structure_ptr"], gp["structure_idx"]
    st_ptr, st_idx = _merge_csr(sp, si, np.asarray(mj["gnp"], np.int64), np.asarray(mj["gnp_point"], np.int64), NG)
    # elements_cnt: CNT junction points, mixed junction points, end points (Complete_cnt_elements),
    # ascending and without repeats per CNT
    nc = len(ep) - 1
    e_cnt = np.repeat(np.arange(nc, dtype=np.int64), np.diff(ep))
    m_cnt = np.asarray(mj["cnt"], np.int64)
    has = np.zeros(nc, bool)
    has[e_cnt] = True
    has[m_cnt] = True
    ends = np.nonzero(has)[0]
    csp, csi = a["structure_ptr"], a["structure_idx"]
    ec = np.concatenate([e_cnt, m_cnt, ends, ends])
    eq = np.concatenate([np.asarray(ei, np.int64), np.asarray(mj["cnt_point"], np.int64), csi[csp[ends]], csi[csp[ends + 1] - 1]])
    span = int(eq.max(initial=0)) + 1
    key = np.unique(ec * span + eq)
    ep2 = np.concatenate([[0], np.cumsum(np.bincount(key // span, minlength=nc))]).astype(np.int64)
    ei2 = (key % span).astype(np.int64)
    # boundary points of each GNP (GNP::pts_boundary, point order) and the junction-point flags
    pg_, pf_ = np.asarray(gw["point_gnp"], np.int64), np.asarray(gw["point_boundary"], np.int64)
    bsel = np.nonzero(pf_ >= 0)[0]
    border = bsel[np.argsort(pg_[bsel], kind="stable")]
    pb_ptr = np.concatenate([[0], np.cumsum(np.bincount(pg_[border], minlength=NG))]).astype(np.int64)
    pb_pt = border.astype(np.int64)
    pb_face = pf_[border].astype(np.int32)
    bp = np.zeros(len(pts), np.int32)
    bp[: len(gp["boundary_used"])] = gp["boundary_used"]
    J = gp["junctions"]
    mst = {"n_labels": nm, "n_cnts": len(lc), "labels_cnt": lc, "n_cnts_inside": len(a["cnts_inside"]), "cnts_inside": a["cnts_inside"],
           "n_gnps": NG, "labels_gnp": lg, "n_gnps_inside": len(gw["gnps_inside"]), "gnps_inside": gw["gnps_inside"],
           "boundary_cnt_ptr": a["boundary_cnt_ptr"], "boundary_cnt_idx": a["boundary_cnt_idx"],
           "boundary_gnp_ptr": gw["boundary_gnp_ptr"], "boundary_gnp_idx": gw["boundary_gnp_idx"],
           "n_junctions_cnt": len(n1), "jc_n1": n1, "jc_n2": n2, "n_junctions_gnp": len(J), "jg_n1": J[:, 1], "jg_n2": J[:, 3],
           "n_junctions_mixed": len(mj["cnt"]), "jm_n1": mj["cnt"], "jm_n2": mj["gnp"], "n_points_gnp": len(pts),
           "structure_gnp_ptr": st_ptr, "structure_gnp_idx": st_idx, "pts_boundary_ptr": pb_ptr, "pts_boundary_point": pb_pt,
           "pts_boundary_face": pb_face, "bp_flags": bp}
    mc = mixed_percolation(ctx, mst)
    t.append(time.perf_counter())
    vol = np.where(np.isnan(gw["volume"]), gv["l"] * gv["l"] * gv["t"], gw["volume"])
    frame = np.concatenate([gv["l"][:, None], gv["center"], gv["rotation"].reshape(NG, 9), gv["planes"][:, 0, :3]], axis=1)
    hst = {"n_clusters": mc["n_percolated"], "family": mc["family"]}
    for k in ("clusters_cnt", "clusters_gnp", "cnt_junctions", "gnp_junctions", "mix_junctions"):
        hst[k + "_ptr"], hst[k + "_idx"] = mc[k + "_ptr"], mc[k + "_idx"]
    hst.update({"n_junctions_cnt": len(n1), "jc_p1": p1, "jc_n1": n1, "jc_p2": p2, "jc_n2": n2, "jc_dist": jd,
                "n_junctions_gnp": len(J), "jg_p1": J[:, 0], "jg_n1": J[:, 1], "jg_p2": J[:, 2], "jg_n2": J[:, 3], "jg_dist": gp["junction_dist"],
                "n_junctions_mixed": len(mj["cnt"]), "jm_p1": mj["cnt_point"], "jm_n1": mj["cnt"], "jm_p2": mj["gnp_point"], "jm_n2": mj["gnp"],
                "jm_dist": mj["dist"], "elements_ptr": ep2, "elements_idx": ei2, "n_gnps": NG, "n_points_gnp": len(pts),
                "points_gnp": pts.ravel(), "structure_gnp_ptr": mc["structure_gnp_ptr"], "structure_gnp_idx": mc["structure_gnp_idx"],
                "pts_boundary_count": np.diff(mc["pts_boundary_ptr"]).astype(np.int32), "gnp_t": gv["t"], "gnp_volume": vol,
                "gnp_frame": frame.ravel(), "boundary_gnp_ptr": gw["boundary_gnp_ptr"], "boundary_gnp_idx": gw["boundary_gnp_idx"],
                "boundary_gnp_pts_ptr": gw["boundary_pts_ptr"], "boundary_gnp_pts_idx": gw["boundary_pts_idx"]})
    r = ctx.hybrid_electrical(hst, p, rho_gnp_surf, rho_gnp_t)
    t.append(time.perf_counter())
    if timings is not None:
        for k, name in enumerate(["read_and_window", "cnt_grid_and_clusters", "gnp_pairs_labels", "mixed_contacts_labels",
                                  "mixed_percolation", "electrical"]):
            timings[name] = t[k + 1] - t[k]
    return r, ctx, {"mixed": mc, "hybrid": hst}
