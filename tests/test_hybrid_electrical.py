"""The electrical stage of a mixed CNT/GNP network restated on the CPU
(oracle/hybrid_oracle.py) against upstream's own stage-by-stage replay of
Perform_analysis_on_clusters (tests/golden/gnp_hybrid_electrical.npz) on both
hybrid samples: node maps, systems, triangulations, backbone, real-resistor
systems, resistances and volumes."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ELEC = os.path.join(ROOT, "tests", "golden", "gnp_hybrid_electrical.npz")
GEOM = {"m": os.path.join(ROOT, "tests", "golden", "gnp_120_s4000000.npz"),
        "s": os.path.join(ROOT, "tests", "golden", "gnp_hybrid_labels.npz")}


def _csr(z, name):
    p, i = z[name + "_ptr"], z[name + "_idx"]
    return [[int(v) for v in i[p[k]:p[k + 1]]] for k in range(len(p) - 1)]


def _junctions(z, name):
    q = z[name].reshape(-1, 4)
    d = z[name + "_dist"]
    return [(int(a), int(b), int(c), int(e), float(x)) for (a, b, c, e), x in zip(q, d)]


def hybrid_state(tag, tmp):
    """Upstream's state after Determine_clusters_and_percolation of a hybrid sample, as
    the electrical stage starts from it, plus the window network and the GNP geometry."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_gnp_golden as M

    from cicy_geom_b200.network import read_network_files

    fz = dict(np.load(ELEC))
    z = {k[2:]: v for k, v in fz.items() if k.startswith(tag + "_")}
    fl = dict(np.load(os.path.join(ROOT, "tests", "golden", "gnp_hybrid_flow.npz")))
    f = {k[2:]: v for k, v in fl.items() if k.startswith(tag + "_")}
    if tag == "m":
        M.hybrid_network(tmp)
        cfg = M.cnt_config()
    else:
        M.sparse_network(tmp)
        cfg = M.sparse_config()
    net = dict(read_network_files(tmp).extract_window(cfg).arrays())
    g = dict(np.load(GEOM[tag]))
    N = len(g["in_l"])
    rot, cen = g["ref_gnp_rotation"].reshape(N, 3, 3), g["ref_gnp_center"].reshape(N, 3)
    F, lt = g["ref_gnp_planes"].reshape(N, 6, 4), g["ref_gnp_lt"].reshape(N, 2)
    pb = _csr(z, "e_pts_boundary")
    h = {"net": net, "points_gnp": [tuple(q) for q in z["flow_points_gnp"].reshape(-1, 3).tolist()],
         "structure_gnp": _csr(z, "e_structure_gnp_start"),
         "pts_boundary": [list(zip(v[0::2], v[1::2])) for v in pb],
         "gnp_t": [float(x) for x in z["e_gnp_t"]], "gnp_volume": [float(x) for x in z["e_gnp_volume"]],
         "gnp_geom": [(lt[k, 0], cen[k], rot[k], F[k, 0, :3]) for k in range(N)],
         "boundary_cnt": _csr(f, "flow_boundary_cnt"), "boundary_gnp": _csr(f, "flow_boundary_gnp"),
         "boundary_cnt_pts": _csr(z, "e_boundary_cnt_pts"), "boundary_gnp_pts": _csr(z, "e_boundary_gnp_pts"),
         "clusters_cnt": _csr(f, "flow_clusters_cnt"), "clusters_gnp": _csr(f, "flow_clusters_gnp"),
         "family": [int(x) for x in f["flow_family"]],
         "cluster_cnt_junctions": _csr(f, "flow_cluster_cnt_junctions"), "cluster_gnp_junctions": _csr(f, "flow_cluster_gnp_junctions"),
         "cluster_mix_junctions": _csr(f, "flow_cluster_mix_junctions"),
         "junctions_cnt": _junctions(z, "e_junctions_cnt"), "junctions_gnp": _junctions(z, "e_junctions_gnp"),
         "junctions_mixed": _junctions(z, "e_junctions_mixed"), "elements": _csr(z, "e_elements_start")}
    c1, c2 = cfg.c1_c2()
    p = {"V": 1.0, "rho_cnt": 1e-3, "rho_gnp_surf": 1e-4, "rho_gnp_t": 1.0, "rho_matrix": 1.03e20, "junction": "exponential",
         "junction_resistance": 1e7, "C1": c1, "C2": c2, "tolerance": 1e-10, "resistances": (1, 0, 0), "scope": 0}
    return h, p, z, f


def hybrid_arrays(h):
    """The oracle's state `h` as the arrays of cicy_hybrid_state (Context.hybrid_electrical)."""
    def csr(lists, dt=np.int32):
        ptr = np.concatenate([[0], np.cumsum([len(x) for x in lists])]).astype(np.int64)
        idx = np.array([v for x in lists for v in x], dtype=dt)
        return ptr, idx

    out = {"n_clusters": len(h["family"]), "family": np.array(h["family"], np.int32)}
    for key, name in (("clusters_cnt", "clusters_cnt"), ("clusters_gnp", "clusters_gnp"), ("cluster_cnt_junctions", "cnt_junctions"),
                      ("cluster_gnp_junctions", "gnp_junctions"), ("cluster_mix_junctions", "mix_junctions")):
        out[name + "_ptr"], out[name + "_idx"] = csr(h[key])
    for key, pre in (("junctions_cnt", "jc"), ("junctions_gnp", "jg"), ("junctions_mixed", "jm")):
        j = h[key]
        out[f"n_{key}"] = len(j)
        out[pre + "_p1"] = np.array([x[0] for x in j], np.int64)
        out[pre + "_n1"] = np.array([x[1] for x in j], np.int32)
        out[pre + "_p2"] = np.array([x[2] for x in j], np.int64)
        out[pre + "_n2"] = np.array([x[3] for x in j], np.int32)
        out[pre + "_dist"] = np.array([x[4] for x in j], np.float64)
    out["elements_ptr"], out["elements_idx"] = csr(h["elements"], np.int64)
    out["n_gnps"] = len(h["gnp_t"])
    out["n_points_gnp"] = len(h["points_gnp"])
    out["points_gnp"] = np.array(h["points_gnp"], np.float64).ravel()
    out["structure_gnp_ptr"], out["structure_gnp_idx"] = csr(h["structure_gnp"], np.int64)
    out["pts_boundary_count"] = np.array([len(x) for x in h["pts_boundary"]], np.int32)
    out["gnp_t"] = np.array(h["gnp_t"])
    out["gnp_volume"] = np.array(h["gnp_volume"])
    out["gnp_frame"] = np.array([np.concatenate([[l], np.ravel(c), np.ravel(r), np.ravel(n)]) for l, c, r, n in h["gnp_geom"]]).ravel()
    out["boundary_gnp_ptr"], out["boundary_gnp_idx"] = csr(h["boundary_gnp"])
    out["boundary_gnp_pts_ptr"], out["boundary_gnp_pts_idx"] = csr(h["boundary_gnp_pts"], np.int64)
    return out


def _check_system(S, z, pfx):
    nodes, res = z[pfx + "nodes"]
    assert (S["nodes"], S["reserved"]) == (nodes, res), pfx
    assert sorted(S["lmm_cnt"].items()) == list(zip(z[pfx + "lmm_cnt_pts"].tolist(), z[pfx + "lmm_cnt_nodes"].tolist())), pfx
    assert sorted(S["lmm_gnp"].items()) == list(zip(z[pfx + "lmm_gnp_pts"].tolist(), z[pfx + "lmm_gnp_nodes"].tolist())), pfx
    assert sorted(S["cnt_rad"].items()) == list(zip(z[pfx + "cnt_rad_pts"].tolist(), z[pfx + "cnt_rad"].tolist())), pfx
    assert np.array_equal(S["row_ptr"], z[pfx + "row_ptr"]) and np.array_equal(S["col_ind"], z[pfx + "col_ind"]), pfx
    for k in ("values", "diag", "b", "x0"):
        assert np.array_equal(S[k], z[pfx + {"diag": "diag"}.get(k, k)]), pfx + k


@pytest.mark.parametrize("tag", ["s", "m"])
def test_hybrid_electrical_stage_matches_upstream(tmp_path, tag):
    from oracle import hybrid_oracle as H

    h, p, z, f = hybrid_state(tag, str(tmp_path))
    res, rec, vols = H.electrical(h, p)
    assert len(rec) == len(f["flow_family"]) >= 1
    for j, r in enumerate(rec):
        pj = f"e_c{j}_"
        _check_system(r["unit"], z, pj + "u_")
        tri = _csr(z, pj + "u_tri")
        assert [[v for e in r["unit_tri"][g] for v in e] for g in h["clusters_gnp"][j]] == tri
        vr = z[pj + "u_voltages"]
        np.testing.assert_allclose(r["unit_voltages"], vr, rtol=0, atol=1e-6 * np.max(np.abs(vr)))
        np.testing.assert_allclose(r["zero_current"], z[pj + "zero_current"][0], rtol=1e-5)
        bb = r["bb"]
        assert bb["elements"] == _csr(z, pj + "bb_elements")
        assert bb["structure_gnp"] == _csr(z, pj + "bb_structure_gnp")
        for k in ("clusters_cnt", "clusters_gnp", "cnt_junctions", "gnp_junctions", "mix_junctions"):
            assert bb[k] == z[pj + "bb_" + k].tolist(), k
        for d in range(3):
            if f"d{d}" in r:
                _check_system(r[f"d{d}"], z, pj + f"d{d}_")
                np.testing.assert_allclose(r[f"d{d}_R"], z[pj + f"d{d}_R"][0], rtol=1e-6)
    np.testing.assert_allclose(res, z["flow_resistances"], rtol=1e-6)
    v = z["e_bn_volumes"]
    assert vols["volumes_cnt"] + vols["volumes_gnp"] + vols["dead_branches"] + vols["dead_gnps"] == v.tolist()
