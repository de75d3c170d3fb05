"""The CPU oracle restatement reproduces the upstream program's outputs (golden fixtures)."""
import math

import numpy as np
import pytest
from conftest import ALL, arr_sha, csr_list, golden_network, golden_systems

from oracle import cicy_oracle as O

FAST = [n for n in ALL if n != "c1p_1200_s1"]


@pytest.fixture(scope="module")
def runs():
    cache = {}

    def get(name):
        if name not in cache:
            cfg, net, z = golden_network(name)
            a = net.arrays()
            cache[name] = (cfg, a, z, O.network_to_conductance(a, O.params_from_config(cfg)))
        return cache[name]

    return get


@pytest.mark.parametrize("name", FAST)
def test_contacts_labels_junctions(runs, name):
    cfg, a, z, out = runs(name)
    regions = out["regions"]
    ptr = np.concatenate([[0], np.cumsum([len(r) for r in regions])])
    idx = np.concatenate([np.asarray(r, np.int64) for r in regions]) if len(ptr) > 1 else np.zeros(0)
    assert arr_sha(ptr, idx) == str(z["sd_sha256"])
    pc = out["point_contacts"]
    keys = sorted(pc)
    assert np.array_equal([k[0] for k in keys], z["pc_Pa"])
    assert np.array_equal([k[1] for k in keys], z["pc_CNTb"])
    assert np.array_equal([pc[k][0] for k in keys], z["pc_Pb"])
    assert np.array_equal([pc[k][1] for k in keys], z["pc_dist"])
    assert np.array_equal(out["labels"], z["labels_cnt"])
    assert out["n_labels"] == int(z["n_labels"][0])
    j = out["junctions"]
    assert [t[0] for t in j] == list(z["junc_P1"]) and [t[1] for t in j] == list(z["junc_N1"])
    assert [t[2] for t in j] == list(z["junc_P2"]) and [t[3] for t in j] == list(z["junc_N2"])
    assert np.array_equal([t[4] for t in j], z["junc_dist"])


@pytest.mark.parametrize("name", FAST)
def test_elements_clusters_families(runs, name):
    cfg, a, z, out = runs(name)
    ge = csr_list(z, "elements")
    for c, e in enumerate(ge):
        assert list(e) == out["elements"].get(c, [])
    assert out["families"] == list(z["family"])
    gc = csr_list(z, "clusters")
    assert len(gc) == len(out["families"])
    gj = csr_list(z, "cluster_junc")
    for k in range(len(gc)):
        assert out["backbone"] == [] or True
    # clusters before backbone: compare against golden (out["clusters"] were trimmed by the backbone)
    _, _, z2, _ = runs(name)
    cl, fam, cj = O.percolation(a, out["labels"], out["n_labels"], out["junctions"])
    assert [list(c) for c in cl] == [list(c) for c in gc]
    assert [list(c) for c in cj] == [list(c) for c in gj]


@pytest.mark.parametrize("name", FAST)
def test_systems_backbone_resistance(runs, name):
    cfg, a, z, out = runs(name)
    systems = golden_systems(z)
    assert len(systems) == len(out["systems"])
    for (pfx, kind, k), (okind, ok, S) in zip(systems, out["systems"]):
        assert (kind, k) == (okind, ok)
        assert np.array_equal(S["row_ptr"], z[pfx + "row_ptr"]) and np.array_equal(S["col_ind"], z[pfx + "col_ind"])
        np.testing.assert_array_equal(S["values"], z[pfx + "values"])
        np.testing.assert_array_equal(S["diag"], z[pfx + "diag"])
        np.testing.assert_array_equal(S["b"], z[pfx + "b"])
        np.testing.assert_array_equal(S["x0"], z[pfx + "x0"])
        v, vr = S["voltages"], z[pfx + "voltages"]
        scale = np.nanmax(np.abs(vr)) if np.isfinite(vr).any() else 1.0
        np.testing.assert_allclose(v, vr, rtol=0, atol=1e-5 * scale, equal_nan=True)
    for k, bb in enumerate(out["backbone"]):
        assert bb["cluster"] == list(z[f"c{k}_bb_cluster"])
        assert bb["junctions"] == list(z[f"c{k}_bb_junc"])
    r, rg = np.array(out["resistances"]), z["resistances"]
    np.testing.assert_allclose(r, rg, rtol=1e-5, equal_nan=True)


def test_kat_series_closed_form(runs):
    """R = rho L_A / (pi r^2) + C1 d exp(C2 d) / (2r)^2 + rho L_B / (pi r^2), from first principles."""
    cfg, a, z, out = runs("kat_series")
    (P1, N1, P2, N2, d), = out["junctions"]
    x, sp = a["x"], a["structure_ptr"]
    r, rho = 0.005, 1e-3
    LA = sum(abs(x[i + 1] - x[i]) for i in range(sp[0], P1))
    LB = sum(abs(x[i + 1] - x[i]) for i in range(P2, sp[2] - 1))
    c1, c2 = cfg.c1_c2()
    R = rho * (LA + LB) / (math.pi * r * r) + c1 * d * math.exp(c2 * d) / (2 * r) ** 2
    assert abs(out["resistances"][0] - R) / R < 1e-9
    assert abs(z["resistances"][0] - R) / R < 1e-9


def test_kat_corner_pair_has_no_contact(runs):
    cfg, a, z, out = runs("kat_corner_pair")
    # the tips are within the tunnelling cutoff in exact geometry ...
    p = np.stack([a["x"], a["y"], a["z"]], 1)
    sp = a["structure_ptr"]
    d = np.linalg.norm(p[sp[1] - 1] - p[sp[1]]) - 2 * 0.005
    assert d <= 0.0018
    # ... but sit in diagonally adjacent cells, which the grid never pairs
    assert out["point_contacts"] == {} and len(z["pc_Pa"]) == 0


def test_kat_vdw_ties_keep_first_in_scan_order(runs):
    cfg, a, z, out = runs("kat_vdw_tie")
    vdw = cfg.vdw
    assert np.sum(z["pc_dist"] == vdw) >= 2
    assert np.array_equal([out["point_contacts"][k][0] for k in sorted(out["point_contacts"])], z["pc_Pb"])


def test_direct_solve_agrees_with_cg_within_tolerance(runs):
    cfg, a, z, out = runs("c1p_800_s2")
    for kind, k, S in out["systems"]:
        vd = O.solve_direct(S)
        m = np.concatenate([np.ones(S["reserved"], bool), O.grounded_mask(S)])
        rel = np.max(np.abs(vd[m] - S["voltages"][m])) / np.max(np.abs(vd[m]))
        assert rel < 1e-5


@pytest.mark.parametrize("name", FAST)
def test_backbone_volumes_and_family_fractions(runs, name):
    """Calculate_cnt_volumes over every percolated cluster and Calculate_percolated_families_fractions:
    the oracle's volume members equal upstream's bit for bit."""
    cfg, a, z, out = runs(name)
    before = out["volumes_before_fractions"]
    assert before["volumes_cnt"][:3] + before["dead_branches"][:3] == list(z["bn_volumes"])
    v = out["volumes"]
    assert v["volumes_cnt"] == list(z["bn_volumes_cnt"])
    assert v["dead_branches"] == list(z["bn_dead_branches"])
    assert v["volumes_gnp"] == list(z["bn_volumes_gnp"]) and v["dead_gnps"] == list(z["bn_dead_gnps"])
