"""GNP part of the contact grid (cicy_gnp_sectioned_domain) and the CNT-GNP
contact pass (cicy_gnp_cnt_contacts) on the device against upstream's region
lists and contacts (golden fixture made by the upstream program) and the CPU
restatement (oracle/gnp_oracle.py) on other seeds and smaller windows."""
import os

import numpy as np
import pytest

from cicy_geom_b200.network import generate_gnps, gnp_sectioned_domain, read_gnps, write_gnp_file
from oracle import gnp_oracle as G

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "gnp_120_s4000000.npz")


def test_gnp_grid_matches_upstream_golden(cuda_ok, tmp_path):
    z = dict(np.load(GOLDEN))
    side, gs, ov_cnt, ov_gnp = float(z["meta"][1]), float(z["meta"][5]), float(z["meta"][6]), float(z["meta"][7])
    g = {"l": z["in_l"], "t": z["in_t"], "theta": z["in_theta"], "phi": z["in_phi"], "center": z["in_center"]}
    write_gnp_file(str(tmp_path), g)
    win = [0.0, 0.0, 0.0, side, side, side, side, side, side]
    n, l, ptr, idx = gnp_sectioned_domain(str(tmp_path), np.arange(len(g["l"])), win, [gs] * 3, ov_cnt, ov_gnp)
    assert list(n) == list(z["ref_sd_n_regions"]) and np.array_equal(l, z["ref_sd_l_regions"])
    assert np.array_equal(ptr, z["ref_sd_ptr"]) and np.array_equal(idx, z["ref_sd_idx"])


def test_gnp_grid_matches_oracle_on_a_window(cuda_ok, tmp_path):
    d = str(tmp_path)
    g = generate_gnps(80, 3.0, 4_000_321)
    write_gnp_file(d, g)
    gs, ov_cnt = 0.07, 0.0118
    ov_gnp = gs / np.sqrt(8.0)
    win = [0.4, 0.5, 0.6, 2.1, 2.2, 2.0, 2.5, 2.7, 2.6]  # a window inside the sample
    inside = np.array([i for i in range(80) if i % 3 != 1], np.int32)  # a subset, in order
    n, l, ptr, idx = gnp_sectioned_domain(d, inside, win, [gs] * 3, ov_cnt, ov_gnp)
    nn, ll = G.region_grid(win, [gs] * 3, ov_cnt, ov_gnp)
    assert list(n) == list(nn) and np.array_equal(l, ll)
    V = read_gnps(d)
    regs = G.fill_sectioned_domain_gnps(win, V["vertices"], V["l"], V["t"], inside, nn, ll, ov_gnp)
    assert len(ptr) == len(regs) + 1
    assert all(list(idx[ptr[k]:ptr[k + 1]]) == regs[k] for k in range(len(regs)))
    assert len(idx) > 1000


def test_gnp_closest_point_matches_upstream_golden(cuda_ok, tmp_path):
    """CNT-GNP distance: closest GNP point to the fixture's query points, bit for bit as upstream."""
    from cicy_geom_b200.network import gnp_closest_points

    z = dict(np.load(GOLDEN))
    g = {"l": z["in_l"], "t": z["in_t"], "theta": z["in_theta"], "phi": z["in_phi"], "center": z["in_center"]}
    write_gnp_file(str(tmp_path), g)
    q = z["in_queries"]
    dist, closest, flag = gnp_closest_points(str(tmp_path), q[:, :3], q[:, 3].astype(np.int32))
    assert np.array_equal(flag, z["ref_query_flag"])
    assert np.array_equal(dist, z["ref_query_dist"])
    assert np.array_equal(closest.ravel(), z["ref_query_point"])


def _hybrid_context_inputs(z, d):
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_gnp_golden as M

    net = {k: v for k, v in M.hybrid_network(d).items() if not k.startswith("boundary")}
    assert M.net_hash(net) == str(z["cnt_sha256"])
    side, gs, ov_cnt, ov_gnp = float(z["meta"][1]), float(z["meta"][5]), float(z["meta"][6]), float(z["meta"][7])
    net["cnts_inside"] = np.arange(len(net["radii"]), dtype=np.int32)
    net["window"] = np.array([0.0, 0.0, 0.0, side, side, side, side, side, side])
    write_gnp_file(d, {"l": z["in_l"], "t": z["in_t"], "theta": z["in_theta"], "phi": z["in_phi"], "center": z["in_center"]})
    p = M.cnt_config().params()
    for a in range(3):
        p.gs_min[a] = gs
    p.gs_overlap_cnt, p.gs_overlap_gnp = ov_cnt, ov_gnp
    return net, p


def test_gnp_cnt_contacts_match_upstream_golden(cuda_ok, tmp_path):
    """The device CNT-GNP contact pass (cicy_gnp_cnt_contacts) gives upstream's
    Find_adjacent_labels contacts on the hybrid fixture: the same (point, GNP)
    pairs with the same contact-point numbers, junction distances and closest
    GNP points, bit for bit; with inside points as errors it fails as upstream's
    default does (the fixture has CNT points inside GNPs)."""
    from cicy_geom_b200 import _abi
    from cicy_geom_b200.device import Context
    from cicy_geom_b200.network import HostNetwork

    z = dict(np.load(GOLDEN))
    d = str(tmp_path)
    net, p = _hybrid_context_inputs(z, d)
    with Context(0) as ctx:
        ctx.upload(HostNetwork.from_arrays(net))
        ctx.contact_grid(p)
        pt, g, dist, q = ctx.gnp_cnt_contacts(d, p)
        order = np.argsort(z["ref_mix_index"])
        assert len(pt) == len(order) > 1000
        assert np.array_equal(pt, z["ref_mix_point"][order]) and np.array_equal(g, z["ref_mix_gnp"][order])
        assert np.array_equal(dist, z["ref_mix_dist"][order])
        assert np.array_equal(q, z["ref_mix_contact_points"].reshape(-1, 3))
        with pytest.raises(_abi.CicyError, match="inside a GNP"):
            ctx.gnp_cnt_contacts(d, p, inside_is_error=True)


def test_gnp_cnt_contacts_match_oracle_on_a_window(cuda_ok, tmp_path):
    """A window of another hybrid sample (a subset of CNTs, region size 0.07 um):
    the device pass against the CPU restatement (oracle/gnp_oracle.py)."""
    from cicy_geom_b200.device import Context
    from cicy_geom_b200.network import HostNetwork, NetworkConfig, generate_cnt_network
    from oracle import cicy_oracle as O

    d = str(tmp_path)
    cfg = NetworkConfig(side=2.5, n_cnts=500, seed=4_000_555, gs_min=0.07)
    net = {k: v for k, v in generate_cnt_network(cfg).arrays().items() if not k.startswith("boundary")}
    net["cnts_inside"] = np.array([i for i in range(cfg.n_cnts) if i % 4 != 3], np.int32)
    net["window"] = np.array([0.3, 0.4, 0.2, 1.9, 1.8, 2.1, 2.2, 2.2, 2.3])
    gn = generate_gnps(70, cfg.side, 4_000_556)
    write_gnp_file(d, gn)
    p = cfg.params()
    p.gs_overlap_gnp = 0.07 / np.sqrt(8.0)
    with Context(0) as ctx:
        ctx.upload(HostNetwork.from_arrays(net))
        ctx.contact_grid(p)
        pt, g, dist, q = ctx.gnp_cnt_contacts(d, p)
    n, l, regs = O.contact_grid(net, {"gs_min": (0.07,) * 3, "gs_overlap_cnt": p.gs_overlap_cnt, "gs_overlap_gnp": p.gs_overlap_gnp})
    V = read_gnps(d)
    sd_gnp = G.fill_sectioned_domain_gnps(net["window"], V["vertices"], V["l"], V["t"], range(70), n, l, p.gs_overlap_gnp)
    out = G.find_adjacent_labels(np.stack([net["x"], net["y"], net["z"]], 1).tolist(), net["flag"], net["radii"], regs, sd_gnp,
                                 V["vertices"].tolist(), V["planes"].tolist(), p.van_der_waals_dist, p.tunneling_dist)
    assert len(out) == len(pt) > 100
    for i in range(len(pt)):
        num, dj, c = out[(int(pt[i]), int(g[i]))]
        assert num == i and dj == dist[i] and tuple(c) == tuple(q[i])


def test_gnp_pair_distance_matches_upstream_golden(cuda_ok, tmp_path):
    """Device GJK / EPA (cicy_gnp_pair_distance) against upstream's distance step on
    the fixture's 2,358 candidate pairs (550 interpenetrating), bit for bit."""
    from cicy_geom_b200.network import gnp_pair_distance

    z = dict(np.load(GOLDEN))
    write_gnp_file(str(tmp_path), {"l": z["in_l"], "t": z["in_t"], "theta": z["in_theta"], "phi": z["in_phi"], "center": z["in_center"]})
    d, N, m, p = gnp_pair_distance(str(tmp_path), z["ref_pair_a"], z["ref_pair_b"], float(z["meta"][3]))
    assert np.array_equal(p, z["ref_pair_penetrating"]) and np.array_equal(d, z["ref_pair_dist"])
    assert np.array_equal(N.ravel(), z["ref_pair_direction"]) and np.array_equal(m.ravel(), z["ref_pair_displacement"])


def test_gnp_contact_pairs_match_oracle(cuda_ok, tmp_path):
    """Device GNP-GNP contact pass (cicy_gnp_contact_pairs) against the CPU
    restatement: the fixture (upstream's region lists) and a window of another
    seed with a subset of the GNPs; same pairs, order, distances and junction
    points, bit for bit."""
    from cicy_geom_b200.network import gnp_contact_pairs

    z = dict(np.load(GOLDEN))
    side, gs, ov_cnt, ov_gnp = float(z["meta"][1]), float(z["meta"][5]), float(z["meta"][6]), float(z["meta"][7])
    vdw, tunnel = float(z["meta"][3]), float(z["meta"][4])
    cases = []
    d1 = os.path.join(str(tmp_path), "a")
    os.makedirs(d1)
    write_gnp_file(d1, {"l": z["in_l"], "t": z["in_t"], "theta": z["in_theta"], "phi": z["in_phi"], "center": z["in_center"]})
    cases.append((d1, np.arange(len(z["in_l"])), [0.0, 0.0, 0.0, side, side, side, side, side, side], gs))
    d2 = os.path.join(str(tmp_path), "b")
    os.makedirs(d2)
    write_gnp_file(d2, generate_gnps(150, 2.5, 4_000_777))
    cases.append((d2, np.array([i for i in range(150) if i % 5 != 2]), [0.2, 0.3, 0.1, 2.0, 1.9, 2.2, 2.2, 2.2, 2.3], 0.07))
    for d, inside, win, g in cases:
        ov = g / np.sqrt(8.0)
        out = gnp_contact_pairs(d, inside, win, [g] * 3, ov_cnt, ov, vdw, tunnel)
        n, l = G.region_grid(win, [g] * 3, ov_cnt, ov)
        V = read_gnps(d)
        sd = G.fill_sectioned_domain_gnps(win, V["vertices"], V["l"], V["t"], inside, n, l, ov)
        ref = G.contact_pairs(sd, V["vertices"].tolist(), vdw, tunnel)
        assert len(out["a"]) == len(ref) > 50
        F = V["planes"].tolist()
        for i, (a, b, dd, N, m, p) in enumerate(ref):
            assert (out["a"][i], out["b"][i], out["penetrating"][i]) == (a, b, int(p)) and out["dist"][i] == dd
            assert tuple(out["direction"][i]) == tuple(N) and tuple(out["displacement"][i]) == tuple(m)
            PA, PB, o = G.pair_junction(V["vertices"][a], F[a], V["vertices"][b], F[b], vdw, win[0:3], win[6:9])
            pts = np.concatenate([out["point_a"][i], out["point_b"][i]])
            assert np.array_equal(pts.view(np.int64), np.array(list(PA) + list(PB)).view(np.int64)) and out["outside"][i] == o


KAT = os.path.join(ROOT, "tests", "golden", "gnp_junction_cases.npz")


@pytest.mark.parametrize("path,side", [(GOLDEN, 2.0), (KAT, 12.0)])
def test_gnp_junction_points_match_upstream_golden(cuda_ok, tmp_path, path, side):
    """Device junction step (cicy_gnp_junction_points) against upstream: points as
    bit patterns (upstream's NaN for parallel edges included), outside codes, and
    a failure where upstream fails."""
    from cicy_geom_b200.network import gnp_junction_points

    z = dict(np.load(path))
    write_gnp_file(str(tmp_path), {"l": z["in_l"], "t": z["in_t"], "theta": z["in_theta"], "phi": z["in_phi"], "center": z["in_center"]})
    jp = z["ref_junc_pair"]
    pa, pb, out, st = gnp_junction_points(str(tmp_path), z["ref_pair_a"][jp], z["ref_pair_b"][jp], 0.00034,
                                          [0.0, 0.0, 0.0, side, side, side, side, side, side])
    ok = z["ref_junc_ok"].astype(bool)
    assert np.array_equal(st == 0, ok)
    pts = np.concatenate([pa, pb], 1)[ok]
    assert np.array_equal(pts.view(np.int64), z["ref_junc_points"].reshape(-1, 6)[ok].view(np.int64))
    assert np.array_equal(out[ok], z["ref_junc_outside"][ok])


LABELS = os.path.join(ROOT, "tests", "golden", "gnp_hybrid_labels.npz")


@pytest.mark.parametrize("path", [GOLDEN, LABELS])
def test_hybrid_labels_match_upstream_golden(cuda_ok, tmp_path, path):
    """The hybrid labelling chain on the device against upstream: CNT labels of
    the hybrid grid (cicy_clusters), GNP labels and point structures from the
    GNP-GNP contact pass with junction points (cicy_gnp_contact_pairs,
    cicy_gnp_labels, cicy_gnp_junction_structures), CNT-GNP contacts
    (cicy_gnp_cnt_contacts), the mixed junctions (cicy_mixed_junctions) and the
    mixed labels (cicy_mixed_labels)."""
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_gnp_golden as M
    from cicy_geom_b200.device import Context
    from cicy_geom_b200.network import HostNetwork, gnp_contact_pairs

    z = dict(np.load(path))
    d = str(tmp_path)
    network, cfg = (M.hybrid_network, M.cnt_config()) if path == GOLDEN else (M.sparse_network, M.sparse_config())
    net = {k: v for k, v in network(d).items() if not k.startswith("boundary")}
    assert M.net_hash(net) == str(z["cnt_sha256"])
    side, gs, ov_cnt, ov_gnp = float(z["meta"][1]), float(z["meta"][5]), float(z["meta"][6]), float(z["meta"][7])
    win = [0.0, 0.0, 0.0, side, side, side, side, side, side]
    net["cnts_inside"] = np.arange(len(net["radii"]), dtype=np.int32)
    net["window"] = np.array(win)
    write_gnp_file(d, {"l": z["in_l"], "t": z["in_t"], "theta": z["in_theta"], "phi": z["in_phi"], "center": z["in_center"]})
    p = cfg.params()
    for a in range(3):
        p.gs_min[a] = gs
    p.gs_overlap_cnt, p.gs_overlap_gnp = ov_cnt, ov_gnp
    with Context(0) as ctx:
        ctx.upload(HostNetwork.from_arrays(net))
        ctx.contact_grid(p)
        ctx.clusters(p)
        lab_cnt, n_cnt = ctx.labels()
        assert np.array_equal(lab_cnt, z["ref_lab_cnt"]) and n_cnt == z["ref_lab_counts"][0]
        tol = 1.5 * float(np.max(z["in_t"]))  # Input_Reader.cpp:1161
        gp = gnp_contact_pairs(d, np.arange(len(z["in_l"])), win, [gs] * 3, ov_cnt, ov_gnp, p.van_der_waals_dist, p.tunneling_dist,
                               n_labels_cnt=n_cnt, tol_gnp2=tol * tol)
        assert np.array_equal(gp["labels_gnp"], z["ref_lab_gnp"]) and gp["n_total_labels"] == z["ref_lab_counts"][1]
        # Add_gnp_junction: point lists and junctions_gnp
        assert np.array_equal(gp["gnp_points"], z["ref_gnpjn_points"].reshape(-1, 3))
        assert np.array_equal(gp["structure_ptr"], z["ref_gnpjn_structure_ptr"]) and np.array_equal(gp["structure_idx"], z["ref_gnpjn_structure_idx"])
        assert np.array_equal(gp["junctions"], z["ref_junctions_gnp"].reshape(-1, 4)) and np.array_equal(gp["junction_dist"], z["ref_junctions_gnp_dist"])
        pt, g, _, _ = ctx.gnp_cnt_contacts(d, p)
        order = np.argsort(z["ref_mix_index"])
        assert np.array_equal(pt, z["ref_mix_point"][order]) and np.array_equal(g, z["ref_mix_gnp"][order])
        # Compress_mixed_contacts: junctions_mixed and the points appended to points_gnp
        mj = ctx.mixed_junctions(len(gp["gnp_points"]), 5)
        ref_j = z["ref_junctions_mixed"].reshape(-1, 4)
        assert np.array_equal(np.stack([mj["cnt_point"], mj["cnt"], mj["gnp_point"], mj["gnp"]], 1), ref_j)
        assert np.array_equal(mj["dist"], z["ref_junctions_mixed_dist"])
        assert np.array_equal(mj["points"], z["ref_mixjn_points"].reshape(-1, 3)[len(gp["gnp_points"]):])
        mc, mg, nm = ctx.mixed_labels(gp["labels_gnp"], gp["n_total_labels"])
        assert np.array_equal(mc, z["ref_mixlab_cnt"]) and np.array_equal(mg, z["ref_mixlab_gnp"]) and nm == z["ref_mixlab_count"][0]
        assert np.array_equal(ctx.labels()[0], mc)
