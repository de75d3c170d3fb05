"""Device path (C ABI) against the upstream program's outputs and the CPU oracle.

Integer and geometry outputs must be bit-exact: sectioned domain, point
contacts (incl. FP64 junction distances), labels, junctions, elements,
percolated clusters, families, backbone.  DEA matrices: structure exact,
values within 4 ulp (junction conductances use exp()).  Voltages: within the
CG tolerance of upstream's iterate; with a tight tolerance, within 1e-9
(relative, max-norm over grounded nodes) of an FP64 direct solve.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest
from conftest import ALL, assert_ulp, ROOT, arr_sha, csr_list, golden_network, golden_systems, net_sha

from cicy_geom_b200.device import Context
from oracle import cicy_oracle as O

pytestmark = pytest.mark.gpu


def run_device(net, cfg, tol=None):
    if tol is not None:
        cfg.tolerance = tol
    p = cfg.params()
    ctx = Context(0)
    ctx.upload(net)
    ctx.contact_grid(p)
    ctx.clusters(p)
    r = ctx.electrical_analysis(p)
    return ctx, r


@pytest.fixture(scope="module")
def device_runs(cuda_ok):
    cache = {}

    def get(name):
        if name not in cache:
            cfg, net, z = golden_network(name)
            assert net_sha(net.arrays()) == str(z["net_sha256"])
            ctx, r = run_device(net, cfg)
            cache[name] = (cfg, net, z, ctx, r)
        return cache[name]

    return get


@pytest.mark.parametrize("name", ALL)
def test_sectioned_domain_and_point_contacts_bit_exact(device_runs, name):
    cfg, net, z, ctx, r = device_runs(name)
    ptr, idx = ctx.sectioned_domain()
    assert arr_sha(ptr, idx) == str(z["sd_sha256"])
    if "sd_idx" in z:
        assert np.array_equal(ptr, z["sd_ptr"]) and np.array_equal(idx, z["sd_idx"])
    pa, cb, pb, d = ctx.point_contacts()
    assert np.array_equal(pa, z["pc_Pa"]) and np.array_equal(cb, z["pc_CNTb"]) and np.array_equal(pb, z["pc_Pb"])
    assert np.array_equal(d, z["pc_dist"])  # FP64 bit-exact


@pytest.mark.parametrize("name", ALL)
def test_labels_junctions_elements_clusters_bit_exact(device_runs, name):
    cfg, net, z, ctx, r = device_runs(name)
    lab, nl = ctx.labels()
    assert np.array_equal(lab, z["labels_cnt"]) and nl == int(z["n_labels"][0])
    p1, n1, p2, n2, d = ctx.junctions()
    for a, k in ((p1, "junc_P1"), (n1, "junc_N1"), (p2, "junc_P2"), (n2, "junc_N2"), (d, "junc_dist")):
        assert np.array_equal(a, z[k]), k
    ep, ei = ctx.elements(0)
    assert np.array_equal(ep, z["elements_ptr"]) and np.array_equal(ei, z["elements_idx"])
    cl = ctx.percolated_clusters(0)
    assert np.array_equal(cl["family"], z["family"])
    assert np.array_equal(cl["ptr"], z["clusters_ptr"]) and np.array_equal(cl["idx"], z["clusters_idx"])
    assert np.array_equal(cl["junc_ptr"], z["cluster_junc_ptr"]) and np.array_equal(cl["junc_idx"], z["cluster_junc_idx"])


@pytest.mark.parametrize("name", ALL)
def test_dea_systems_backbone_resistance(device_runs, name):
    cfg, net, z, ctx, r = device_runs(name)
    systems = golden_systems(z)
    assert r.n_solves == len(systems)
    for i, (pfx, kind, k) in enumerate(systems):
        S = ctx.system(i)
        assert (S["nodes"], S["reserved"]) == tuple(z[pfx + "nodes"])
        assert np.array_equal(S["row_ptr"], z[pfx + "row_ptr"]) and np.array_equal(S["col_ind"], z[pfx + "col_ind"])
        for f in ("values", "diag", "b", "x0"):
            assert_ulp(S[f], z[pfx + f], 4, pfx + f)
        vr = z[pfx + "voltages"]
        scale = np.nanmax(np.abs(vr)) if np.isfinite(vr).any() else 1.0
        np.testing.assert_allclose(S["voltages"], vr, rtol=0, atol=1e-5 * scale, equal_nan=True)
    if len(z["family"]):
        bp, bi = ctx.elements(1)
        last = len(z["family"]) - 1
        assert np.array_equal(bp, z[f"c{last}_bb_elements_ptr"]) and np.array_equal(bi, z[f"c{last}_bb_elements_idx"])
        cb = ctx.percolated_clusters(1)
        for k in range(len(z["family"])):
            assert list(cb["idx"][cb["ptr"][k]:cb["ptr"][k + 1]]) == list(z[f"c{k}_bb_cluster"])
            assert list(cb["junc_idx"][cb["junc_ptr"][k]:cb["junc_ptr"][k + 1]]) == list(z[f"c{k}_bb_junc"])
    vol = ctx.volumes()
    assert list(vol["volumes_cnt"]) == list(z["bn_volumes_cnt"]) and list(vol["dead_branches"]) == list(z["bn_dead_branches"])
    tv = 0.0
    for v in z["bn_volumes_cnt"]:
        tv = tv + float(v) + 0.0
    assert list(vol["total_volumes"]) == [0.0 + float(v) + 0.0 for v in z["bn_volumes_cnt"]]
    assert list(vol["fractions"]) == [float(np.float64(v) / np.float64(tv)) for v in z["bn_volumes_cnt"]]
    # upstream's own CG iterate (tolerance 1e-10) is up to 2.9e-7 off the exact R on these
    # fixtures (c1p_800_s5, against an FP64 direct solve), and so is the device's
    np.testing.assert_allclose(np.array(r.resistances), z["resistances"], rtol=1e-6, equal_nan=True)


@pytest.mark.parametrize("name", ["c1p_1200_s1", "c1p_800_s2", "c1p_800_s5", "kat_series", "kat_three_chain"])
def test_voltages_match_fp64_direct_solve(cuda_ok, name):
    """Solved tight, the device voltages agree with an FP64 direct solve of the same system within 1e-9."""
    cfg, net, z = golden_network(name)
    ctx, r = run_device(net, cfg, tol=1e-14)
    for i in range(r.n_solves):
        S = ctx.system(i)
        if len(S["diag"]) == 0:
            continue
        vd = O.solve_direct({**S, "vef": S["voltages"][: S["reserved"]]})
        m = np.concatenate([np.ones(S["reserved"], bool), O.grounded_mask(S)])
        rel = np.max(np.abs(S["voltages"][m] - vd[m])) / np.max(np.abs(vd[m]))
        assert rel < 1e-9, (i, rel)
    # effective resistance against the oracle driven by the direct solver
    a = net.arrays()
    ref = O.network_to_conductance(a, O.params_from_config(cfg), solver="direct")
    np.testing.assert_allclose(np.array(r.resistances), ref["resistances"], rtol=1e-9)


def test_kat_series_closed_form_on_device(cuda_ok):
    import math

    cfg, net, z = golden_network("kat_series")
    ctx, r = run_device(net, cfg, tol=1e-14)
    p1, n1, p2, n2, d = ctx.junctions()
    a = net.arrays()
    x, sp = a["x"], a["structure_ptr"]
    LA = sum(abs(x[i + 1] - x[i]) for i in range(sp[0], p1[0]))
    LB = sum(abs(x[i + 1] - x[i]) for i in range(p2[0], sp[2] - 1))
    c1, c2 = cfg.c1_c2()
    R = 1e-3 * (LA + LB) / (math.pi * 0.005 ** 2) + c1 * d[0] * math.exp(c2 * d[0]) / 0.01 ** 2
    assert abs(r.resistances[0] - R) / R < 1e-12


@pytest.mark.parametrize("seed", [101, 202])
def test_random_seeds_against_oracle(cuda_ok, seed):
    """Fresh seeds (no fixture): device vs the CPU oracle restatement."""
    from cicy_geom_b200.network import NetworkConfig, generate_cnt_network

    cfg = NetworkConfig(side=1.6, n_cnts=700, seed=seed)
    net = generate_cnt_network(cfg).extract_window(cfg)
    ctx, r = run_device(net, cfg)
    ref = O.network_to_conductance(net.arrays(), O.params_from_config(cfg))
    lab, nl = ctx.labels()
    assert np.array_equal(lab, ref["labels"]) and nl == ref["n_labels"]
    p1, n1, p2, n2, d = ctx.junctions()
    assert [tuple(t) for t in zip(p1, n1, p2, n2)] == [t[:4] for t in ref["junctions"]]
    assert np.array_equal(d, [t[4] for t in ref["junctions"]])
    cl = ctx.percolated_clusters(0)
    assert list(cl["family"]) == ref["families"]
    np.testing.assert_allclose(np.array(r.resistances), ref["resistances"], rtol=1e-6)


def test_medium_network_against_upstream_binary(cuda_ok):
    """3.2 um / 8,000-CNT network (~0.8M points) run through the upstream program at test time."""
    from cicy_geom_b200.network import NetworkConfig, generate_cnt_network, write_read_network_files
    from oracle.dumpio import read_dump

    refbin = os.path.join(ROOT, "oracle", "_ref", "ref_dump")
    if not os.path.exists(refbin):
        pytest.skip("oracle/_ref/ref_dump not built")
    cfg = NetworkConfig(side=3.2, n_cnts=8000, seed=1)
    raw = generate_cnt_network(cfg)
    net = raw.extract_window(cfg)
    ctx, r = run_device(net, cfg)
    with tempfile.TemporaryDirectory(prefix="cicy_ref_") as dd:
        write_read_network_files(dd, raw, cfg)
        subprocess.run([refbin, "dump", dd, os.path.join(dd, "d.bin")], check=True, capture_output=True, timeout=600)
        D = read_dump(os.path.join(dd, "d.bin"))
    ptr, idx = ctx.sectioned_domain()
    assert np.array_equal(ptr, D["sd_ptr"]) and np.array_equal(idx, D["sd_idx"])
    pa, cb, pb, d = ctx.point_contacts()
    assert np.array_equal(pa, D["pc_Pa"]) and np.array_equal(pb, D["pc_Pb"]) and np.array_equal(d, D["pc_dist"])
    lab, nl = ctx.labels()
    assert np.array_equal(lab, D["labels_cnt"])
    p1, n1, p2, n2, jd = ctx.junctions()
    assert np.array_equal(p1, D["junc_P1"]) and np.array_equal(p2, D["junc_P2"]) and np.array_equal(jd, D["junc_dist"])
    cl = ctx.percolated_clusters(0)
    assert np.array_equal(cl["idx"], D["clusters_idx"]) and np.array_equal(cl["family"], D["family"])
    if len(D["family"]):
        bp, bi = ctx.elements(1)
        last = len(D["family"]) - 1
        assert np.array_equal(bi, D[f"c{last}_bb_elements_idx"])
    np.testing.assert_allclose(np.array(r.resistances), D["resistances"], rtol=1e-6)


def test_headline_network_against_upstream_binary(cuda_ok):
    """The benchmark's 6 um / 25,000-CNT network (seed 2,000,000, ~2.5 M points) with the
    benchmark's tolerances (unit-resistor pass 1e-12, real-resistor pass 1e-8), through the
    upstream program at test time (oracle/_ref/ref_dump with the unit-pass tolerance).

    Bit-exact: sectioned domain, point contacts with distances, labels, junctions,
    elements, percolated clusters, families, cluster junctions, the backbone (elements,
    clusters, junctions) and the structure of both DEA systems; matrix values, diagonal
    and right-hand side within 4 ulp (FP64 exp of CUDA vs glibc).  Voltages and R:
    both sides stop at |r| <= 1e-8 |r0| (upstream Jacobi-PCG, here the default
    multigrid PCG), so they agree within that solve tolerance, not bit for bit."""
    from cicy_geom_b200.network import NetworkConfig, generate_cnt_network, write_read_network_files
    from oracle.dumpio import read_dump

    refbin = os.path.join(ROOT, "oracle", "_ref", "ref_dump")
    if not os.path.exists(refbin):
        pytest.skip("oracle/_ref/ref_dump not built")
    tol_unit = 1e-12
    cfg = NetworkConfig(side=6.0, n_cnts=25000, seed=2_000_000, tolerance=1e-8, tolerance_unit=tol_unit)
    raw = generate_cnt_network(cfg)
    net = raw.extract_window(cfg)
    ctx, r = run_device(net, cfg)
    with tempfile.TemporaryDirectory(prefix="cicy_ref_") as dd:
        write_read_network_files(dd, raw, cfg)
        subprocess.run([refbin, "dump", dd, os.path.join(dd, "d.bin"), repr(tol_unit)], check=True, capture_output=True, timeout=900)
        D = read_dump(os.path.join(dd, "d.bin"))
    ptr, idx = ctx.sectioned_domain()
    assert np.array_equal(ptr, D["sd_ptr"]) and np.array_equal(idx, D["sd_idx"])
    pa, cb, pb, d = ctx.point_contacts()
    assert np.array_equal(pa, D["pc_Pa"]) and np.array_equal(cb, D["pc_CNTb"]) and np.array_equal(pb, D["pc_Pb"])
    assert np.array_equal(d, D["pc_dist"])
    lab, nl = ctx.labels()
    assert np.array_equal(lab, D["labels_cnt"]) and nl == int(D["n_labels"][0])
    p1, n1, p2, n2, jd = ctx.junctions()
    for a, k in ((p1, "junc_P1"), (n1, "junc_N1"), (p2, "junc_P2"), (n2, "junc_N2"), (jd, "junc_dist")):
        assert np.array_equal(a, D[k]), k
    ep, ei = ctx.elements(0)
    assert np.array_equal(ep, D["elements_ptr"]) and np.array_equal(ei, D["elements_idx"])
    cl = ctx.percolated_clusters(0)
    assert np.array_equal(cl["family"], D["family"])
    assert np.array_equal(cl["ptr"], D["clusters_ptr"]) and np.array_equal(cl["idx"], D["clusters_idx"])
    assert np.array_equal(cl["junc_ptr"], D["cluster_junc_ptr"]) and np.array_equal(cl["junc_idx"], D["cluster_junc_idx"])
    assert len(D["family"]) >= 1
    systems = golden_systems(D)
    assert r.n_solves == len(systems)
    for i, (pfx, kind, k) in enumerate(systems):
        S = ctx.system(i)
        assert (S["nodes"], S["reserved"]) == tuple(D[pfx + "nodes"])
        assert np.array_equal(S["row_ptr"], D[pfx + "row_ptr"]) and np.array_equal(S["col_ind"], D[pfx + "col_ind"])
        for f in ("values", "diag", "b", "x0"):
            assert_ulp(S[f], D[pfx + f], 4, pfx + f)
    bp, bi = ctx.elements(1)
    last = len(D["family"]) - 1
    assert np.array_equal(bp, D[f"c{last}_bb_elements_ptr"]) and np.array_equal(bi, D[f"c{last}_bb_elements_idx"])
    cbb = ctx.percolated_clusters(1)
    for k in range(len(D["family"])):
        assert list(cbb["idx"][cbb["ptr"][k]:cbb["ptr"][k + 1]]) == list(D[f"c{k}_bb_cluster"])
        assert list(cbb["junc_idx"][cbb["junc_ptr"][k]:cbb["junc_ptr"][k + 1]]) == list(D[f"c{k}_bb_junc"])
    vol = ctx.volumes()
    assert list(vol["volumes_cnt"]) == list(D["bn_volumes_cnt"]) and list(vol["dead_branches"]) == list(D["bn_dead_branches"])
    # both solves at |r| <= 1e-8 |r0|: R agrees within what that residual leaves
    rel = abs(r.resistances[0] - D["resistances"][0]) / abs(D["resistances"][0])
    assert rel < 1e-6, rel
