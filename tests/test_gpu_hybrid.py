"""The electrical stage of a mixed CNT/GNP network on the device (cicy_hybrid_electrical)
against upstream's own stage-by-stage replay (tests/golden/gnp_hybrid_electrical.npz) on
both hybrid samples: the unit- and real-resistor systems (structure exact; values,
diagonal and right-hand side within 4 ulp: FP64 exp of CUDA vs glibc), the backbone
(CNT clusters and junctions, GNP point lists, GNP and mixed junction lists), the volume
members, and R along x within what the two CG tolerances leave (1e-6)."""
import numpy as np
import pytest
from conftest import assert_ulp
from test_hybrid_electrical import _csr, hybrid_arrays, hybrid_state

from cicy_geom_b200.device import Context
from cicy_geom_b200.network import HostNetwork

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["s", "m"])
def test_hybrid_electrical_on_device_matches_upstream(cuda_ok, tmp_path, tag):
    h, p, z, f = hybrid_state(tag, str(tmp_path))
    from cicy_geom_b200.network import NetworkConfig

    cfg = NetworkConfig(side=2.0, n_cnts=1, seed=0, tolerance=1e-10, vdw=0.00034, tunnel=0.0018)
    prm = cfg.params()
    prm.resistances[0], prm.resistances[1], prm.resistances[2] = 1, 0, 0
    ctx = Context(0)
    ctx.upload(HostNetwork.from_arrays(h["net"]))
    r = ctx.hybrid_electrical(hybrid_arrays(h), prm, 1e-4, 1.0)
    nclu = len(f["flow_family"])
    pref = []
    for j in range(nclu):
        pref.append(f"e_c{j}_u_")
        pref += [f"e_c{j}_d{d}_" for d in range(3) if f"e_c{j}_d{d}_nodes" in z]
    assert r.n_solves == len(pref)
    for i, pfx in enumerate(pref):
        S = ctx.system(i)
        assert (S["nodes"], S["reserved"]) == tuple(z[pfx + "nodes"]), pfx
        assert np.array_equal(S["row_ptr"], z[pfx + "row_ptr"]) and np.array_equal(S["col_ind"], z[pfx + "col_ind"]), pfx
        for k in ("values", "diag", "b", "x0"):
            assert_ulp(S[k], z[pfx + k], 4, pfx + k)
        vr = z[pfx + "voltages"]
        np.testing.assert_allclose(S["voltages"], vr, rtol=0, atol=1e-6 * np.max(np.abs(vr)), err_msg=pfx)
    ptr, idx = ctx.hybrid_structure()
    st = [list(idx[ptr[g]:ptr[g + 1]]) for g in range(len(ptr) - 1)]
    assert st == _csr(z, f"e_c{nclu - 1}_bb_structure_gnp")
    cb = ctx.percolated_clusters(1)
    for j in range(nclu):
        assert list(cb["idx"][cb["ptr"][j]:cb["ptr"][j + 1]]) == z[f"e_c{j}_bb_clusters_cnt"].tolist()
        assert list(cb["junc_idx"][cb["junc_ptr"][j]:cb["junc_ptr"][j + 1]]) == z[f"e_c{j}_bb_cnt_junctions"].tolist()
        g, m = ctx.hybrid_junctions(j)
        assert g.tolist() == z[f"e_c{j}_bb_gnp_junctions"].tolist() and m.tolist() == z[f"e_c{j}_bb_mix_junctions"].tolist()
    bp, bi = ctx.elements(1)
    assert [list(bi[bp[c]:bp[c + 1]]) for c in range(len(bp) - 1)] == _csr(z, f"e_c{nclu - 1}_bb_elements")
    assert ctx.hybrid_volumes().tolist() == z["e_bn_volumes"].tolist()
    np.testing.assert_allclose(np.array(r.resistances), z["flow_resistances"], rtol=1e-6)


@pytest.mark.parametrize("tag", ["s", "m"])
def test_hybrid_chain_on_device_matches_upstream_flow(cuda_ok, tmp_path, tag):
    """The whole GNP_CNT_mix path on the device from the network files
    (cicy_geom_b200.hybrid): window extraction, contact grid, CNT, GNP and mixed
    contacts and labels, mixed percolation (clusters, isolated particles, families,
    junction groups, equal to upstream's) and the electrical stage, whose
    resistances agree with upstream's end-to-end run (tests/golden/gnp_hybrid_flow.npz)."""
    import os
    import sys

    from cicy_geom_b200.hybrid import hybrid_network_to_conductance
    from cicy_geom_b200.network import generate_gnps, write_gnp_file

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "tests", "golden"))
    import make_gnp_golden as M

    fz = dict(np.load(os.path.join(root, "tests", "golden", "gnp_hybrid_flow.npz")))
    f = {k[2:]: v for k, v in fz.items() if k.startswith(tag + "_")}
    d = str(tmp_path)
    if tag == "m":
        M.hybrid_network(d)
        write_gnp_file(d, generate_gnps(M.N, M.SIDE, M.SEED))
        cfg = M.cnt_config()
    else:
        M.sparse_network(d)
        write_gnp_file(d, generate_gnps(M.SPARSE_N, M.SIDE, M.SPARSE_SEED, l_range=(0.3, 0.5)))
        cfg = M.sparse_config()
    cfg.resistances = (1, 0, 0)
    r, ctx, st = hybrid_network_to_conductance(d, cfg, float(M.OVERLAP_GNP))
    mc = st["mixed"]
    assert mc["family"].tolist() == f["flow_family"].tolist()
    for key in ("clusters_cnt", "clusters_gnp", "isolated_cnt", "isolated_gnp"):
        got = [list(mc[key + "_idx"][mc[key + "_ptr"][k]:mc[key + "_ptr"][k + 1]]) for k in range(len(mc[key + "_ptr"]) - 1)]
        assert got == _csr(f, "flow_" + key), key
    for key, fk in (("cnt_junctions", "cluster_cnt_junctions"), ("gnp_junctions", "cluster_gnp_junctions"), ("mix_junctions", "cluster_mix_junctions")):
        got = [list(mc[key + "_idx"][mc[key + "_ptr"][k]:mc[key + "_ptr"][k + 1]]) for k in range(len(mc[key + "_ptr"]) - 1)]
        want = _csr(f, "flow_" + fk)
        assert got == want or (want == [] and all(not g for g in got)), key
    np.testing.assert_allclose(np.array(r.resistances), f["flow_resistances"], rtol=1e-6)


def test_hybrid_configuration_against_upstream_binary(cuda_ok, tmp_path):
    """The hybrid configuration at its full size (4 um cube, 8,000 CNTs, 1,500 GNPs,
    seeded; eight GNPs lie outside Cutoff_Wins::gnps_inside) through the whole device
    path, against upstream's own stages run at test time (oracle/_ref/gnp_dump, flow
    mode, unit-resistor pass to 1e-12 on both sides, real pass to 1e-10): equal
    clusters, isolated particles, families and junction groups, and R_x within what
    the CG tolerances leave."""
    import os
    import subprocess

    from cicy_geom_b200.hybrid import hybrid_network_to_conductance
    from cicy_geom_b200.network import NetworkConfig, generate_cnt_network, generate_gnps, write_gnp_file, write_read_network_files
    from oracle.dumpio import read_dump

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "oracle", "_ref", "gnp_dump")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/gnp_dump not built")
    cfg = NetworkConfig(side=4.0, n_cnts=8000, seed=4_200_001, resistances=(1, 0, 0), tolerance_unit=1e-12)
    d = str(tmp_path)
    write_read_network_files(d, generate_cnt_network(cfg), cfg)
    write_gnp_file(d, generate_gnps(1500, 4.0, 4_200_002))
    ov_gnp = float(cfg.gs_min / np.sqrt(8.0))
    subprocess.run([exe, d, os.path.join(d, "ref.bin"), repr(cfg.vdw), repr(cfg.tunnel), repr(cfg.gs_min), repr(2 * cfg.radius + cfg.tunnel),
                    repr(ov_gnp), "-1", "flow", repr(cfg.step), "electrical_time", "1e-12"], check=True, capture_output=True, timeout=900)
    z = read_dump(os.path.join(d, "ref.bin"))
    assert len(z["flow_gnps_inside"]) < 1500
    ctx = Context(0)
    ctx.set_solver(0, 3)
    r, _, st = hybrid_network_to_conductance(d, cfg, ov_gnp, ctx=ctx)
    mc = st["mixed"]
    assert mc["family"].tolist() == z["flow_family"].tolist()
    for key, fk in (("clusters_cnt", "clusters_cnt"), ("clusters_gnp", "clusters_gnp"), ("isolated_cnt", "isolated_cnt"),
                    ("isolated_gnp", "isolated_gnp"), ("cnt_junctions", "cluster_cnt_junctions"), ("gnp_junctions", "cluster_gnp_junctions"),
                    ("mix_junctions", "cluster_mix_junctions")):
        got = [list(mc[key + "_idx"][mc[key + "_ptr"][k]:mc[key + "_ptr"][k + 1]]) for k in range(len(mc[key + "_ptr"]) - 1)]
        want = _csr(z, "flow_" + fk)
        assert got == want or (want == [] and all(not g for g in got)), key
    np.testing.assert_allclose(np.array(r.resistances), z["flow_resistances"], rtol=1e-6)
