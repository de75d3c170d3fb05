"""Network construction on the device through the C ABI: the window trim
(cicy_ctx_extract_window) against the host restatement cicy_extract_window
(bit-exact with upstream's Shells + Cutoff_Wins), the seeded generator
(cicy_ctx_generate_cnt_network) against the host generator, and the whole
device-built network through the hot path against the host-built one."""
import time
from dataclasses import replace

import numpy as np
import pytest

from cicy_geom_b200.device import Context
from cicy_geom_b200.network import NetworkConfig, generate_cnt_network

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def assert_same_network(got, ref, exact_xyz=True):
    for k in ("x", "y", "z"):
        if exact_xyz:
            assert np.array_equal(bits(got[k]), bits(ref[k])), k
        else:
            np.testing.assert_allclose(got[k], ref[k], rtol=0, atol=1e-9)
    assert np.array_equal(got["flag"], ref["flag"])
    assert np.array_equal(got["structure_ptr"], ref["structure_ptr"])
    assert np.array_equal(got["structure_idx"], ref["structure_idx"])
    assert np.array_equal(bits(got["radii"]), bits(ref["radii"]))
    assert np.array_equal(got["cnts_inside"], ref["cnts_inside"])
    for k in ("boundary_cnt_ptr", "boundary_cnt_idx", "boundary_pts_ptr", "boundary_pts_idx"):
        assert np.array_equal(got[k].astype(np.int64), ref[k].astype(np.int64)), k
    assert np.array_equal(bits(got["window"]), bits(ref["window"]))


@pytest.mark.parametrize("side,n,seed,turn", [(0.6, 250, 13, 40.0), (1.6, 700, 7, 10.0), (6.0, 25000, 2000000, 10.0)])
def test_device_window_trim_equals_host_restatement(cuda_ok, side, n, seed, turn):
    cfg = replace(NetworkConfig(side=side, n_cnts=n, seed=seed), max_turn_deg=turn)
    raw = generate_cnt_network(cfg)
    ref = raw.extract_window(cfg).arrays()
    with Context(0) as ctx:
        ctx.upload(raw)
        ctx.extract_window(cfg)
        got = ctx.network()
    assert_same_network(got, ref)


def test_device_generator_matches_host_generator(cuda_ok):
    cfg = NetworkConfig(side=2.0, n_cnts=1500, seed=5)
    ref = generate_cnt_network(cfg).arrays()
    with Context(0) as ctx:
        ctx.generate_network(cfg, trim=False)
        got = ctx.network()
    # counts, structure and flags from the same Philox draws; start points bit-exact; the
    # rest within the device's sin/cos rounding
    assert np.array_equal(got["structure_ptr"], ref["structure_ptr"])
    assert np.array_equal(got["flag"], ref["flag"])
    starts = ref["structure_ptr"][:-1]
    for k in ("x", "y", "z"):
        assert np.array_equal(bits(got[k][starts]), bits(ref[k][starts]))
        np.testing.assert_allclose(got[k], ref[k], rtol=0, atol=1e-10)
    assert np.array_equal(bits(got["radii"]), bits(ref["radii"]))


def test_device_built_network_through_the_hot_path(cuda_ok):
    # generator + window trim on the device, then the stages; against the host-built network
    cfg = NetworkConfig(side=1.6, n_cnts=700, seed=7, tolerance=1e-14)
    host = generate_cnt_network(cfg).extract_window(cfg)
    p = cfg.params()
    with Context(0) as ctx:
        ctx.upload(host)
        r_host = ctx.network_to_conductance(p)
        lab_h, nl_h = ctx.labels()
        j_h = ctx.junctions()
    with Context(0) as ctx:
        ctx.generate_network(cfg)
        got = ctx.network()
        r_dev = ctx.network_to_conductance(p)
        lab_d, nl_d = ctx.labels()
        j_d = ctx.junctions()
    assert_same_network(got, host.arrays(), exact_xyz=False)
    assert nl_d == nl_h and np.array_equal(lab_d, lab_h)
    assert all(np.array_equal(a, b) for a, b in zip(j_d[:4], j_h[:4]))
    np.testing.assert_allclose(np.array(r_dev.resistances), np.array(r_host.resistances), rtol=1e-9)


def test_device_construction_time_at_the_bench_size(cuda_ok):
    # the 25k-CNT / 6 um network: host generation + trim + upload against the device path
    cfg = NetworkConfig(side=6.0, n_cnts=25000, seed=2000000)
    with Context(0) as ctx:
        ctx.generate_network(cfg)  # warm-up (allocations); every call returns with its work complete
        t0 = time.perf_counter()
        for _ in range(3):
            ctx.generate_network(cfg)
        dev_s = (time.perf_counter() - t0) / 3
        got = ctx.network()
        t0 = time.perf_counter()
        host = generate_cnt_network(cfg).extract_window(cfg)
        ctx.upload(host)
        host_s = time.perf_counter() - t0
    ref = host.arrays()
    assert np.array_equal(got["structure_ptr"], ref["structure_ptr"]) and np.array_equal(got["cnts_inside"], ref["cnts_inside"])
    print(f"network construction, 25k CNTs / 6 um: device {dev_s * 1e3:.2f} ms, host generate + trim + upload {host_s * 1e3:.1f} ms")
