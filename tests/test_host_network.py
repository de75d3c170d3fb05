"""Host-side network sources: seeded generator and window extraction (CPU)."""
import numpy as np
import pytest
from conftest import KATS, SEEDED, golden_network, load_golden, net_sha

from cicy_geom_b200.network import NetworkConfig, generate_cnt_network


def test_generator_is_deterministic_and_has_the_requested_statistics():
    cfg = NetworkConfig(side=2.0, n_cnts=300, seed=11)
    a = generate_cnt_network(cfg).arrays()
    b = generate_cnt_network(cfg).arrays()
    for k in ("x", "y", "z", "structure_ptr"):
        assert np.array_equal(a[k], b[k])
    counts = np.diff(a["structure_ptr"])
    assert counts.min() >= 1 + int(0.5 / 0.01) and counts.max() <= 1 + int(1.5 / 0.01)
    p = np.stack([a["x"], a["y"], a["z"]], 1)
    sp = a["structure_ptr"]
    steps = np.linalg.norm(np.diff(p, axis=0), axis=1)
    inner = np.ones(len(steps), bool)
    inner[sp[1:-1] - 1] = False  # drop jumps between CNTs
    assert np.allclose(steps[inner], 0.01, rtol=1e-9)
    starts = p[sp[:-1]]
    assert starts.min() >= 0 and starts.max() <= 2.0
    # turning angle between consecutive steps is at most 10 degrees
    d = np.diff(p, axis=0)[inner]
    d /= np.linalg.norm(d, axis=1)[:, None]
    same = inner[:-1] & inner[1:]
    cos = np.einsum("ij,ij->i", np.diff(p, axis=0)[:-1][same] / 0.01, np.diff(p, axis=0)[1:][same] / 0.01)
    assert np.degrees(np.arccos(np.clip(cos, -1, 1))).max() <= 10.0 + 1e-6


def test_seeds_give_independent_networks():
    a = generate_cnt_network(NetworkConfig(side=2.0, n_cnts=50, seed=1)).arrays()
    b = generate_cnt_network(NetworkConfig(side=2.0, n_cnts=50, seed=2)).arrays()
    assert not np.array_equal(a["x"][:10], b["x"][:10])


@pytest.mark.parametrize("name", list(SEEDED) + KATS)
def test_window_extraction_matches_upstream(name):
    """Shells + Cutoff_Wins restatement reproduces the upstream trimmed network bit for bit."""
    cfg, net, z = golden_network(name)
    assert net_sha(net.arrays()) == str(z["net_sha256"])


def test_window_extraction_boundary_lists_are_consistent():
    cfg, net, z = golden_network("c1p_1200_s1")
    a = net.arrays()
    w = a["window"]
    tol = 1e-10
    faces = {0: (2, w[8]), 1: (2, w[2]), 2: (0, w[6]), 3: (1, w[7]), 4: (0, w[0]), 5: (1, w[1])}
    coord = [a["x"], a["y"], a["z"]]
    for f in range(6):
        pts = a["boundary_pts_idx"][a["boundary_pts_ptr"][f]:a["boundary_pts_ptr"][f + 1]]
        ax, val = faces[f]
        assert np.all(np.abs(coord[ax][pts] - val) < tol)
    # the CNT of every point listed at a face is listed at that face too (the converse
    # does not hold upstream: a segment can register its CNT and then shift its end point)
    for f in range(6):
        cnts = set(a["boundary_cnt_idx"][a["boundary_cnt_ptr"][f]:a["boundary_cnt_ptr"][f + 1]])
        pts = a["boundary_pts_idx"][a["boundary_pts_ptr"][f]:a["boundary_pts_ptr"][f + 1]]
        assert set(a["flag"][pts]) <= cnts


def test_window_rejects_multiwindow_runs():
    from cicy_geom_b200._abi import CicyError

    cfg = NetworkConfig(side=2.0, n_cnts=20, seed=1)
    net = generate_cnt_network(cfg)
    wp = cfg.window_params()
    wp.win_min[0] = wp.win_min[1] = wp.win_min[2] = 1.0
    import ctypes as C

    from cicy_geom_b200._abi import lib

    out = C.c_void_p()
    assert lib().cicy_extract_window(net.handle, C.byref(wp), C.byref(out)) == 1
