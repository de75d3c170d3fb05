"""GNP part of the contact grid on the device (cicy_gnp_sectioned_domain) against
upstream's region lists (golden fixture made by the upstream program) and the
CPU restatement (oracle/gnp_oracle.py) on another seed and a smaller window."""
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
