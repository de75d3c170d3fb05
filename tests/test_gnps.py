"""GNP input of the hybrid CNT/GNP configuration: cicy_read_gnps builds the GNPs
(rotation, vertices, face planes) bit for bit as upstream's Read_Network does,
checked against the golden fixture made by the upstream program
(tests/golden/make_gnp_golden.py) and, when oracle/_ref/gnp_dump is built, live
on another seed.  The fixture's GNP-GNP distances (upstream GJK / EPA) and GNP
region lists are the oracle of the GNP contact search; the distances' upstream
invariants and the CPU restatement of the region filling are checked here."""
import os
import subprocess

import numpy as np
import pytest

from cicy_geom_b200 import _abi
from cicy_geom_b200.network import generate_gnps, read_gnps, write_gnp_file

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "gnp_120_s4000000.npz")
REF = os.path.join(ROOT, "oracle", "_ref", "gnp_dump")


def golden():
    return dict(np.load(GOLDEN))


def check_against(z, ours, prefix):
    n = len(ours["l"])
    assert np.array_equal(z[prefix + "gnp_lt"].reshape(n, 2), np.stack([ours["l"], ours["t"]], 1))
    assert np.array_equal(z[prefix + "gnp_center"].reshape(n, 3), ours["center"])
    assert np.array_equal(z[prefix + "gnp_rotation"].reshape(n, 3, 3), ours["rotation"])
    assert np.array_equal(z[prefix + "gnp_vertices"].reshape(n, 8, 3), ours["vertices"])
    assert np.array_equal(z[prefix + "gnp_planes"].reshape(n, 6, 4), ours["planes"])


def test_gnp_geometry_matches_upstream_golden(tmp_path):
    z = golden()
    g = {"l": z["in_l"], "t": z["in_t"], "theta": z["in_theta"], "phi": z["in_phi"], "center": z["in_center"]}
    write_gnp_file(str(tmp_path), g)
    check_against(z, read_gnps(str(tmp_path)), "ref_")


def test_golden_gnp_distances_keep_upstream_invariants():
    z = golden()
    vdw, tunnel = float(z["meta"][3]), float(z["meta"][4])
    a, b = z["ref_pair_a"], z["ref_pair_b"]
    pen = z["ref_pair_penetrating"].astype(bool)
    d = z["ref_pair_dist"]
    n_dir = z["ref_pair_direction"].reshape(-1, 3)
    disp = z["ref_pair_displacement"].reshape(-1, 3)
    assert np.all(a < b) and len(a) > 1000
    assert pen.sum() > 100 and (~pen).sum() > 100  # both GJK-only and EPA cases
    assert np.all(d[pen] == vdw)  # interpenetrating: moved apart to the van der Waals distance
    assert np.all(d[~pen] > 0) and np.all(disp[~pen] == 0)
    assert np.allclose(np.linalg.norm(n_dir, axis=1), 1.0, atol=1e-15)
    # the move of GNP b is along the direction, by the penetration depth plus the van der Waals distance
    mag = np.linalg.norm(disp[pen], axis=1)
    assert np.all(mag > vdw)
    np.testing.assert_allclose(disp[pen] / mag[:, None], n_dir[pen], atol=1e-12)
    assert ((d <= tunnel) & ~pen).sum() > 0  # separated pairs within the tunnelling cutoff


@pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref/gnp_dump not built")
def test_gnp_geometry_matches_upstream_live(tmp_path):
    from oracle.dumpio import read_dump

    d = str(tmp_path)
    g = generate_gnps(60, 3.0, 4_000_123)
    write_gnp_file(d, g)
    with open(os.path.join(d, "sample_geom.csv"), "w") as f:
        f.write("0,0,0\n3.0,3.0,3.0\n")
    subprocess.run([REF, d, os.path.join(d, "g.bin"), "0.00034", "0.0018"], check=True, capture_output=True, timeout=600)
    check_against(read_dump(os.path.join(d, "g.bin")), read_gnps(d), "")


def test_gnp_file_errors(tmp_path):
    d = str(tmp_path)
    with pytest.raises(_abi.CicyError, match="gnp_data.dat"):
        read_gnps(d)
    write_gnp_file(d, generate_gnps(5, 2.0, 1))
    path = os.path.join(d, "gnp_data.dat")
    data = open(path, "rb").read()
    open(path, "wb").write(data[:-8])
    with pytest.raises(_abi.CicyError, match="end-of-file of gnp_data.dat"):
        read_gnps(d)


def test_gnp_contact_grid_oracle_matches_upstream_golden():
    """The CPU restatement of upstream's GNP region filling (oracle/gnp_oracle.py)
    gives upstream's region lists on the fixture."""
    from oracle import gnp_oracle as G

    z = golden()
    side, gs, ov_cnt, ov_gnp = float(z["meta"][1]), float(z["meta"][5]), float(z["meta"][6]), float(z["meta"][7])
    win = [0.0, 0.0, 0.0, side, side, side, side, side, side]
    n, l = G.region_grid(win, [gs] * 3, ov_cnt, ov_gnp)
    assert list(n) == list(z["ref_sd_n_regions"]) and np.array_equal(l, z["ref_sd_l_regions"])
    N = len(z["in_l"])
    regs = G.fill_sectioned_domain_gnps(win, z["ref_gnp_vertices"].reshape(N, 8, 3), z["in_l"], z["in_t"], range(N), n, l, ov_gnp)
    ptr, idx = z["ref_sd_ptr"], z["ref_sd_idx"]
    assert len(regs) == len(ptr) - 1
    assert all(list(idx[ptr[k]:ptr[k + 1]]) == regs[k] for k in range(len(regs)))
    assert len(idx) > 10000


def test_golden_gnp_closest_points_keep_upstream_invariants():
    """Upstream's closest GNP points: inside points flagged -1 at distance 0, the
    others at the returned distance from the query, every branch represented."""
    z = golden()
    q = z["in_queries"]
    fl, d, c = z["ref_query_flag"], z["ref_query_dist"], z["ref_query_point"].reshape(-1, 3)
    assert set(np.unique(fl)) == {-1, 0}
    assert np.all(d[fl == -1] == 0)
    out = fl == 0
    assert out.sum() > 500 and (~out).sum() > 500
    np.testing.assert_allclose(np.linalg.norm(q[out, :3] - c[out], axis=1), d[out], rtol=1e-9, atol=1e-12)
