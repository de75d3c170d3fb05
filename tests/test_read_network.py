"""Read_Network's files (cicy_read_network): the binary and CSV readers against
the writer (bit-exact round trip), the upstream error cases, and, when the
upstream program is built (oracle/_ref/ref_dump), against upstream's own
Read_Network + Cutoff_Wins on the same files."""
import os
import subprocess

import numpy as np
import pytest

from cicy_geom_b200 import _abi
from cicy_geom_b200.network import NetworkConfig, generate_cnt_network, read_network_files, write_read_network_files

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_dump")
KEYS = ("x", "y", "z", "flag", "radii", "structure_ptr", "structure_idx")
WINDOW_KEYS = KEYS + ("cnts_inside", "boundary_cnt_ptr", "boundary_cnt_idx", "boundary_pts_ptr", "boundary_pts_idx")


def small(seed=7, n=400):
    cfg = NetworkConfig(side=2.0, n_cnts=n, seed=seed)
    return cfg, generate_cnt_network(cfg)


@pytest.mark.parametrize("file_type", ["dat", "csv"])
def test_round_trip_bit_exact(tmp_path, file_type):
    cfg, raw = small()
    write_read_network_files(str(tmp_path), raw, cfg, file_type)
    got = read_network_files(str(tmp_path), file_type)
    a, b = raw.arrays(), got.arrays()
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(np.asarray(a["window"]), np.asarray(b["window"]))
    # the read network goes through the same window extraction
    wa, wb = raw.extract_window(cfg).arrays(), got.extract_window(cfg).arrays()
    for k in WINDOW_KEYS:
        assert np.array_equal(wa[k], wb[k]), k


def test_upstream_error_cases(tmp_path):
    cfg, raw = small(n=50)
    d = str(tmp_path)
    with pytest.raises(_abi.CicyError, match="sample_geom.csv"):
        read_network_files(d, "dat")
    write_read_network_files(d, raw, cfg, "dat")
    path = os.path.join(d, "cnt_coordinates.dat")
    data = open(path, "rb").read()
    open(path, "wb").write(data[: len(data) - 24])  # one point short
    with pytest.raises(_abi.CicyError, match="end-of-file of cnt_coordinates.dat"):
        read_network_files(d, "dat")
    write_read_network_files(d, raw, cfg, "csv")
    path = os.path.join(d, "cnt_struct.csv")
    lines = open(path).read().splitlines()
    open(path, "w").write("\n".join([f"{len(lines) - 1},{len(lines)}"] + lines[1:]) + "\n")
    with pytest.raises(_abi.CicyError, match="different number of CNTs"):
        read_network_files(d, "csv")
    with pytest.raises(KeyError):
        read_network_files(d, "vtk")


@pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref/ref_dump not built")
def test_csv_reader_and_window_match_upstream(tmp_path):
    """Upstream reads the same CSV files (Read_cnt_data_from_csv) and extracts the
    window; its points, CNT structure and boundary lists equal ours bit for bit."""
    from oracle.dumpio import read_dump

    cfg, raw = small(seed=11)
    d = str(tmp_path)
    write_read_network_files(d, raw, cfg, "csv")
    subprocess.run([REF, "dump", d, os.path.join(d, "dump.bin")], check=True, capture_output=True, timeout=600)
    z = read_dump(os.path.join(d, "dump.bin"))
    w = read_network_files(d, "csv").extract_window(cfg).arrays()
    xyz = z["points_xyz"].reshape(-1, 3)
    idx = np.arange(len(w["x"]))
    assert np.array_equal(xyz[:, 0], w["x"][idx]) and np.array_equal(xyz[:, 1], w["y"][idx]) and np.array_equal(xyz[:, 2], w["z"][idx])
    assert np.array_equal(z["points_flag"], w["flag"])
    assert np.array_equal(z["structure_ptr"], w["structure_ptr"]) and np.array_equal(z["structure_idx"], w["structure_idx"])
    assert np.array_equal(z["radii"], w["radii"])
    assert np.array_equal(z["cnts_inside"], w["cnts_inside"])
    assert np.array_equal(z["boundary_cnt_ptr"], w["boundary_cnt_ptr"]) and np.array_equal(z["boundary_cnt_idx"], w["boundary_cnt_idx"])
    assert np.array_equal(z["boundary_pts_ptr"], w["boundary_pts_ptr"]) and np.array_equal(z["boundary_pts_idx"], w["boundary_pts_idx"])


@pytest.mark.parametrize("n", [1, 3, 40])
def test_csv_edge_cases(tmp_path, n):
    """Tiny files (fewer lines than parsing threads), no final newline, a missing
    point, and a line without its numbers."""
    cfg, raw = small(seed=5, n=n)
    d = str(tmp_path)
    write_read_network_files(d, raw, cfg, "csv")
    a = raw.arrays()
    path = os.path.join(d, "cnt_coordinates.csv")
    text = open(path).read()
    open(path, "w").write(text.rstrip("\n"))
    b = read_network_files(d, "csv").arrays()
    for k in ("x", "y", "z", "flag", "structure_ptr"):
        assert np.array_equal(a[k], b[k]), k
    open(path, "w").write("\n".join(text.splitlines()[:-1]) + "\n")
    with pytest.raises(_abi.CicyError, match="end-of-file of cnt_coordinates.csv"):
        read_network_files(d, "csv")
    open(path, "w").write(text.replace("\n", "\n\n", 1))
    with pytest.raises(_abi.CicyError, match="not x,y,z"):
        read_network_files(d, "csv")
