"""The device geometry headers built for the host: gnp_geom.cuh (closest GNP
point), gnp_gjk.cuh (GJK / EPA), gnp_junction.cuh (junction points) and
gnp_triangulation.cuh (per-GNP triangulation) are compiled by g++ without FMA
contraction from the same source the CUDA kernels use (tests/host_geometry.cpp
drives them) and compared with upstream's results in the golden fixtures: 2,400
closest points, 2,358 GNP-GNP distance steps, 565 junction steps (the random
fixture and the hand-placed cases), the triangulation edges of 150 GNPs."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cicy_geom_b200", "csrc")
GOLDEN = os.path.join(ROOT, "tests", "golden", "gnp_120_s4000000.npz")
KAT = os.path.join(ROOT, "tests", "golden", "gnp_junction_cases.npz")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("hostgeom") / "host_geometry")
    subprocess.run([cxx, "-O2", "-std=c++17", "-ffp-contract=off", f"-I{CSRC}", os.path.join(ROOT, "tests", "host_geometry.cpp"), "-o", out],
                   check=True, capture_output=True, timeout=300)
    return out


def run(exe, tmp_path, mode, z, items, extra=()):
    V, F = z["ref_gnp_vertices"], z["ref_gnp_planes"]
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(inp, "wb") as f:
        f.write(np.array([len(V) // 24, len(items)], "<i4").tobytes())
        f.write(V.astype("<f8").tobytes() + F.astype("<f8").tobytes())
        f.write(np.asarray(items, "<f8").tobytes() + np.asarray(extra, "<f8").tobytes())
    subprocess.run([exe, mode, inp, out], check=True, timeout=300)
    return np.fromfile(out, "<f8").reshape(len(items), -1)


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def test_closest_point_host_build_matches_upstream(exe, tmp_path):
    z = dict(np.load(GOLDEN))
    r = run(exe, tmp_path, "closest", z, z["in_queries"])
    assert np.array_equal(r[:, 0], z["ref_query_flag"])
    assert np.array_equal(bits(r[:, 1]), bits(z["ref_query_dist"]))
    ok = z["ref_query_flag"] == 0
    assert np.array_equal(bits(r[ok, 2:5]), bits(z["ref_query_point"].reshape(-1, 3)[ok]))


def test_gjk_epa_host_build_matches_upstream(exe, tmp_path):
    z = dict(np.load(GOLDEN))
    r = run(exe, tmp_path, "pairs", z, np.stack([z["ref_pair_a"], z["ref_pair_b"]], 1), [float(z["meta"][3])])
    assert np.all(r[:, 0] == 0) and np.array_equal(r[:, 1], z["ref_pair_penetrating"])
    assert np.array_equal(bits(r[:, 2]), bits(z["ref_pair_dist"]))
    assert np.array_equal(bits(r[:, 3:6]), bits(z["ref_pair_direction"].reshape(-1, 3)))
    assert np.array_equal(bits(r[:, 6:9]), bits(z["ref_pair_displacement"].reshape(-1, 3)))


@pytest.mark.parametrize("path,side", [(GOLDEN, 2.0), (KAT, 12.0)])
def test_junction_points_host_build_match_upstream(exe, tmp_path, path, side):
    z = dict(np.load(path))
    jp = z["ref_junc_pair"]
    r = run(exe, tmp_path, "junction", z, np.stack([z["ref_pair_a"][jp], z["ref_pair_b"][jp]], 1), [0.00034, 0, 0, 0, side, side, side])
    ok = z["ref_junc_ok"].astype(bool)
    assert np.all(r[:, 0] == 0) and np.array_equal(r[:, 1] == 0, ok)
    assert np.array_equal(r[ok, 2], z["ref_junc_outside"][ok])
    assert np.array_equal(bits(r[ok, 3:9]), bits(z["ref_junc_points"].reshape(-1, 6)[ok]))


LABELS = os.path.join(ROOT, "tests", "golden", "gnp_hybrid_labels.npz")


@pytest.mark.parametrize("path", [GOLDEN, LABELS])
def test_triangulation_host_build_matches_upstream(exe, tmp_path, path):
    z = dict(np.load(path))
    N = len(z["in_l"])
    pts = z["ref_mixjn_points"]
    sp, si = z["ref_mixjn_structure_ptr"], z["ref_mixjn_structure_idx"]
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(inp, "wb") as f:
        f.write(np.array([N, len(pts) // 3], "<i4").tobytes() + pts.astype("<f8").tobytes())
        f.write(sp.astype("<i4").tobytes() + si.astype("<i4").tobytes())
        f.write(z["ref_gnp_lt"].reshape(N, 2)[:, 0].astype("<f8").tobytes() + z["ref_gnp_center"].astype("<f8").tobytes())
        f.write(z["ref_gnp_rotation"].astype("<f8").tobytes() + z["ref_gnp_planes"].astype("<f8").tobytes())
    subprocess.run([exe, "triangulate", inp, out], check=True, timeout=300)
    r = np.fromfile(out, "<i4")
    assert np.array_equal(r[:N + 1], z["ref_tri_ptr"]) and np.array_equal(r[N + 1:], z["ref_tri_edges"])
