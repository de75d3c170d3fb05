"""The device window trim (window_trim.cuh, the code of cicy_ctx_extract_window)
built for the host and driven through the device's sequence of passes
(tests/host_window.cpp), against the host restatement cicy_extract_window
(itself bit-exact with upstream's Shells + Cutoff_Wins, tests/test_host_network.py).
Seeded networks whose CNTs leave and re-enter the window many times, so the
pieces, their second trim and the face lists' run-length rule are all exercised;
coordinates compared bit for bit."""
import os
import shutil
import subprocess
from dataclasses import replace

import numpy as np
import pytest

from cicy_geom_b200.network import NetworkConfig, generate_cnt_network

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cicy_geom_b200", "csrc")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("hostwin") / "host_window")
    subprocess.run([cxx, "-O2", "-std=c++17", "-ffp-contract=off", f"-I{CSRC}", os.path.join(ROOT, "tests", "host_window.cpp"), "-o", out],
                   check=True, capture_output=True, timeout=300)
    return out


def runs(a):
    sp, si = a["structure_ptr"], a["structure_idx"]
    ln = np.diff(sp).astype(np.int32)
    st = np.where(ln > 0, si[np.minimum(sp[:-1], max(len(si) - 1, 0))] if len(si) else 0, 0).astype(np.int32)
    return st, ln


def emulate(exe, tmp_path, raw, cfg):
    w = cfg.window_params()
    st, ln = runs(raw)
    n, c = len(raw["x"]), len(raw["radii"])
    inp, out = str(tmp_path / "win_in.bin"), str(tmp_path / "win_out.bin")
    s = w.sample
    wd = [s.min_x, s.min_y, s.min_z, s.len_x, s.len_y, s.len_z, s.max_x, s.max_y, s.max_z, *w.win_max, *w.win_min, *w.win_delt,
          w.step_length, 0.0, 0.0, 0.0]
    with open(inp, "wb") as f:
        f.write(np.array([n, c, w.min_points], "<i4").tobytes())
        f.write(np.array(wd, "<f8").tobytes())
        for k in ("x", "y", "z"):
            f.write(raw[k].astype("<f8").tobytes())
        f.write(raw["flag"].astype("<i4").tobytes() + st.astype("<i4").tobytes() + ln.astype("<i4").tobytes())
        f.write(raw["radii"].astype("<f8").tobytes())
    subprocess.run([exe, inp, out], check=True, timeout=300)
    b = open(out, "rb").read()
    h = np.frombuffer(b[:24], "<i4")
    status, n, U, ni, nb, nq = (int(v) for v in h)
    o = 24
    res = {"status": status}

    def take(name, dt, count):
        nonlocal o
        sz = np.dtype(dt).itemsize * count
        res[name] = np.frombuffer(b[o:o + sz], dt).copy()
        o += sz

    for k in ("x", "y", "z"):
        take(k, "<f8", n)
    take("flag", "<i4", n)
    take("cs", "<i4", U)
    take("cl", "<i4", U)
    take("radii", "<f8", U)
    take("cnts_inside", "<i4", ni)
    take("boundary_cnt_ptr", "<i4", 7)
    take("boundary_cnt_idx", "<i4", nb)
    take("boundary_pts_ptr", "<i4", 7)
    take("boundary_pts_idx", "<i4", nq)
    take("window", "<f8", 9)
    cl = res["cl"].astype(np.int64)
    res["structure_ptr"] = np.concatenate([[0], np.cumsum(cl)]).astype(np.int64)
    res["structure_idx"] = (np.repeat(res["cs"].astype(np.int64) - res["structure_ptr"][:-1], cl) +
                            np.arange(res["structure_ptr"][-1], dtype=np.int64))
    return res


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


CASES = [
    # (side, CNTs, seed, max turn): small cubes of long, curly CNTs cross the faces many times
    (1.0, 300, 11, 10.0),
    (0.8, 400, 12, 25.0),
    (1.6, 700, 7, 10.0),
    (2.0, 1200, 1, 10.0),
    (0.6, 250, 13, 40.0),
]


@pytest.mark.parametrize("side,n,seed,turn", CASES)
def test_device_window_trim_equals_host_restatement(exe, tmp_path, side, n, seed, turn):
    cfg = replace(NetworkConfig(side=side, n_cnts=n, seed=seed), max_turn_deg=turn)
    raw_net = generate_cnt_network(cfg)
    raw = raw_net.arrays()
    ref = raw_net.extract_window(cfg).arrays()
    got = emulate(exe, tmp_path, raw, cfg)
    assert got["status"] == 0
    assert np.array_equal(bits(got["x"]), bits(ref["x"]))
    assert np.array_equal(bits(got["y"]), bits(ref["y"]))
    assert np.array_equal(bits(got["z"]), bits(ref["z"]))
    assert np.array_equal(got["flag"], ref["flag"])
    assert np.array_equal(got["structure_ptr"], ref["structure_ptr"])
    assert np.array_equal(got["structure_idx"], ref["structure_idx"])
    assert np.array_equal(bits(got["radii"]), bits(ref["radii"]))
    assert np.array_equal(got["cnts_inside"], ref["cnts_inside"])
    for k in ("boundary_cnt_ptr", "boundary_cnt_idx", "boundary_pts_ptr", "boundary_pts_idx"):
        assert np.array_equal(got[k].astype(np.int64), ref[k].astype(np.int64)), k
    assert np.array_equal(bits(got["window"]), bits(ref["window"]))
    # the cases cut CNTs into pieces (new indices beyond the generated CNTs)
    assert len(ref["radii"]) > n


def test_device_window_trim_edge_cases(exe, tmp_path):
    # short CNTs far from the faces (no pieces, possibly no boundary entries), and an empty network
    for cfg in (replace(NetworkConfig(side=6.0, n_cnts=40, seed=21), len_min=0.06, len_max=0.08),
                NetworkConfig(side=1.0, n_cnts=0, seed=22)):
        raw_net = generate_cnt_network(cfg)
        raw = raw_net.arrays()
        ref = raw_net.extract_window(cfg).arrays()
        got = emulate(exe, tmp_path, raw, cfg)
        assert got["status"] == 0
        for k in ("x", "y", "z"):
            assert np.array_equal(bits(got[k]), bits(ref[k]))
        for k in ("flag", "structure_ptr", "structure_idx", "cnts_inside", "boundary_cnt_ptr", "boundary_cnt_idx", "boundary_pts_ptr",
                  "boundary_pts_idx"):
            assert np.array_equal(got[k].astype(np.int64), ref[k].astype(np.int64)), k


def test_layout_check_rejects_a_network_out_of_generator_order(exe, tmp_path):
    cfg = NetworkConfig(side=1.0, n_cnts=50, seed=3)
    raw = generate_cnt_network(cfg).arrays()
    raw["flag"] = raw["flag"].copy()
    raw["flag"][raw["structure_ptr"][7]] = 8  # a point of CNT 7 flagged as CNT 8
    assert emulate(exe, tmp_path, raw, cfg)["status"] == 5  # WIN_LAYOUT
