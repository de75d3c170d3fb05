import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the device path through the C ABI")


SEEDED = {"c1_400_s1": (2.0, 400, 1), "c1p_1200_s1": (2.0, 1200, 1), "c1p_800_s2": (2.0, 800, 2), "c1p_800_s3": (2.0, 800, 3),
          "c1p_800_s5": (2.0, 800, 5)}
KATS = ["kat_two_parallel", "kat_spanning_single", "kat_series", "kat_three_chain", "kat_corner_pair", "kat_vdw_tie"]
ALL = list(SEEDED) + KATS


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_network(name):
    """(config, window network as a HostNetwork, golden dict) of a fixture."""
    from cicy_geom_b200.network import HostNetwork, NetworkConfig, generate_cnt_network

    z = load_golden(name)
    if name in SEEDED:
        side, n, seed = SEEDED[name]
        cfg = NetworkConfig(side=side, n_cnts=n, seed=seed)
        net = generate_cnt_network(cfg).extract_window(cfg)
    else:
        cfg = NetworkConfig(side=1.0, n_cnts=int(z["meta_n_cnts"]), seed=0)
        net = HostNetwork.from_arrays({k[3:]: z[k] for k in z if k.startswith("in_")})
    return cfg, net, z


def net_sha(a):
    import hashlib

    h = hashlib.sha256()
    for k in ("x", "y", "z", "flag", "structure_ptr", "structure_idx", "radii", "cnts_inside", "boundary_cnt_ptr", "boundary_cnt_idx",
              "boundary_pts_ptr", "boundary_pts_idx"):
        h.update(np.ascontiguousarray(a[k]).tobytes())
    return h.hexdigest()


def arr_sha(*arrs):
    import hashlib

    h = hashlib.sha256()
    for a in arrs:
        h.update(np.ascontiguousarray(np.asarray(a, dtype=np.int64)).tobytes())
    return h.hexdigest()


def csr_list(z, name):
    p, i = z[name + "_ptr"], z[name + "_idx"]
    return [list(i[p[k]:p[k + 1]]) for k in range(len(p) - 1)]


def assert_ulp(actual, desired, n_ulp, msg=""):
    """|actual - desired| <= n_ulp units in the last place of the larger magnitude, per entry.

    DEA values built from exp() (exponential tunnelling junctions) differ between CUDA's and
    glibc's exp by at most 1 ulp; the products and the reciprocal after it carry that through
    as a few ulp of the conductance."""
    a = np.asarray(actual, dtype=np.float64)
    d = np.asarray(desired, dtype=np.float64)
    assert a.shape == d.shape, (msg, a.shape, d.shape)
    tol = n_ulp * np.spacing(np.maximum(np.abs(a), np.abs(d)))
    bad = np.abs(a - d) > tol
    assert not bad.any(), f"{msg}: {int(bad.sum())} of {a.size} entries beyond {n_ulp} ulp; first at {int(np.argmax(bad))}"


def golden_systems(z):
    """[(prefix, kind, cluster)] of the DEA systems a fixture holds, in solve order."""
    out = []
    for k in range(len(z["family"])):
        if f"c{k}_u_nodes" in z:
            out.append((f"c{k}_u_", "unit", k))
        for d in range(3):
            if f"c{k}_d{d}_nodes" in z:
                out.append((f"c{k}_d{d}_", d, k))
    return out


@pytest.fixture(scope="session")
def cuda_ok():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
