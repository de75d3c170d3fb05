"""Generate the golden fixtures under tests/golden/ from the upstream program.

Runs oracle/_ref/ref_dump (the upstream CICY_geom sources compiled in place by
oracle/Makefile) on seeded synthetic networks and on hand-made known-answer
networks, and stores the upstream outputs of every hot-path stage as .npz.
Needs the upstream tree only to build ref_dump (its path in the environment
variable CICY_REF_DIR); the fixtures themselves are self-contained.

    CICY_REF_DIR=<upstream CICY_geom source tree> python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cicy_geom_b200.network import HostNetwork, NetworkConfig, generate_cnt_network, write_read_network_files  # noqa: E402
from oracle.dumpio import read_dump  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "ref_dump")

# (name, side, n_cnts, seed, full_sectioned_domain)
SEEDED = [
    ("c1_400_s1", 2.0, 400, 1, True),       # configuration 1: 2 um, 400 CNTs (does not percolate)
    ("c1p_1200_s1", 2.0, 1200, 1, False),   # percolating variant of configuration 1
    ("c1p_800_s2", 2.0, 800, 2, False),
    ("c1p_800_s3", 2.0, 800, 3, False),     # two clusters percolating along y only
    ("c1p_800_s5", 2.0, 800, 5, False),     # two percolated clusters (XYZ and Y)
]


def net_hash(a: dict) -> str:
    h = hashlib.sha256()
    for k in ("x", "y", "z", "flag", "structure_ptr", "structure_idx", "radii", "cnts_inside", "boundary_cnt_ptr",
              "boundary_cnt_idx", "boundary_pts_ptr", "boundary_pts_idx"):
        h.update(np.ascontiguousarray(a[k]).tobytes())
    return h.hexdigest()


def arr_hash(*arrs) -> str:
    h = hashlib.sha256()
    for a in arrs:
        h.update(np.ascontiguousarray(np.asarray(a, dtype=np.int64)).tobytes())
    return h.hexdigest()


def polyline(p0, p1, step=0.01):
    p0, p1 = np.asarray(p0, float), np.asarray(p1, float)
    L = np.linalg.norm(p1 - p0)
    n = 1 + int(L / step)
    t = np.arange(n) * step / L
    return p0[None, :] + t[:, None] * (p1 - p0)[None, :]


def kat_networks():
    """Hand-made known-answer networks in a 1 um cube (r = 5 nm, d_t = 1.8 nm)."""
    r = 0.005
    g = 2 * r + 0.001  # centre distance: junction distance 1 nm
    nets = {}
    # two parallel wires, each touching both x faces: upstream counts the element at
    # either end of such a CNT when summing the current through face b1
    # (Electrical_analysis.cpp:547-605), in- and out-currents cancel, R = inf upstream
    nets["kat_two_parallel"] = [polyline((-0.05, 0.5, 0.5), (1.05, 0.5, 0.5)), polyline((-0.05, 0.5 + g, 0.5), (1.05, 0.5 + g, 0.5))]
    # one spanning wire plus a dangling side CNT: the real-resistor system has one free
    # node whose linear-ramp initial guess is exact, so r0 = 0 and the first CG step
    # divides 0 by 0 (Direct_Electrifying.cpp:1586-1596): upstream reports R = nan
    nets["kat_spanning_single"] = [polyline((-0.05, 0.3, 0.3), (1.05, 0.3, 0.3)), polyline((0.5, 0.3 + g, 0.3), (0.5, 0.8, 0.3))]
    # two overlapping CNTs in series: R = R_cnt(A: face..P1) + R_junction + R_cnt(B: P2..face), closed form
    nets["kat_series"] = [polyline((-0.05, 0.5, 0.5), (0.6, 0.5, 0.5)), polyline((0.45, 0.5 + g, 0.5), (1.05, 0.5 + g, 0.5))]
    # chain of three CNTs along x
    nets["kat_three_chain"] = [polyline((-0.05, 0.5, 0.5), (0.45, 0.5, 0.5)), polyline((0.40, 0.5 + g, 0.5), (0.85, 0.5 + g, 0.5)),
                               polyline((0.80, 0.5 + 2 * g, 0.5), (1.05, 0.5 + 2 * g, 0.5))]
    # two CNT tips straddling a grid-cell corner diagonally: within the cutoff but never tested (no contact)
    c, dl = 0.5, 0.003
    nets["kat_corner_pair"] = [polyline((c - dl - 0.2, c - dl, c - dl), (c - dl, c - dl, c - dl)),
                               polyline((c + dl, c + dl, c + dl), (c + dl + 0.2, c + dl, c + dl))]
    # interpenetrating crossing CNTs: several pairs clamp to d_vdW (ties broken by scan order)
    nets["kat_vdw_tie"] = [polyline((0.2, 0.5, 0.5), (0.8, 0.5, 0.5)), polyline((0.5, 0.2, 0.5 + 0.004), (0.5, 0.8, 0.5 + 0.004)),
                           polyline((-0.05, 0.52, 0.5), (1.05, 0.52, 0.5))]
    return nets


def host_network_from_polylines(lines) -> HostNetwork:
    xs = np.concatenate(lines)
    counts = [len(l) for l in lines]
    sp = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    flag = np.concatenate([np.full(c, i, np.int32) for i, c in enumerate(counts)])
    return HostNetwork.from_arrays({"x": xs[:, 0], "y": xs[:, 1], "z": xs[:, 2], "flag": flag, "structure_ptr": sp,
                                    "structure_idx": np.arange(len(xs), dtype=np.int64), "radii": np.full(len(lines), 0.005),
                                    "window": np.zeros(9)})


def capture(name, cfg: NetworkConfig, raw: HostNetwork, full_sd: bool, store_inputs: bool):
    with tempfile.TemporaryDirectory(prefix="cicy_golden_") as d:
        write_read_network_files(d, raw, cfg)
        dump = os.path.join(d, "dump.bin")
        subprocess.run([REF, "dump", d, dump], check=True, capture_output=True)
        D = read_dump(dump)
    win = raw.extract_window(cfg).arrays()
    xyz = D["points_xyz"].reshape(-1, 3)
    assert np.array_equal(win["x"], xyz[:, 0]) and np.array_equal(win["flag"], D["points_flag"]), name
    assert np.array_equal(win["boundary_pts_idx"], D["boundary_pts_idx"]), name
    out = {"meta_side": cfg.side, "meta_n_cnts": cfg.n_cnts, "meta_seed": cfg.seed, "meta_tolerance": cfg.tolerance,
           "net_sha256": np.array(net_hash(win)), "params": D["params"], "resistances": D["resistances"],
           "sd_sha256": np.array(arr_hash(D["sd_ptr"], D["sd_idx"])), "n_slots": np.array(len(D["sd_idx"]))}
    if full_sd:
        out["sd_ptr"] = D["sd_ptr"].astype(np.int32)
        out["sd_idx"] = D["sd_idx"].astype(np.int32)
    if store_inputs:
        for k, v in win.items():
            out["in_" + k] = v
    for k in ("pc_Pa", "pc_CNTb", "pc_Pb", "pc_dist", "labels_cnt", "n_labels", "junc_P1", "junc_N1", "junc_P2", "junc_N2",
              "junc_dist", "elements_ptr", "elements_idx", "clusters_ptr", "clusters_idx", "family", "cluster_junc_ptr",
              "cluster_junc_idx", "isolated_ptr", "isolated_idx", "bn_volumes", "bn_volumes_cnt", "bn_volumes_gnp",
              "bn_dead_branches", "bn_dead_gnps"):
        out[k] = D[k]
    for k in list(D):
        if k.startswith("c") and k[1].isdigit() and not k.endswith("times"):
            out[k] = D[k]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: points {len(win['x'])} slots {len(D['sd_idx'])} contacts {len(D['pc_Pa'])} labels {int(D['n_labels'][0])} "
          f"junctions {len(D['junc_P1'])} percolated {len(D['family'])} R {D['resistances']}")


def main():
    if not os.path.exists(REF):
        ref_dir = os.environ.get("CICY_REF_DIR")
        if not ref_dir:
            sys.exit("set CICY_REF_DIR to the upstream CICY_geom source tree to build oracle/_ref/ref_dump")
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF_DIR={ref_dir}", "-j8"], check=True)
    for name, side, n, seed, full in SEEDED:
        cfg = NetworkConfig(side=side, n_cnts=n, seed=seed)
        capture(name, cfg, generate_cnt_network(cfg), full, False)
    for name, lines in kat_networks().items():
        cfg = NetworkConfig(side=1.0, n_cnts=len(lines), seed=0)
        capture(name, cfg, host_network_from_polylines(lines), True, True)


if __name__ == "__main__":
    main()
