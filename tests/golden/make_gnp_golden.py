"""Generate tests/golden/gnp_120_s4000000.npz from the upstream program.

Runs oracle/_ref/gnp_dump (upstream CICY_geom objects compiled in place by
oracle/Makefile) on 120 seeded GNPs in a 2 um cube (side U[0.5, 1.0] um,
thickness 10 nm, normal uniform on the sphere) and stores, next to the inputs,
upstream's GNPs as it reads them (rotation, vertices, face planes), upstream's
closest GNP point to 20 query points around each GNP (the CNT-GNP distance),
upstream's
GNP part of the contact grid (0.05 um regions, overlaps as Input_Reader sets
them) and, for every candidate pair, upstream's GNP-GNP distance step (GJK
distance, EPA when the GNPs interpenetrate, the move of the second GNP) and,
for the pairs within the tunnelling cutoff, upstream's junction points: the
oracle of the GNP contact search.  The hybrid sample also gets upstream's
labels, GNP point structures, GNP / mixed junction lists and the triangulation
of every GNP's points.  With a seeded 400-CNT network in the same
cube (regenerated by the tests from its seed and checked against the stored
SHA-256), it also stores upstream's CNT-GNP contacts of the mixed contact pass
(Find_adjacent_labels: point, GNP, contact-point number, junction distance,
closest GNP point) and the SHA-256 of upstream's CNT region lists.  The fixture
itself is self-contained apart from the seeded CNT network.

Also writes tests/golden/gnp_hybrid_labels.npz: upstream's CNT, GNP and mixed
labels of a sparser hybrid sample (30 GNPs, 250 CNTs), whose clusters stay
apart, and tests/golden/gnp_windows.npz: upstream's GNP window extraction
(Fill_gnps_inside) for two centred windows smaller than the sample (the
120-GNP fixture itself carries it for the whole sample as the window), and
tests/golden/gnp_hybrid_flow.npz: upstream's own stage sequence for GNP_CNT_mix
on both hybrid samples up to the percolated clusters, and
tests/golden/gnp_hybrid_electrical.npz: its electrical stage, stage by stage.

    python tests/golden/make_gnp_golden.py
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cicy_geom_b200.network import (NetworkConfig, generate_cnt_network, generate_gnps, read_network_files,  # noqa: E402
                                    write_gnp_file, write_read_network_files)
from oracle.dumpio import read_dump  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "gnp_dump")
N, SIDE, SEED = 120, 2.0, 4_000_000
VDW, TUNNEL = 0.00034, 0.0018  # um, as the CNT configurations
GS_MIN = 0.05
OVERLAP_CNT = 2 * 0.005 + TUNNEL          # Input_Reader.cpp:1035 (2 r_max + tunnelling cutoff)
OVERLAP_GNP = GS_MIN / np.sqrt(8.0)       # Input_Reader.cpp:1368
CNT_N, CNT_SEED = 400, SEED + 2


def cnt_config() -> NetworkConfig:
    return NetworkConfig(side=SIDE, n_cnts=CNT_N, seed=CNT_SEED, vdw=VDW, tunnel=TUNNEL)


def hybrid_network(directory: str) -> dict:
    """Write the seeded CNT network's Read_Network files into `directory` and
    return it as upstream reads them (point numbers in CNT order)."""
    cfg = cnt_config()
    write_read_network_files(directory, generate_cnt_network(cfg), cfg)
    return read_network_files(directory).arrays()


def net_hash(a: dict) -> str:
    h = hashlib.sha256()
    for k in ("x", "y", "z", "flag", "structure_ptr", "structure_idx", "radii"):
        h.update(np.ascontiguousarray(a[k]).tobytes())
    return h.hexdigest()


def arr_hash(*arrs) -> str:
    h = hashlib.sha256()
    for a in arrs:
        h.update(np.ascontiguousarray(np.asarray(a, dtype=np.int64)).tobytes())
    return h.hexdigest()


def queries(gnps: dict, per: int, seed: int) -> np.ndarray:
    """Points around each GNP at three scales (far, near the faces, inside): x, y, z, GNP index."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(len(gnps["l"])):
        c, l = gnps["center"][i], gnps["l"][i]
        for _ in range(per):
            out.append([*(c + rng.uniform(-0.7 * l, 0.7 * l, 3) * rng.choice([1.0, 0.02, 0.005])), float(i)])
    return np.array(out)


def dump(gnps: dict, side: float, directory: str, q: np.ndarray) -> dict:
    write_gnp_file(directory, gnps)
    with open(os.path.join(directory, "gnp_queries.dat"), "wb") as f:
        f.write(np.int32(len(q)).tobytes())
        f.write(q.astype("<f8").tobytes())
    with open(os.path.join(directory, "sample_geom.csv"), "w") as f:
        f.write(f"0,0,0\n{side!r},{side!r},{side!r}\n")
    out = os.path.join(directory, "gnp.bin")
    subprocess.run([REF, directory, out, repr(VDW), repr(TUNNEL), repr(GS_MIN), repr(OVERLAP_CNT), repr(float(OVERLAP_GNP))],
                   check=True, capture_output=True, timeout=600)
    return read_dump(out)


def main():
    g = generate_gnps(N, SIDE, SEED)
    q = queries(g, 20, SEED + 1)
    with tempfile.TemporaryDirectory() as d:
        net = hybrid_network(d)
        z = dump(g, SIDE, d, q)
    sd_sha = arr_hash(z.pop("mix_sd_cnt_ptr"), z.pop("mix_sd_cnt_idx"))
    z.pop("ref_seconds", None)  # timings, not results
    np.savez_compressed(os.path.join(HERE, f"gnp_{N}_s{SEED}.npz"),
                        in_l=g["l"], in_t=g["t"], in_theta=g["theta"], in_phi=g["phi"], in_center=g["center"], in_queries=q,
                        meta=np.array([N, SIDE, SEED, VDW, TUNNEL, GS_MIN, OVERLAP_CNT, OVERLAP_GNP]),
                        cnt_meta=np.array([CNT_N, CNT_SEED]), cnt_sha256=np.array(net_hash(net)), mix_sd_sha256=np.array(sd_sha),
                        **{"ref_" + k: v for k, v in z.items()})
    print(f"{N} GNPs, {len(z['pair_a'])} candidate pairs, {int(z['pair_penetrating'].sum())} interpenetrating, "
          f"{int((z['pair_dist'] <= TUNNEL).sum())} within the tunnelling cutoff; {len(net['x'])} CNT points, "
          f"{len(z['mix_point'])} CNT-GNP contacts")


# A sparser hybrid sample whose labels stay apart: 30 GNPs (side 0.3-0.5 um) and 250 CNTs in 2 um
SPARSE_N, SPARSE_SEED, SPARSE_CNTS, SPARSE_CNT_SEED = 30, 4_100_002, 250, 4_100_001


def sparse_config() -> NetworkConfig:
    return NetworkConfig(side=SIDE, n_cnts=SPARSE_CNTS, seed=SPARSE_CNT_SEED, vdw=VDW, tunnel=TUNNEL)


def sparse_network(directory: str) -> dict:
    cfg = sparse_config()
    write_read_network_files(directory, generate_cnt_network(cfg), cfg)
    return read_network_files(directory).arrays()


def main_labels():
    """tests/golden/gnp_hybrid_labels.npz: upstream's CNT, GNP and mixed labels of
    the sparse hybrid sample (Make_cnt_clusters, Make_gnp_clusters,
    Make_mixed_clusters) with its CNT-GNP contacts, the GNP point structures and
    junctions after Add_gnp_junction and after Compress_mixed_contacts."""
    g = generate_gnps(SPARSE_N, SIDE, SPARSE_SEED, l_range=(0.3, 0.5))
    with tempfile.TemporaryDirectory() as d:
        net = sparse_network(d)
        write_gnp_file(d, g)
        with open(os.path.join(d, "sample_geom.csv"), "w") as f:
            f.write(f"0,0,0\n{SIDE!r},{SIDE!r},{SIDE!r}\n")
        out = os.path.join(d, "gnp.bin")
        subprocess.run([REF, d, out, repr(VDW), repr(TUNNEL), repr(GS_MIN), repr(OVERLAP_CNT), repr(float(OVERLAP_GNP))],
                       check=True, capture_output=True, timeout=600)
        z = read_dump(out)
    keep = ("gnp_vertices", "gnp_planes", "lab_cnt", "lab_gnp", "lab_counts", "mixlab_cnt", "mixlab_gnp", "mixlab_count", "mix_point", "mix_gnp",
            "mix_index", "gnpjn_points", "gnpjn_structure_ptr", "gnpjn_structure_idx", "junctions_gnp", "junctions_gnp_dist", "mixjn_points",
            "mixjn_structure_ptr", "mixjn_structure_idx", "junctions_mixed", "junctions_mixed_dist", "gnp_rotation", "gnp_center", "gnp_lt",
            "tri_ptr", "tri_edges")
    np.savez_compressed(os.path.join(HERE, "gnp_hybrid_labels.npz"), in_l=g["l"], in_t=g["t"], in_theta=g["theta"], in_phi=g["phi"],
                        in_center=g["center"], meta=np.array([SPARSE_N, SIDE, SPARSE_SEED, VDW, TUNNEL, GS_MIN, OVERLAP_CNT, OVERLAP_GNP]),
                        cnt_meta=np.array([SPARSE_CNTS, SPARSE_CNT_SEED]), cnt_sha256=np.array(net_hash(net)),
                        **{"ref_" + k: z[k] for k in keep})
    print(f"sparse hybrid: {int(z['lab_counts'][0])} CNT labels, {int(z['lab_counts'][1])} with the GNPs, "
          f"{int(z['mixlab_count'][0])} mixed clusters, {len(z['mix_point'])} CNT-GNP contacts")


# Window extraction cases: (GNPs, sample side, seed, window side)
WINDOW_CASES = [(120, 2.0, SEED, 1.5), (300, 3.0, 4_300_001, 2.2)]


def main_windows():
    """tests/golden/gnp_windows.npz: upstream's GNP window extraction
    (Fill_gnps_inside) for centred windows smaller than the sample."""
    out = {}
    for k, (n, side, seed, ws) in enumerate(WINDOW_CASES):
        g = generate_gnps(n, side, seed)
        with tempfile.TemporaryDirectory() as d:
            write_gnp_file(d, g)
            with open(os.path.join(d, "sample_geom.csv"), "w") as f:
                f.write(f"0,0,0\n{side!r},{side!r},{side!r}\n")
            subprocess.run([REF, d, os.path.join(d, "g.bin"), repr(VDW), repr(TUNNEL), repr(GS_MIN), repr(OVERLAP_CNT), repr(float(OVERLAP_GNP)),
                            repr(float(ws))], check=True, capture_output=True, timeout=600)
            z = read_dump(os.path.join(d, "g.bin"))
        for key in ("l", "t", "theta", "phi", "center"):
            out[f"c{k}_in_{key}"] = g[key]
        out[f"c{k}_meta"] = np.array([n, side, seed, ws])
        for key in ("win_inside", "win_bgnp_ptr", "win_bgnp_idx", "win_bpts_ptr", "win_bpts_idx", "win_structure_ptr", "win_structure_idx",
                    "win_points", "win_box", "win_volume"):
            out[f"c{k}_ref_{key}"] = z[key]
        print(f"window case {k}: {n} GNPs in {side} um, window {ws} um: {len(z['win_inside'])} inside, {len(z['win_points']) // 3} boundary points")
    np.savez_compressed(os.path.join(HERE, "gnp_windows.npz"), **out)


def main_flow():
    """tests/golden/gnp_hybrid_flow.npz: upstream's own stages for GNP_CNT_mix
    (window extraction, contact grid, Determine_clusters_and_percolation) on the
    two hybrid samples: cnts/gnps inside, boundary lists, percolated clusters,
    isolated particles, families and junction groups (flow_* records), and the
    resistances of Electrical_analysis along x (flow_resistances), the
    end-to-end result of the hybrid configuration's path."""
    out = {}
    samples = (("m", hybrid_network, generate_gnps(N, SIDE, SEED)),
               ("s", sparse_network, generate_gnps(SPARSE_N, SIDE, SPARSE_SEED, l_range=(0.3, 0.5))))
    for tag, network, g in samples:
        with tempfile.TemporaryDirectory() as d:
            network(d)
            write_gnp_file(d, g)
            subprocess.run([REF, d, os.path.join(d, "g.bin"), repr(VDW), repr(TUNNEL), repr(GS_MIN), repr(OVERLAP_CNT), repr(float(OVERLAP_GNP)),
                            "-1", "flow", repr(cnt_config().step), "electrical"], check=True, capture_output=True, timeout=1200)
            z = read_dump(os.path.join(d, "g.bin"))
        for k, v in z.items():
            if k.startswith("flow_") and k not in ("flow_points_gnp", "flow_structure_gnp_ptr", "flow_structure_gnp_idx"):
                out[f"{tag}_{k}"] = v
        print(f"flow {tag}: family {list(z['flow_family'])}, {len(z['flow_cnts_inside'])} CNTs and {len(z['flow_gnps_inside'])} GNPs inside, "
              f"R_x {z['flow_resistances'][0]:.6g} Ohm")
    np.savez_compressed(os.path.join(HERE, "gnp_hybrid_flow.npz"), **out)


def main_electrical():
    """tests/golden/gnp_hybrid_electrical.npz: upstream's electrical stage of both
    hybrid samples, replayed by the harness through the public members of
    Electrical_analysis, Direct_Electrifying and Backbone_Network in
    Perform_analysis_on_clusters' order (e_* records): per percolated cluster
    the unit-resistor system (node maps of CNT and GNP points, the SSS matrix,
    right-hand side, voltages, the GNP triangulations and the GNP points with a
    CNT radius), the zero current, the backbone (CNT elements, GNP point lists,
    clusters and junction groups after it), and per percolated direction the
    real-resistor system and its resistor; the GNP points, point lists and
    boundary points the stage starts from, and the volume members at the end."""
    out = {}
    samples = (("m", hybrid_network, generate_gnps(N, SIDE, SEED)),
               ("s", sparse_network, generate_gnps(SPARSE_N, SIDE, SPARSE_SEED, l_range=(0.3, 0.5))))
    for tag, network, g in samples:
        with tempfile.TemporaryDirectory() as d:
            network(d)
            write_gnp_file(d, g)
            subprocess.run([REF, d, os.path.join(d, "g.bin"), repr(VDW), repr(TUNNEL), repr(GS_MIN), repr(OVERLAP_CNT), repr(float(OVERLAP_GNP)),
                            "-1", "flow", repr(cnt_config().step), "electrical"], check=True, capture_output=True, timeout=1200)
            z = read_dump(os.path.join(d, "g.bin"))
        for k, v in z.items():
            if k.startswith("e_") or k in ("flow_points_gnp", "flow_structure_gnp_ptr", "flow_structure_gnp_idx", "flow_resistances"):
                out[f"{tag}_{k}"] = v
        print(f"electrical {tag}: {sum(1 for k in z if k.endswith('_u_nodes'))} clusters, R_x {z['flow_resistances'][0]:.6g} Ohm")
    np.savez_compressed(os.path.join(HERE, "gnp_hybrid_electrical.npz"), **out)


def main_resistors():
    """tests/golden/gnp_resistors.npz: upstream's Calculate_resistance_gnp on the
    triangulation edges of the 120-GNP fixture's GNPs (radii t/2, or the CNT
    radius at a mixed-junction point, as Fill_2d_matrices_gnp takes them; GNP
    in-plane 1e-4 and through-plane 1 Ohm um) and one edge of coincident points."""
    z = dict(np.load(os.path.join(HERE, f"gnp_{N}_s{SEED}.npz")))
    pts = z["ref_mixjn_points"].reshape(-1, 3)
    n_before_mixed = len(z["ref_gnpjn_points"]) // 3
    t = z["ref_gnp_lt"].reshape(-1, 2)[:, 1]
    tp, te = z["ref_tri_ptr"], z["ref_tri_edges"].reshape(-1, 2)
    cases = []
    for g in range(len(tp) - 1):
        for v1, v2 in te[tp[g]:tp[g + 1]]:
            r = [0.005 if v >= n_before_mixed else t[g] / 2 for v in (v1, v2)]
            cases.append([*pts[v1], *pts[v2], r[0], r[1], 1e-4, 1.0])
    cases.append([*pts[0], *pts[0], 0.005, 0.005, 1e-4, 1.0])  # coincident points: upstream fails
    cases = np.array(cases)
    g = generate_gnps(N, SIDE, SEED)
    with tempfile.TemporaryDirectory() as d:
        write_gnp_file(d, g)
        with open(os.path.join(d, "sample_geom.csv"), "w") as f:
            f.write(f"0,0,0\n{SIDE!r},{SIDE!r},{SIDE!r}\n")
        with open(os.path.join(d, "gnp_resistor_cases.dat"), "wb") as f:
            f.write(np.int32(len(cases)).tobytes() + cases.astype("<f8").tobytes())
        subprocess.run([REF, d, os.path.join(d, "g.bin"), repr(VDW), repr(TUNNEL)], check=True, capture_output=True, timeout=600)
        r = read_dump(os.path.join(d, "g.bin"))["gnp_resistances"]
    np.savez_compressed(os.path.join(HERE, "gnp_resistors.npz"), cases=cases, ref_resistance=r)
    print(f"GNP resistors: {len(cases)} cases")


if __name__ == "__main__":
    main()
    main_labels()
    main_windows()
    main_flow()
    main_electrical()
    main_resistors()
