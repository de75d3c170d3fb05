"""Generate tests/golden/gnp_junction_cases.npz from the upstream program.

Hand-placed GNP pairs, one pair per 3 um cell of a 12 um sample, each separated
by about 1 nm (within the 1.8 nm tunnelling cutoff) in a configuration that
makes upstream's junction step (Find_junction_points_for_gnps) take one case:
face on face (partial overlap, one face inside the other, side faces), an edge
on a face (inside it and crossing its boundary), parallel edges, vertex on
vertex, vertex on edge, vertex on face, and the face-inside
case with the larger GNP first, where upstream reports an error.  Runs
oracle/_ref/gnp_dump (upstream objects compiled in place by oracle/Makefile)
and stores the GNPs as upstream reads them, the distance step of every pair
within the cutoff and upstream's junction points (or its failure).

    python tests/golden/make_gnp_junction_golden.py
"""
from __future__ import annotations

import math
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cicy_geom_b200.network import write_gnp_file  # noqa: E402
from oracle.dumpio import read_dump  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "gnp_dump")
SIDE, VDW, TUNNEL, T = 12.0, 0.00034, 0.0018, 0.01
G = 0.001  # gap (um)


def cases():
    """(name, [(l, theta, phi, centre offset from the cell centre)] for GNPs A, B)."""
    th = 0.3  # tilt of B about y (its lowest edge stays along y)
    lb = 0.6
    drop = math.sin(th) * lb / 2 + math.cos(th) * T / 2  # height of B's centre above its lowest edge
    reach = math.cos(th) * lb / 2 - math.sin(th) * T / 2  # x of that edge from B's centre
    ph = 0.2  # rotation of B about z: its bottom corner (-l/2, +l/2) is the leftmost
    corner_x = -math.cos(ph) * lb / 2 - math.sin(ph) * lb / 2
    corner_y = -math.sin(ph) * lb / 2 + math.cos(ph) * lb / 2
    return [
        ("face_face_partial", [(0.8, 0, 0, (0, 0, 0)), (0.8, 0, 0, (0.3, 0.2, T + G))]),
        ("face_inside_small_first", [(0.5, 0, 0, (0.1, 0.05, T + G)), (0.9, 0, 0, (0, 0, 0))]),
        ("face_inside_large_first", [(0.9, 0, 0, (0, 0, 0)), (0.5, 0, 0, (0.1, 0.05, T + G))]),
        ("side_faces", [(0.7, 0, 0, (0, 0, 0)), (0.7, 0, 0, (0.7 + G, 0.1, 0))]),
        ("edge_on_face", [(0.9, 0, 0, (0, 0, 0)), (lb, th, 0, (-reach, 0.0, T / 2 + G + drop))]),
        ("edge_across_face", [(0.9, 0, 0, (0, 0, 0)), (lb, th, 0, (-reach, 0.35, T / 2 + G + drop))]),
        ("parallel_edges", [(0.7, 0, 0, (0, 0, 0)), (0.7, 0, 0, (0.7 + 0.0007, 0.1, T + 0.0007))]),
        ("vertex_vertex", [(0.6, 0, 0, (0, 0, 0)), (0.6, 0, 0, (0.6 + 0.0006, 0.6 + 0.0006, T + 0.0006))]),
        ("vertex_edge", [(0.8, 0, 0, (0, 0, 0)), (lb, 0, ph, (0.4 + 0.0006 - corner_x, 0.1 - corner_y, T + 0.0006))]),
        ("vertex_face", [(0.9, 0, 0, (0, 0, 0)), (0.5, 0.4, 0.7, (0.0, 0.0, 0.0))]),
    ]


def layout():
    g = {"l": [], "t": [], "theta": [], "phi": [], "center": []}
    names = []
    for k, (name, pair) in enumerate(cases()):
        cell = np.array([1.5 + 3.0 * (k % 4), 1.5 + 3.0 * ((k // 4) % 4), 1.5 + 3.0 * (k // 16)]) + np.array([0.0, 0.0, 4.5])
        for l, theta, phi, off in pair:
            g["l"].append(l)
            g["t"].append(T)
            g["theta"].append(theta)
            g["phi"].append(phi)
            g["center"].append(cell + np.asarray(off, dtype=float))
        names.append(name)
    return {k: np.asarray(v, dtype=float) for k, v in g.items()}, names


def place_vertex_face(g):
    """Put B of the vertex_face case (tilted both ways) with its lowest vertex G above A's top face."""
    from cicy_geom_b200.network import read_gnps

    k = layout()[1].index("vertex_face")
    with tempfile.TemporaryDirectory() as d:
        write_gnp_file(d, g)
        V = read_gnps(d)["vertices"]
    a, b = 2 * k, 2 * k + 1
    top = V[a][:, 2].max()
    low = V[b][:, 2].min()
    g["center"][b][2] += top + G - low


def main():
    g, names = layout()
    place_vertex_face(g)
    with tempfile.TemporaryDirectory() as d:
        write_gnp_file(d, g)
        with open(os.path.join(d, "sample_geom.csv"), "w") as f:
            f.write(f"0,0,0\n{SIDE!r},{SIDE!r},{SIDE!r}\n")
        out = os.path.join(d, "gnp.bin")
        subprocess.run([REF, d, out, repr(VDW), repr(TUNNEL)], check=True, capture_output=True, timeout=600)
        z = read_dump(out)
    np.savez_compressed(os.path.join(HERE, "gnp_junction_cases.npz"), in_l=g["l"], in_t=g["t"], in_theta=g["theta"], in_phi=g["phi"],
                        in_center=g["center"], names=np.array(names), meta=np.array([SIDE, VDW, TUNNEL]),
                        **{"ref_" + k: v for k, v in z.items()})
    jp = z["junc_pair"]
    print(f"{len(names)} cases, {len(z['pair_a'])} pairs measured, {len(jp)} within the cutoff, {int(z['junc_ok'].sum())} junctions found")
    for i, p in enumerate(jp):
        print(f"  pair ({z['pair_a'][p]}, {z['pair_b'][p]}) {names[z['pair_a'][p] // 2]}: ok {z['junc_ok'][i]} dist {z['pair_dist'][p]:.6g}")


if __name__ == "__main__":
    main()
