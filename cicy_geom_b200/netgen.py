"""Seeded synthetic CNT networks written to `Read_Network` files without the library.

The same network as `cicy_generate_cnt_network` (csrc/host_network.cpp):
Philox-4x32-10 draws keyed by the seed, one stream per CNT; draw 0 sets the
CNT's length, draws 1-2 its start point, draw 3 its initial direction and draw
3 + k the turn of step k.  Integer arithmetic is exact in numpy, the
floating-point steps are the same IEEE operations in the same order, and the
cosines and sines come from the C library through Python's `math` module (as
the C++ generator's std::cos / std::sin do), so the files are byte-identical
to `write_read_network_files(generate_cnt_network(cfg))`.

This module loads nothing of libcicy_b200.so: it serves processes that must
not map it, such as the benchmark's reference arm, which runs the upstream
program on these files.
"""
from __future__ import annotations

import math
import os

import numpy as np

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
_C2, _C3 = 0x43494359, 0x42323030
_TWO_PI = 6.283185307179586476925286766559
_INV53 = 1.0 / 9007199254740992.0
_cos = np.frompyfunc(math.cos, 1, 1)
_sin = np.frompyfunc(math.sin, 1, 1)


def _philox_uniform2(seed: int, stream, draw):
    """Two uniforms in [0, 1) per (stream, draw), Philox-4x32-10 on counter (stream, draw, C2, C3)."""
    stream = np.asarray(stream, dtype=np.uint32)
    draw = np.broadcast_to(np.asarray(draw, dtype=np.uint32), stream.shape)
    c0, c1 = stream.astype(np.uint32), draw.astype(np.uint32)
    c2 = np.full(stream.shape, _C2, dtype=np.uint32)
    c3 = np.full(stream.shape, _C3, dtype=np.uint32)
    k0, k1 = np.uint32(seed & 0xFFFFFFFF), np.uint32((seed >> 32) & 0xFFFFFFFF)
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = _M0 * c0.astype(np.uint64)
            p1 = _M1 * c2.astype(np.uint64)
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), p0.astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), p1.astype(np.uint32)
            c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
            k0 = np.uint32(k0 + _W0)
            k1 = np.uint32(k1 + _W1)
    a = (c0.astype(np.uint64) << np.uint64(32)) | c1.astype(np.uint64)
    b = (c2.astype(np.uint64) << np.uint64(32)) | c3.astype(np.uint64)
    u0 = (a >> np.uint64(11)).astype(np.float64) * _INV53
    u1 = (b >> np.uint64(11)).astype(np.float64) * _INV53
    return u0, u1


def generate_cnt_arrays(side: float, n_cnts: int, seed: int, step: float = 0.01, len_min: float = 0.5, len_max: float = 1.5,
                        max_turn_deg: float = 10.0):
    """(counts[n_cnts], xyz[n_points, 3]) of the seeded network in a cube of `side` at the origin."""
    ids = np.arange(n_cnts, dtype=np.uint32)
    u0, _ = _philox_uniform2(seed, ids, 0)
    L = len_min + u0 * (len_max - len_min)
    counts = (1 + np.floor(L / step)).astype(np.int64)
    starts = np.concatenate([[0], np.cumsum(counts)])
    xyz = np.empty((int(starts[-1]), 3), dtype=np.float64)
    max_turn = math.radians(max_turn_deg)
    a0, a1 = _philox_uniform2(seed, ids, 1)
    a2, _ = _philox_uniform2(seed, ids, 2)
    px, py, pz = 0.0 + a0 * side, 0.0 + a1 * side, 0.0 + a2 * side
    v0, v1 = _philox_uniform2(seed, ids, 3)
    ct = 2.0 * v0 - 1.0
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    ph = _TWO_PI * v1
    dx = st * _cos(ph).astype(np.float64)
    dy = st * _sin(ph).astype(np.float64)
    dz = ct.copy()
    xyz[starts[:-1], 0], xyz[starts[:-1], 1], xyz[starts[:-1], 2] = px, py, pz
    act = np.arange(n_cnts)
    for k in range(1, int(counts.max(initial=1))):
        keep = counts[act] > k
        act, px, py, pz, dx, dy, dz = act[keep], px[keep], py[keep], pz[keep], dx[keep], dy[keep], dz[keep]
        if len(act) == 0:
            break
        w0, w1 = _philox_uniform2(seed, act.astype(np.uint32), 3 + k)
        th = w0 * max_turn
        az = _TWO_PI * w1
        # orthonormal frame (e1, e2) perpendicular to d: e1 = a x d with a = x or y
        ax = np.where(np.abs(dx) < 0.9, 1.0, 0.0)
        ay = 1.0 - ax
        e1x = ay * dz - 0.0 * dy
        e1y = 0.0 * dx - ax * dz
        e1z = ax * dy - ay * dx
        n1 = np.sqrt(e1x * e1x + e1y * e1y + e1z * e1z)
        e1x, e1y, e1z = e1x / n1, e1y / n1, e1z / n1
        e2x = dy * e1z - dz * e1y
        e2y = dz * e1x - dx * e1z
        e2z = dx * e1y - dy * e1x
        c, s = _cos(th).astype(np.float64), _sin(th).astype(np.float64)
        ca, sa = _cos(az).astype(np.float64), _sin(az).astype(np.float64)
        nx = c * dx + s * (ca * e1x + sa * e2x)
        ny = c * dy + s * (ca * e1y + sa * e2y)
        nz = c * dz + s * (ca * e1z + sa * e2z)
        nn = np.sqrt(nx * nx + ny * ny + nz * nz)
        dx, dy, dz = nx / nn, ny / nn, nz / nn
        px = px + step * dx
        py = py + step * dy
        pz = pz + step * dz
        row = starts[act] + k
        xyz[row, 0], xyz[row, 1], xyz[row, 2] = px, py, pz
    return counts, xyz


def write_network_files(directory: str, cfg) -> None:
    """The `Read_Network` binary files and input.dat of `cfg` (a NetworkConfig), as
    network.write_read_network_files writes them for the library's generator."""
    from .network import input_dat

    os.makedirs(directory, exist_ok=True)
    counts, xyz = generate_cnt_arrays(cfg.side, cfg.n_cnts, cfg.seed, cfg.step, cfg.len_min, cfg.len_max, cfg.max_turn_deg)
    rec = np.zeros(len(counts), dtype=np.dtype([("np", "<i4"), ("r", "<f8")], align=False))
    rec["np"] = counts.astype(np.int32)
    rec["r"] = cfg.radius
    with open(os.path.join(directory, "cnt_struct.dat"), "wb") as f:
        f.write(np.int32(len(counts)).tobytes())
        f.write(rec.tobytes())
    with open(os.path.join(directory, "cnt_coordinates.dat"), "wb") as f:
        f.write(np.ascontiguousarray(xyz, dtype="<f8").tobytes())
    s = cfg.side
    with open(os.path.join(directory, "sample_geom.csv"), "w") as f:
        f.write(f"0,0,0\n{s!r},{s!r},{s!r}\n")
    with open(os.path.join(directory, "input.dat"), "w") as f:
        f.write(input_dat(cfg, "dat"))
