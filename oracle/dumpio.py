"""Reader of the named-array dumps written by oracle/_ref/ref_dump (test infrastructure).

Layout per record: u32 name length, name bytes, u8 type ('i' int32, 'l' int64,
'd' float64), u64 count, payload.
"""
from __future__ import annotations

import numpy as np

_DT = {b"i": np.int32, b"l": np.int64, b"d": np.float64}


def read_dump(path: str) -> dict:
    out = {}
    with open(path, "rb") as f:
        buf = f.read()
    o = 0
    while o < len(buf):
        nl = int(np.frombuffer(buf, np.uint32, 1, o)[0]); o += 4
        name = buf[o:o + nl].decode(); o += nl
        t = buf[o:o + 1]; o += 1
        cnt = int(np.frombuffer(buf, np.uint64, 1, o)[0]); o += 8
        dt = _DT[t]
        out[name] = np.frombuffer(buf, dt, cnt, o).copy(); o += cnt * np.dtype(dt).itemsize
    return out


def csr(d: dict, name: str):
    """List of arrays from a `<name>_ptr` / `<name>_idx` pair."""
    p, i = d[name + "_ptr"], d[name + "_idx"]
    return [i[p[k]:p[k + 1]] for k in range(len(p) - 1)]
