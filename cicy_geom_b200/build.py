"""Build libcicy_b200.so in-tree with nvcc for sm_100a.

Every CUDA and C++ source under csrc/ is compiled to an object in
csrc/_build/ (one nvcc process per file, in parallel, skipped when the object
is newer than its source and the shared headers) and linked into
cicy_geom_b200/libcicy_b200.so, which travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(CSRC, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libcicy_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3,-ffp-contract=off", f"-I{INCLUDE}", f"-I{CSRC}"]
# FP64 contact geometry and Kirchhoff assembly must round like the upstream host
# code: no fused multiply-add contraction in the sources that reproduce upstream
# arithmetic bit for bit.  The iterative solvers (their results are checked
# against an FP64 direct solve within a tolerance, not bit for bit) keep FMA.
CUDA_ONLY = ["-Xptxas", "-O3"]
SOLVER_SOURCES = {"solver.cu", "solver_cluster.cu", "solver_mg.cu", "spmv.cu", "batch.cu", "learned.cu", "noalloc.cu"}


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def _headers_mtime() -> float:
    m = os.path.getmtime(os.path.join(INCLUDE, "cicy_b200.h"))
    for f in os.listdir(CSRC):
        if f.endswith((".h", ".cuh")):
            m = max(m, os.path.getmtime(os.path.join(CSRC, f)))
    return m


def _compile(src: str, force: bool, hm: float, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hm):
        return obj
    cmd = [_nvcc(), *ARCH, *COMMON]
    if src.endswith(".cu"):
        cmd += CUDA_ONLY + ([] if os.path.basename(src) in SOLVER_SOURCES else ["--fmad=false"])
    else:
        cmd += ["-x", "c++"]
    if verbose and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    cmd += ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stderr or r.stdout):
        sys.stderr.write(r.stdout + r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hm = _headers_mtime()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hm, verbose), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
