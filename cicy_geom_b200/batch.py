"""Batched Monte-Carlo solves through the C ABI (cicy_batch_*).

Realisations are drawn like the Monte-Carlo sweep (per-sample seed, cube side
and CNT volume fraction; N_c = round(phi L^3 / (pi r^2 * 1 um)) for the 1 um
mean CNT length), each run through the device path to its real-resistor
system, and all systems are then solved together by one persistent,
graph-captured launch.  PyTorch only holds the device arrays.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi


def monte_carlo_configs(count: int, seed0: int = 3_000_000, side=(2.0, 5.0), fraction=(0.005, 0.03), radius=0.005):
    from .network import NetworkConfig

    rng = np.random.default_rng(seed0)
    out = []
    for k in range(count):
        L = float(rng.uniform(*side))
        phi = float(rng.uniform(*fraction))
        n = int(round(phi * L ** 3 / (math.pi * radius ** 2 * 1.0)))
        out.append(NetworkConfig(side=L, n_cnts=max(n, 1), seed=seed0 + k, tolerance=1e-8, tolerance_unit=1e-12))
    return out


def realisation_systems(configs, device: int = 0, preconditioner: int = 3, construction: str = "device"):
    """Run each realisation through the device path; keep its real-resistor systems.

    construction "device": each network is generated and window-trimmed on the
    device (Context.generate_network); "host": generated and trimmed on the host,
    then uploaded.  One context serves every realisation.

    Returns (systems, info): systems are dicts with the full CSR (host), chains,
    right-hand side, initial guess and the per-network solver's solution and
    time; info counts the realisations that do not percolate (their resistance
    is the matrix resistance, no system to solve) and holds each realisation's
    device time of the whole hot path by seed ("device_seconds")."""
    from .device import Context
    from .learned import full_csr
    from .network import generate_cnt_network

    systems, info = [], {"realisations": len(configs), "percolating": 0, "not_percolating": 0, "rejected": 0}
    device_seconds = {}  # seed -> device time of the whole hot path (cicy_result.stage_seconds[5])
    if construction not in ("device", "host"):
        raise ValueError(f"construction must be 'device' or 'host', not {construction!r}")
    ctx = Context(device)
    ctx.set_solver(preconditioner=preconditioner)
    for cfg in configs:
        try:
            if construction == "device":
                ctx.generate_network(cfg)
            else:
                ctx.upload(generate_cnt_network(cfg).extract_window(cfg))
            r = ctx.network_to_conductance(cfg.params())
        except _abi.CicyError:
            info["rejected"] += 1
            continue
        device_seconds[cfg.seed] = float(r.stage_seconds[5])
        real = [i for i in range(r.n_solves) if r.solves[i].pass_ >= 0]
        if not real:
            info["not_percolating"] += 1
        else:
            info["percolating"] += 1
        for i in real:
            S = ctx.system(i)
            if len(S["diag"]) == 0:
                continue
            st, ln = ctx.chains(i)
            keep = ln > 0  # a CNT whose element nodes are all prescribed has an empty chain
            st, ln = st[keep], ln[keep]
            systems.append({"A": full_csr(S), "b": S["b"], "x0": S["x0"], "chain_start": st, "chain_len": ln,
                            "x_ref": S["voltages"][S["reserved"]:], "seconds_ref": r.solves[i].seconds,
                            "iterations_ref": r.solves[i].iterations, "seed": cfg.seed})
    ctx.close()
    info["construction"] = construction
    info["device_seconds"] = device_seconds
    return systems, info


METHODS = ["cta_pcg", "cluster_multigrid", "sequential_grid"]
PRECONDITIONERS = {"jacobi": 0, "learned": 1, "chain": 2}


def edge_weights(tensors, params, device: int, stream) -> list:
    """Learned coupling weights of each system (cicy_gnn_forward; one FP32 value per CSR entry)."""
    import torch

    L = _abi.lib()
    dev = torch.device(f"cuda:{device}")
    P = torch.tensor(np.asarray(params, np.float32), device=dev)
    gnn = C.c_void_p()
    _abi.check(L.cicy_gnn_create(C.byref(gnn), device), "cicy_gnn_create")
    out = []
    try:
        for t in tensors:
            n, nnz = t["rp"].numel() - 1, t["ci"].numel()
            d = _abi.GnnSystem(n, nnz, t["rp"].data_ptr(), t["ci"].data_ptr(), t["v"].data_ptr(), t["cs"].numel(), t["cs"].data_ptr(),
                               t["cl"].data_ptr())
            w = torch.empty(nnz, dtype=torch.float32, device=dev)
            _abi.check(L.cicy_gnn_set_system(gnn, C.byref(d), C.c_void_p(stream)), "cicy_gnn_set_system")
            _abi.check(L.cicy_gnn_forward(gnn, C.c_void_p(P.data_ptr()), C.c_void_p(w.data_ptr()), C.c_void_p(stream)), "cicy_gnn_forward")
            out.append(w)
        torch.cuda.synchronize(dev)
    finally:
        L.cicy_gnn_destroy(gnn)
    return out


class BatchSolver:
    """The systems in device memory and one cicy_batch over them.

    learned: None, True (the shipped parameters) or a parameter vector; when
    given, the graph network's coupling weights of every system are computed
    once here so the learned preconditioner can be selected."""

    def __init__(self, systems, tol: float = 1e-8, precision: int = 0, max_iter_factor: int = 300, device: int = 0, learned=None):
        import torch

        self.dev = torch.device(f"cuda:{device}")
        self._keep = []
        descs = (_abi.BatchSystem * len(systems))()
        self.x = []
        tensors = []
        for s in systems:
            A = s["A"]
            tensors.append({
                "rp": torch.tensor(A.indptr.astype(np.int32), device=self.dev),
                "ci": torch.tensor(A.indices.astype(np.int32), device=self.dev),
                "v": torch.tensor(A.data, dtype=torch.float64, device=self.dev),
                "cs": torch.tensor(np.asarray(s["chain_start"], np.int32), device=self.dev),
                "cl": torch.tensor(np.asarray(s["chain_len"], np.int32), device=self.dev),
            })
        self.gnn_seconds = 0.0
        if learned is not None:
            import time

            from .learned import default_params

            params = default_params() if learned is True else learned
            t0 = time.perf_counter()
            ws = edge_weights(tensors, params, device, torch.cuda.current_stream(self.dev).cuda_stream)
            self.gnn_seconds = time.perf_counter() - t0
            for t, w in zip(tensors, ws):
                t["ew"] = w
        for k, s in enumerate(systems):
            A = s["A"]
            t = tensors[k]
            t["b"] = torch.tensor(s["b"], dtype=torch.float64, device=self.dev)
            t["x0"] = torch.tensor(s["x0"], dtype=torch.float64, device=self.dev)
            t["x"] = torch.zeros(A.shape[0], dtype=torch.float64, device=self.dev)
            self._keep.append(t)
            self.x.append(t["x"])
            descs[k] = _abi.BatchSystem(A.shape[0], A.nnz, t["rp"].data_ptr(), t["ci"].data_ptr(), t["v"].data_ptr(), t["b"].data_ptr(),
                                        t["x0"].data_ptr(), t["x"].data_ptr(), len(s["chain_start"]), t["cs"].data_ptr(), t["cl"].data_ptr(),
                                        t["ew"].data_ptr() if "ew" in t else None)
        torch.cuda.synchronize(self.dev)
        self.count = len(systems)
        self.h = C.c_void_p()
        _abi.check(_abi.lib().cicy_batch_create(C.byref(self.h), device, descs, self.count, tol, max_iter_factor, precision),
                   "cicy_batch_create")

    def enable_multigrid(self) -> float:
        """Build the per-system multigrid hierarchies; returns the setup time (s)."""
        t = C.c_double()
        _abi.check(_abi.lib().cicy_batch_enable_multigrid(self.h, C.byref(t)), "cicy_batch_enable_multigrid")
        return t.value

    def set_method(self, method):
        """0 / "cta_pcg", 1 / "cluster_multigrid", 2 / "sequential_grid"."""
        m = METHODS.index(method) if isinstance(method, str) else int(method)
        _abi.check(_abi.lib().cicy_batch_set_method(self.h, m), "cicy_batch_set_method")

    def set_solver(self, preconditioner, precision: int = 0):
        """Preconditioner of methods 0 and 2 ("jacobi", "learned", "chain" or its CICY_PRECOND value); precision 0 FP64, 1 mixed."""
        pk = PRECONDITIONERS[preconditioner] if isinstance(preconditioner, str) else int(preconditioner)
        _abi.check(_abi.lib().cicy_batch_set_solver(self.h, pk, precision), "cicy_batch_set_solver")

    def autotune(self):
        m, t, c, sp, s = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        _abi.check(_abi.lib().cicy_batch_autotune(self.h, C.byref(m), C.byref(t), C.byref(c), C.byref(sp), C.byref(s)),
                   "cicy_batch_autotune")
        return {"method": METHODS[m.value], "threads": t.value, "ctas_per_sm": c.value, "cluster_split_rows": sp.value,
                "seconds": s.value}

    def set_split(self, rows: int):
        """Method 0: systems of at least `rows` rows run on one 16-CTA cluster each (0: none)."""
        _abi.check(_abi.lib().cicy_batch_set_split(self.h, rows), "cicy_batch_set_split")

    def set_shape(self, threads: int, ctas_per_sm: int):
        _abi.check(_abi.lib().cicy_batch_set_shape(self.h, threads, ctas_per_sm), "cicy_batch_set_shape")

    def solve(self) -> float:
        s = C.c_double()
        _abi.check(_abi.lib().cicy_batch_solve(self.h, C.byref(s)), "cicy_batch_solve")
        return s.value

    def results(self):
        it = np.zeros(self.count, np.int64)
        rel = np.zeros(self.count)
        fl = np.zeros(self.count, np.int32)
        _abi.check(_abi.lib().cicy_batch_results(self.h, it.ctypes.data_as(_abi.i64p), rel.ctypes.data_as(_abi.f64p),
                                                 fl.ctypes.data_as(_abi.i32p)), "cicy_batch_results")
        return it, rel, fl

    def solutions(self):
        return [x.cpu().numpy() for x in self.x]

    def close(self):
        if self.h:
            _abi.lib().cicy_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def main(argv=None):
    """Seeded Monte-Carlo realisations solved by one batched call; prints one JSON line.

    python -m cicy_geom_b200.batch --count 32 --precond learned --precision 1"""
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--count", type=int, default=32)
    ap.add_argument("--seed0", type=int, default=3_000_000)
    ap.add_argument("--precond", default="learned", choices=list(PRECONDITIONERS) + ["multigrid"])
    ap.add_argument("--precision", type=int, default=1)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--threads", type=int, default=1024)
    ap.add_argument("--ctas-per-sm", type=int, default=2)
    ap.add_argument("--split", type=int, default=0, help="systems of at least this many rows on 16-CTA clusters (0: none)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    t0 = time.time()
    systems, info = realisation_systems(monte_carlo_configs(a.count, seed0=a.seed0), device=a.device)
    prep = time.time() - t0
    bs = BatchSolver(systems, tol=a.tol, device=a.device, learned=True if a.precond == "learned" else None)
    if a.precond == "multigrid":
        bs.enable_multigrid()
        bs.set_method(1)
    else:
        bs.set_solver(a.precond, a.precision)
        bs.set_shape(a.threads, a.ctas_per_sm)
        bs.set_split(a.split)
    times = [bs.solve() for _ in range(a.reps)]
    it, rel, fl = bs.results()
    bs.close()
    print(json.dumps({**info, "systems": len(systems), "unknowns_total": int(sum(s["A"].shape[0] for s in systems)),
                      "precond": a.precond, "precision": a.precision, "seconds": min(times), "iterations_total": int(it.sum()),
                      "iterations_max": int(it.max()), "converged": int((fl == 1).sum()), "max_rel_residual": float(rel.max()),
                      "prep_seconds": prep}))


if __name__ == "__main__":
    main()
