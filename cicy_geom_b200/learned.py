"""Training of the learned preconditioner on the GPU, with the library's own
forward and backward kernels (cicy_gnn_* in include/cicy_b200.h).

The training data are the DEA systems this library assembles: seeded CNT
networks drawn like the Monte-Carlo realisations (cube side and CNT volume
fraction per sample), each network run through the device path with the
chain preconditioner, and every real-resistor system (full symmetric CSR plus
its CNT chains) kept with its solution.  Probe vectors per step: the initial
error x* - x0 of the solve and random vectors smoothed by 20 damped chain
block-Jacobi sweeps (the modes the blocks leave behind).  PyTorch only holds
device memory and draws the random probes.

  python -m cicy_geom_b200.learned --out cicy_geom_b200/learned_params.f32
"""
from __future__ import annotations

import argparse
import ctypes as C
import math
import os

import numpy as np

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
PARAMS_PATH = os.path.join(HERE, "learned_params.f32")
# the same network trained on 2,000 real-resistor Laplacians of the Monte-Carlo generator
# (python -m cicy_geom_b200.learned --monte-carlo 2000 --steps 4000 --out <this file>)
MC_PARAMS_PATH = os.path.join(HERE, "learned_params_mc2000.f32")
WIDTH, LAYERS = 32, 3


def param_count() -> int:
    return int(_abi.lib().cicy_gnn_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """Initial parameters (the flat layout of cicy_gnn_param_count): small random
    weights and an edge output that starts every weight at 0.8."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, 0.5, 2 * WIDTH), np.full(WIDTH, 0.1)]
    for _ in range(LAYERS):
        parts += [rng.normal(0, 1 / math.sqrt(WIDTH), WIDTH * WIDTH), rng.normal(0, 0.5 / math.sqrt(WIDTH), WIDTH * WIDTH),
                  np.zeros(WIDTH), np.array([0.5, 0.0, 0.0])]
    parts += [np.zeros(WIDTH), np.array([0.0, math.log(0.8 / 0.2)])]
    p = np.concatenate(parts).astype(np.float32)
    assert len(p) == param_count()
    return p


def default_params() -> np.ndarray:
    """The trained parameters shipped with the package."""
    if not os.path.exists(PARAMS_PATH):
        raise RuntimeError(f"{PARAMS_PATH} is missing: train it with `python -m cicy_geom_b200.learned`")
    p = np.fromfile(PARAMS_PATH, dtype=np.float32)
    if len(p) != param_count():
        raise RuntimeError(f"{PARAMS_PATH}: {len(p)} parameters, the library expects {param_count()}")
    return p


def monte_carlo_params() -> np.ndarray:
    """The parameters trained on 2,000 Monte-Carlo Laplacians (MC_PARAMS_PATH)."""
    p = np.fromfile(MC_PARAMS_PATH, dtype=np.float32)
    if len(p) != param_count():
        raise RuntimeError(f"{MC_PARAMS_PATH}: {len(p)} parameters, the library expects {param_count()}")
    return p


def full_csr(S: dict):
    """Full symmetric CSR (columns ascending, diagonal included) of a system from Context.system()."""
    import scipy.sparse as sp

    n = len(S["diag"])
    L = sp.csr_matrix((S["values"], S["col_ind"], S["row_ptr"]), shape=(n, n))
    A = (L + L.T + sp.diags(S["diag"])).tocsr()
    A.sort_indices()
    return A


def collect_systems(networks, device: int = 0, real_only: bool = True, ctx=None, preconditioner: int = 2):
    """Solve each (NetworkConfig, window network) (chain preconditioner by default) and keep its
    DEA systems; with `ctx`, every network goes through that one context."""
    from .device import Context

    out = []
    own = ctx is None
    for cfg, net in networks:
        if own:
            ctx = Context(device)
        ctx.set_solver(preconditioner=preconditioner)
        ctx.upload(net)
        try:
            r = ctx.network_to_conductance(cfg.params())
        except _abi.CicyError:  # networks upstream rejects too (e.g. a zero stiffness diagonal) are skipped
            if own:
                ctx.close()
            continue
        for i in range(r.n_solves):
            if real_only and r.solves[i].pass_ < 0:
                continue
            S = ctx.system(i)
            if len(S["diag"]) < 64:
                continue
            A = full_csr(S)
            st, ln = ctx.chains(i)
            keep = ln > 0  # a CNT whose element nodes are all prescribed has an empty chain
            st, ln = st[keep], ln[keep]
            x = S["voltages"][S["reserved"]:]
            out.append({"A": A, "chain_start": st, "chain_len": ln, "err0": x - S["x0"], "n": A.shape[0]})
        if own:
            ctx.close()
    return out


class DeviceSystem:
    """A training system in device memory, bound to a cicy_gnn handle."""

    def __init__(self, gnn, sysd, device, stream):
        import torch

        self.dev = torch.device(f"cuda:{device}")
        A = sysd["A"]
        self.n, self.nnz = A.shape[0], A.nnz
        self.rp = torch.tensor(A.indptr.astype(np.int32), device=self.dev)
        self.ci = torch.tensor(A.indices.astype(np.int32), device=self.dev)
        self.val = torch.tensor(A.data, dtype=torch.float64, device=self.dev)
        self.cs = torch.tensor(np.asarray(sysd["chain_start"], np.int32), device=self.dev)
        self.cl = torch.tensor(np.asarray(sysd["chain_len"], np.int32), device=self.dev)
        self.err0 = torch.tensor(sysd["err0"], dtype=torch.float64, device=self.dev)
        self.desc = _abi.GnnSystem(self.n, self.nnz, self.rp.data_ptr(), self.ci.data_ptr(), self.val.data_ptr(), len(sysd["chain_start"]),
                                   self.cs.data_ptr(), self.cl.data_ptr())
        self.gnn, self.stream = gnn, stream

    def bind(self):
        _abi.check(_abi.lib().cicy_gnn_set_system(self.gnn, C.byref(self.desc), C.c_void_p(self.stream)), "cicy_gnn_set_system")


def train(systems, steps: int = 300, lr: float = 3e-3, n_random: int = 3, sweeps: int = 20, seed: int = 0, device: int = 0,
          params=None, log=print):
    """Adam on the residual-reduction loss, one system per step (cycling); returns the parameters."""
    import torch

    torch.cuda.set_device(device)
    dev = torch.device(f"cuda:{device}")
    stream = torch.cuda.current_stream(dev).cuda_stream
    L = _abi.lib()
    gnn = C.c_void_p()
    _abi.check(L.cicy_gnn_create(C.byref(gnn), device), "cicy_gnn_create")
    try:
        dsys = [DeviceSystem(gnn, s, device, stream) for s in systems]
        P = torch.tensor(init_params(seed) if params is None else params, dtype=torch.float32, device=dev)
        G = torch.zeros_like(P)
        M = torch.zeros_like(P)
        V = torch.zeros_like(P)
        gen = torch.Generator(device=dev)
        gen.manual_seed(seed)
        loss = C.c_double()
        history = []
        for step in range(1, steps + 1):
            ds = dsys[(step - 1) % len(dsys)]
            ds.bind()
            U = torch.empty((1 + n_random, ds.n), dtype=torch.float64, device=dev)
            U[0] = ds.err0
            U[1:] = torch.randn((n_random, ds.n), dtype=torch.float64, device=dev, generator=gen)
            _abi.check(L.cicy_gnn_smooth_probes(gnn, n_random, C.c_void_p(U[1:].data_ptr()), sweeps, C.c_void_p(stream)),
                       "cicy_gnn_smooth_probes")
            _abi.check(L.cicy_gnn_loss_grad(gnn, C.c_void_p(P.data_ptr()), 1 + n_random, C.c_void_p(U.data_ptr()), C.byref(loss),
                                            C.c_void_p(G.data_ptr()), C.c_void_p(stream)), "cicy_gnn_loss_grad")
            _abi.check(L.cicy_gnn_adam(C.c_void_p(P.data_ptr()), C.c_void_p(G.data_ptr()), C.c_void_p(M.data_ptr()),
                                       C.c_void_p(V.data_ptr()), len(P), step, lr, C.c_void_p(stream)), "cicy_gnn_adam")
            history.append(loss.value)
            if log and (step % 50 == 0 or step == 1):
                log(f"step {step}: loss {np.mean(history[-50:]):.4e}")
        torch.cuda.synchronize(dev)
        return P.cpu().numpy(), history
    finally:
        L.cicy_gnn_destroy(gnn)


def training_networks(count: int, seed0: int = 5_000_000, side=(2.0, 3.0), fraction=(0.012, 0.03)):
    """Seeded networks like the Monte-Carlo realisations (side and CNT volume fraction
    drawn per sample; smaller sides than the 2-5 um of the full sweep, for training speed)."""
    from .network import NetworkConfig, generate_cnt_network

    rng = np.random.default_rng(seed0)
    nets = []
    for k in range(count):
        L = float(rng.uniform(*side))
        phi = float(rng.uniform(*fraction))
        n_cnts = int(round(phi * L ** 3 / (math.pi * 0.005 ** 2 * 1.0)))
        cfg = NetworkConfig(side=L, n_cnts=n_cnts, seed=seed0 + k, tolerance=1e-8, tolerance_unit=1e-10)
        nets.append((cfg, generate_cnt_network(cfg).extract_window(cfg)))
    return nets


def monte_carlo_training_systems(count: int, seed0: int = 5_000_000, device: int = 0, log=print):
    """`count` real-resistor Laplacians from the Monte-Carlo sweep's generator (cube side
    U[2,5] um, CNT volume fraction U[0.5%,3%]) on seeds seed0, seed0 + 1, ... -- disjoint
    from the sweep's own seeds (3,000,000 + k), so the sweep evaluates on fresh networks.
    Realisations that do not percolate give no system and are skipped."""
    from .batch import monte_carlo_configs
    from .device import Context
    from .network import generate_cnt_network

    out, k, batch = [], 0, 64
    with Context(device) as ctx:  # one context; the multigrid solve gives the same systems faster
        while len(out) < count:
            cfgs = monte_carlo_configs(batch, seed0=seed0 + k)
            for cfg in cfgs:
                cfg.seed = seed0 + k
                k += 1
                got = collect_systems([(cfg, generate_cnt_network(cfg).extract_window(cfg))], device=device, ctx=ctx, preconditioner=3)
                out += got[: count - len(out)]
                if len(out) >= count:
                    break
            if log:
                log(f"{k} realisations, {len(out)} systems")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--networks", type=int, default=24)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--monte-carlo", type=int, default=0,
                    help="train on this many real-resistor Laplacians of the Monte-Carlo sweep's generator instead")
    ap.add_argument("--out", default=PARAMS_PATH)
    a = ap.parse_args()
    if a.monte_carlo:
        systems = monte_carlo_training_systems(a.monte_carlo)
    else:
        systems = collect_systems(training_networks(a.networks))
    print(f"{len(systems)} training systems, n = {min(s['n'] for s in systems)} .. {max(s['n'] for s in systems)}")
    P, hist = train(systems, steps=a.steps, lr=a.lr)
    P.astype(np.float32).tofile(a.out)
    print("wrote", a.out, f"loss first 100 steps {np.mean(hist[:100]):.4e}, last 100 steps {np.mean(hist[-100:]):.4e}")


if __name__ == "__main__":
    main()
