"""The learned preconditioner on the device: its forward pass and gradient
against the CPU oracle (oracle/learned_oracle.py), training on the GPU with
the library's kernels, what the trained network gains over the chain
block-Jacobi without it, and the Jacobi fallback."""
import ctypes as C

import numpy as np
import pytest
from conftest import golden_network

from cicy_geom_b200 import _abi
from cicy_geom_b200 import learned as LG
from cicy_geom_b200.device import Context
from oracle import cicy_oracle as O
from oracle import learned_oracle as LO

pytestmark = pytest.mark.gpu


def real_system(name):
    cfg, net, z = golden_network(name)
    ctx = Context(0)
    ctx.set_solver(preconditioner=2)
    ctx.upload(net)
    r = ctx.network_to_conductance(cfg.params())
    i = [k for k in range(r.n_solves) if r.solves[k].pass_ >= 0][0]
    S = ctx.system(i)
    A = LG.full_csr(S)
    st, ln = ctx.chains(i)
    x = S["voltages"][S["reserved"]:]
    return {"A": A, "chain_start": st, "chain_len": ln, "err0": x - S["x0"], "n": A.shape[0]}, LO.System(A.indptr, A.indices, A.data, st, ln)


@pytest.fixture(scope="module")
def sys1(cuda_ok):
    return real_system("c1p_1200_s1")


@pytest.fixture(scope="module")
def gnn(cuda_ok):
    import torch

    h = C.c_void_p()
    _abi.check(_abi.lib().cicy_gnn_create(C.byref(h), 0), "cicy_gnn_create")
    yield h, torch.cuda.current_stream().cuda_stream
    _abi.lib().cicy_gnn_destroy(h)


def random_params(seed):
    rng = np.random.default_rng(seed)
    P = LO.unpack(LO.init_params(seed))
    P["v"] = rng.normal(0, 0.4, P["v"].shape)
    P["q"] = np.array([0.3, 0.5])
    return LO.pack(P).astype(np.float32)


def test_forward_matches_the_oracle(sys1, gnn):
    import torch

    sd, S = sys1
    h, stream = gnn
    ds = LG.DeviceSystem(h, sd, 0, stream)
    ds.bind()
    theta = random_params(1)
    P = torch.tensor(theta, device="cuda:0")
    w = torch.zeros(ds.nnz, dtype=torch.float32, device="cuda:0")
    _abi.check(_abi.lib().cicy_gnn_forward(h, C.c_void_p(P.data_ptr()), C.c_void_p(w.data_ptr()), C.c_void_p(stream)), "forward")
    wd = w.cpu().numpy()
    wo, _ = LO.forward(theta.astype(np.float64), S, rounding=True)
    m = S.offblock
    assert m.sum() > 100
    err = np.abs(wd[m] - wo[m])
    assert np.all(wd[~m] == 0)
    assert np.median(err) < 1e-4 and err.max() < 2e-2, (np.median(err), err.max())
    assert np.std(wo[m]) > 1e-3  # the weights do vary across couplings


def test_gradient_matches_the_oracle(sys1, gnn):
    import torch

    sd, S = sys1
    h, stream = gnn
    ds = LG.DeviceSystem(h, sd, 0, stream)
    ds.bind()
    theta = random_params(2)
    rng = np.random.default_rng(7)
    U = np.stack([sd["err0"]] + [rng.normal(size=S.n) for _ in range(2)])
    L_o, g_o = LO.loss_and_grad(theta.astype(np.float64), S, list(U), rounding=True)
    P = torch.tensor(theta, device="cuda:0")
    G = torch.zeros_like(P)
    Ud = torch.tensor(U, device="cuda:0")
    loss = C.c_double()
    _abi.check(_abi.lib().cicy_gnn_loss_grad(h, C.c_void_p(P.data_ptr()), len(U), C.c_void_p(Ud.data_ptr()), C.byref(loss),
                                             C.c_void_p(G.data_ptr()), C.c_void_p(stream)), "loss_grad")
    g_d = G.cpu().numpy().astype(np.float64)
    assert abs(loss.value - L_o) <= 1e-3 * abs(L_o) + 1e-12, (loss.value, L_o)
    rel = np.linalg.norm(g_d - g_o) / np.linalg.norm(g_o)
    cos = g_d @ g_o / (np.linalg.norm(g_d) * np.linalg.norm(g_o))
    assert rel < 3e-2 and cos > 0.999, (rel, cos)
    # every parameter tensor gets a gradient, matching the oracle's per tensor
    o = 0
    for name, shape in LO.layout():
        k = int(np.prod(shape))
        a, b = g_d[o:o + k], g_o[o:o + k]
        assert np.linalg.norm(a - b) <= 0.05 * np.linalg.norm(b) + 1e-9, name
        o += k


def test_training_on_the_gpu_reduces_the_loss(sys1):
    sd, S = sys1
    sd2, _ = real_system("c1p_800_s2")
    theta0 = LG.init_params(0)
    rng = np.random.default_rng(11)
    probes = [sd["err0"]] + [rng.normal(size=S.n) for _ in range(2)]
    for p in probes[1:]:  # smooth like the training probes
        for _ in range(20):
            p -= 0.9 * S.tsolve(S.matvec(p))
    before = LO.loss_and_grad(theta0.astype(np.float64), S, probes)[0]
    theta, hist = LG.train([sd, sd2], steps=80, lr=3e-3, seed=0, log=None)
    after = LO.loss_and_grad(theta.astype(np.float64), S, probes)[0]
    assert np.all(np.isfinite(theta)) and len(hist) == 80
    assert after < before, (before, after)


@pytest.fixture(scope="module")
def held_out(cuda_ok):
    # seeds outside the training set of the shipped parameters (5,000,000 + k)
    return LG.training_networks(2, seed0=6_000_000)


def solve_real(cfg, net, preconditioner, params=None, cluster=False, max_iter_factor=300):
    ctx = Context(0)
    ctx.upload(net)
    ctx.set_solver(preconditioner=preconditioner, cluster=cluster, max_iter_factor=max_iter_factor)
    if params is not None:
        ctx.set_learned_params(params)
    r = ctx.network_to_conductance(cfg.params())
    return r, [s for s in r.solves[: r.n_solves] if s.pass_ >= 0]


def test_trained_network_gains_over_the_blocks_without_it(held_out):
    """Same grid-wide PCG kernel, same chain blocks: with the trained network's
    sparse-approximate-inverse term the real-resistor solves take clearly fewer
    iterations, and far fewer than upstream Jacobi-PCG; same resistance."""
    for cfg, net in held_out:
        rj, sj = solve_real(cfg, net, 0)
        rc, sc = solve_real(cfg, net, 2)
        rl, sl = solve_real(cfg, net, 1)
        for j, c, l in zip(sj, sc, sl):
            assert l.kernel == 0 and c.kernel == 0 and l.fallback == 0
            assert l.rel_residual <= 1.01 * cfg.tolerance
            assert l.iterations * 1.4 < c.iterations, (l.iterations, c.iterations)
            assert l.iterations * 10 < j.iterations, (l.iterations, j.iterations)
        np.testing.assert_allclose(rl.resistances[0], rj.resistances[0], rtol=1e-6)


def test_jacobi_fallback_when_the_learned_preconditioner_fails():
    """Parameters that make the network output NaN: the solve falls back to
    Jacobi-PCG from the initial guess and still meets the tolerance."""
    cfg, net, z = golden_network("c1p_800_s2")
    bad = LG.init_params(0)
    bad[:] = np.nan
    r, s = solve_real(cfg, net, 1, params=bad, max_iter_factor=20)
    assert all(x.fallback == 1 for x in s)
    assert all(x.rel_residual <= 1.01 * cfg.tolerance for x in s)
    ref = O.network_to_conductance(net.arrays(), O.params_from_config(cfg), solver="direct")
    np.testing.assert_allclose(np.array(r.resistances), ref["resistances"], rtol=1e-6)
