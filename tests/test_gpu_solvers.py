"""Solver options of the DEA solve (chain block-Jacobi, chain-aggregation
multigrid) against an FP64 direct solve and against the upstream Jacobi-PCG.

The preconditioners change the iteration, not the system: solved tight, every
option must give the voltages of the FP64 direct solve within 1e-9 relative
(on the nodes a prescribed voltage reaches), and at the bench's tolerances the
same effective resistance as upstream Jacobi-PCG within the CG tolerance.
"""
import numpy as np
import pytest
from conftest import golden_network

from cicy_geom_b200.device import Context
from oracle import cicy_oracle as O

pytestmark = pytest.mark.gpu

PRECONDS = {"chain": 2, "mg": 3}


def run(net, cfg, preconditioner, tol):
    cfg.tolerance = tol
    p = cfg.params()
    ctx = Context(0)
    ctx.set_solver(preconditioner=preconditioner)
    ctx.upload(net)
    r = ctx.network_to_conductance(p)
    return ctx, r


@pytest.mark.parametrize("pre", list(PRECONDS))
@pytest.mark.parametrize("name", ["c1p_1200_s1", "c1p_800_s2", "c1p_800_s5", "kat_series", "kat_three_chain"])
def test_voltages_match_fp64_direct_solve(cuda_ok, name, pre):
    cfg, net, z = golden_network(name)
    ctx, r = run(net, cfg, PRECONDS[pre], 1e-14)
    for i in range(r.n_solves):
        S = ctx.system(i)
        if len(S["diag"]) == 0:
            continue
        vd = O.solve_direct({**S, "vef": S["voltages"][: S["reserved"]]})
        m = np.concatenate([np.ones(S["reserved"], bool), O.grounded_mask(S)])
        rel = np.max(np.abs(S["voltages"][m] - vd[m])) / np.max(np.abs(vd[m]))
        assert rel < 1e-9, (i, rel)
        if pre == "mg":
            assert r.solves[i].kernel == 2 and r.solves[i].levels >= 2
    ref = O.network_to_conductance(net.arrays(), O.params_from_config(cfg), solver="direct")
    np.testing.assert_allclose(np.array(r.resistances), ref["resistances"], rtol=1e-9)


def direct_errors(ctx, r):
    out = []
    for i in range(r.n_solves):
        S = ctx.system(i)
        if len(S["diag"]) == 0:
            continue
        vd = O.solve_direct({**S, "vef": S["voltages"][: S["reserved"]]})
        m = np.concatenate([np.ones(S["reserved"], bool), O.grounded_mask(S)])
        out.append(np.max(np.abs(S["voltages"][m] - vd[m])) / np.max(np.abs(vd[m])))
    return np.array(out)


@pytest.mark.parametrize("pre", [0, 2, 1])  # Jacobi, chain blocks, learned
@pytest.mark.parametrize("name", ["c1p_1200_s1", "c1p_800_s2"])
def test_mixed_precision_against_fp64(cuda_ok, name, pre):
    """FP32 difference-form SpMV and preconditioner apply with FP64 residual
    replacement, at 1e-10 on the FP64 true residual.  The FP64 solve at that
    tolerance is within ~1e-8 of the direct solve's voltages; mixed precision's
    FP32 SpMV noise lands partly in small-eigenvalue directions, so at the same
    residual its voltages are within ~1e-5 (bound 1e-4) and its effective
    resistance within 1e-6."""
    cfg, net, z = golden_network(name)
    cfg.tolerance = 1e-10
    cfg.tolerance_unit = 1e-10
    err = {}
    for prec in (0, 1):
        ctx = Context(0)
        ctx.set_solver(precision=prec, preconditioner=pre)
        ctx.upload(net)
        r = ctx.network_to_conductance(cfg.params())
        for i in range(r.n_solves):
            assert r.solves[i].fallback == 0
            if prec:
                assert r.solves[i].kernel == 0
        err[prec] = direct_errors(ctx, r)
        ref = O.network_to_conductance(net.arrays(), O.params_from_config(cfg), solver="direct")
        np.testing.assert_allclose(np.array(r.resistances), ref["resistances"], rtol=1e-6 if prec else 1e-7)
    assert np.all(err[0] <= 5e-7) and np.all(err[1] <= 1e-4), err


@pytest.fixture(scope="module")
def medium(cuda_ok):
    from cicy_geom_b200.network import NetworkConfig, generate_cnt_network

    cfg = NetworkConfig(side=3.2, n_cnts=8000, seed=1, tolerance=1e-8, tolerance_unit=1e-10)
    return cfg, generate_cnt_network(cfg).extract_window(cfg)


def test_smoothed_multigrid_against_direct_solve(medium):
    """Systems above 20,000 rows (the 8k-CNT network's two passes): the default hierarchy
    (smoothed level-1 prolongator, dense coarsest of up to 1,280 rows inverted by the grid
    Gauss-Jordan and solved on all CTAs) and the piecewise-constant one (CICY_SOLVER_NO_SMOOTHED)
    both reach the FP64 direct solve's voltages; the smoothed one in fewer iterations."""
    import copy

    cfg = copy.copy(medium[0])
    net = medium[1]
    cfg.tolerance = 1e-13
    cfg.tolerance_unit = 1e-13
    p = cfg.params()
    out = {}
    for smoothed in (True, False):
        ctx = Context(0)
        ctx.set_solver(preconditioner=3, smoothed=smoothed)
        ctx.upload(net)
        r = ctx.network_to_conductance(p)
        assert r.n_solves >= 2
        for i in range(r.n_solves):
            assert r.solves[i].kernel == 2 and r.solves[i].nodes - r.solves[i].reserved > 20000
        err = direct_errors(ctx, r)
        assert np.all(err < 1e-9), (smoothed, err)
        out[smoothed] = (r, sum(int(r.solves[i].iterations) for i in range(r.n_solves)))
        ctx.close()
    assert out[True][1] < out[False][1], (out[True][1], out[False][1])
    np.testing.assert_allclose(out[True][0].resistances[0], out[False][0].resistances[0], rtol=1e-9)


def test_multigrid_matches_jacobi_on_a_medium_network(medium):
    cfg, net = medium
    _, rj = run(net, cfg, 0, 1e-8)
    _, rm = run(net, cfg, 3, 1e-8)
    assert rm.n_solves == rj.n_solves
    for sj, sm in zip(rj.solves[: rj.n_solves], rm.solves[: rm.n_solves]):
        assert sm.nodes == sj.nodes and sm.nnz_lower == sj.nnz_lower
        assert sm.rel_residual <= 1e-8 * 1.01
        assert sm.iterations * 4 < sj.iterations
    np.testing.assert_allclose(rm.resistances[0], rj.resistances[0], rtol=1e-6)


def test_multigrid_cluster_and_grid_kernels_agree(cuda_ok):
    """The 16-CTA cluster kernel (systems up to 20k rows) and the grid-wide
    kernel (smoothed level-1 prolongator, dense coarsest of up to 1,280 rows
    solved on all CTAs) converge to the same answer; the grid-wide hierarchy
    is the stronger one."""
    cfg, net, z = golden_network("c1p_1200_s1")
    cfg.tolerance = 1e-10
    out = []
    for cluster in (True, False):
        ctx = Context(0)
        ctx.set_solver(preconditioner=3, cluster=cluster)
        ctx.upload(net)
        out.append(ctx.network_to_conductance(cfg.params()))
    a, b = out
    for sa, sb in zip(a.solves[: a.n_solves], b.solves[: b.n_solves]):
        assert sa.kernel == sb.kernel == 2
        assert sb.iterations <= sa.iterations + 2
        assert sa.rel_residual <= 1.01e-10 and sb.rel_residual <= 1.01e-10
    # two different preconditioners stopped at a 1e-10 relative residual: R agrees to the
    # solves' accuracy (each is within 1e-9 of an FP64 direct solve in the tests above)
    np.testing.assert_allclose(a.resistances[0], b.resistances[0], rtol=5e-9)


def test_spmv_matches_scipy(medium):
    """cicy_spmv_csr on a DEA system against scipy (FP64, summation order aside)."""
    import ctypes as C

    import torch

    from cicy_geom_b200 import _abi
    from cicy_geom_b200.learned import full_csr

    cfg, net = medium
    ctx = Context(0)
    ctx.set_solver(preconditioner=3)
    ctx.upload(net)
    r = ctx.network_to_conductance(cfg.params())
    A = full_csr(ctx.system(0))
    x = np.random.default_rng(0).normal(size=A.shape[0])
    dev = torch.device("cuda:0")
    t = [torch.tensor(a, device=dev) for a in (A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data, x)]
    y = torch.zeros(A.shape[0], dtype=torch.float64, device=dev)
    st = _abi.lib().cicy_spmv_csr(A.shape[0], *[C.c_void_p(v.data_ptr()) for v in t], C.c_void_p(y.data_ptr()), None)
    assert st == 0
    torch.cuda.synchronize()
    ref = A @ x
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(A.data).max() * np.abs(x).max())
