"""Batched Monte-Carlo solves (cicy_batch_*): one persistent graph-captured
launch over many real-resistor systems, checked against an FP64 direct solve
and against the per-network solver, in FP64 and with the FP32
preconditioner apply."""
import numpy as np
import pytest
from conftest import golden_network

from cicy_geom_b200 import batch as BT
from oracle import cicy_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mc_systems(cuda_ok):
    cfgs = BT.monte_carlo_configs(12, seed0=3_100_000, side=(2.0, 2.6), fraction=(0.012, 0.03))
    systems, info = BT.realisation_systems(cfgs)
    assert info["percolating"] >= 6 and len(systems) >= 6
    return systems


def grounded(A):
    """Rows of components that reach a prescribed voltage (a positive row sum)."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components

    n = A.shape[0]
    C = A.tocoo()
    off = C.row != C.col
    nc, comp = connected_components(sp.coo_matrix((np.ones(off.sum()), (C.row[off], C.col[off])), shape=(n, n)), directed=False)
    rs = np.asarray(A.sum(axis=1)).ravel()
    g = np.zeros(nc, bool)
    g[comp[rs > 1e-9 * A.diagonal()]] = True
    return g[comp]


def test_batch_matches_fp64_direct_solve(cuda_ok):
    from cicy_geom_b200.device import Context
    from cicy_geom_b200.learned import full_csr

    systems = []
    for name in ("c1p_1200_s1", "c1p_800_s2", "c1p_800_s5"):
        cfg, net, z = golden_network(name)
        ctx = Context(0)
        ctx.set_solver(preconditioner=2)
        ctx.upload(net)
        r = ctx.network_to_conductance(cfg.params())
        for i in range(r.n_solves):
            S = ctx.system(i)
            st, ln = ctx.chains(i)
            systems.append({"A": full_csr(S), "b": S["b"], "x0": S["x0"], "chain_start": st, "chain_len": ln, "S": S})
    bs = BT.BatchSolver(systems, tol=1e-13)
    bs.solve()
    it, rel, fl = bs.results()
    X = bs.solutions()
    for s, x, f in zip(systems, X, fl):
        S = s["S"]
        vd = O.solve_direct({**S, "vef": S["voltages"][: S["reserved"]]})[S["reserved"]:]
        m = O.grounded_mask(S)
        err = np.max(np.abs(x[m] - vd[m])) / np.max(np.abs(vd[m]))
        assert err < 1e-9, err
    assert np.all(it > 0)
    bs.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_of_realisations_reaches_the_tolerance(mc_systems, precision):
    bs = BT.BatchSolver(mc_systems, tol=1e-8, precision=precision)
    if precision == 0:
        assert bs.enable_multigrid() > 0
    shape = bs.autotune()
    assert shape["threads"] in (256, 512, 1024) and shape["seconds"] > 0
    t1 = bs.solve()
    x1 = bs.solutions()
    t2 = bs.solve()
    x2 = bs.solutions()
    it, rel, fl = bs.results()
    assert np.all(fl == 1), fl
    assert np.all(rel <= 1.01e-8), rel
    for a, b in zip(x1, x2):  # replaying the graph gives the same answer
        np.testing.assert_array_equal(a, b)
    for s, x in zip(mc_systems, x1):  # the per-network solver's answer, both at 1e-8
        ref, m = s["x_ref"], grounded(s["A"])
        assert np.max(np.abs(x[m] - ref[m])) <= 2e-2 * np.max(np.abs(ref[m]))
    assert t1 > 0 and t2 > 0
    bs.close()


def test_batch_methods_agree(mc_systems):
    """One CTA per system (chain PCG) and one cluster per system (multigrid PCG)."""
    bs = BT.BatchSolver(mc_systems, tol=1e-10)
    bs.enable_multigrid()
    out = []
    for method in (0, 1):
        bs.set_method(method)
        bs.solve()
        it, rel, fl = bs.results()
        assert np.all(fl == 1) and np.all(rel <= 1.01e-10), (method, fl, rel)
        out.append((it, bs.solutions()))
    assert np.all(out[1][0] * 3 < out[0][0])  # multigrid: a fraction of the iterations
    for s, a, b in zip(mc_systems, out[0][1], out[1][1]):
        m = grounded(s["A"])
        assert np.max(np.abs(a[m] - b[m])) <= 1e-4 * np.max(np.abs(a[m]))
    bs.close()
