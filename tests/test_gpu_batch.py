"""Batched Monte-Carlo solves (cicy_batch_*): one persistent graph-captured
launch over many real-resistor systems, checked against an FP64 direct solve
and against the per-network solver, for the Jacobi, chain and learned
preconditioners, in FP64 and mixed precision (FP32 difference-form SpMV and
preconditioner factors, FP64 residual replacement)."""
import numpy as np
import pytest
from conftest import golden_network

from cicy_geom_b200 import batch as BT
from oracle import cicy_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mc_systems(cuda_ok):
    cfgs = BT.monte_carlo_configs(12, seed0=3_100_000, side=(2.0, 2.6), fraction=(0.012, 0.03))
    systems, info = BT.realisation_systems(cfgs, construction="host")
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


@pytest.mark.parametrize("precond", ["chain", "jacobi", "learned"])
def test_batch_matches_fp64_direct_solve(cuda_ok, precond):
    """FP64 solved tight: the direct solve's voltages within 1e-9.  At 1e-10
    on the FP64 true residual: FP64 within ~1e-8, mixed precision within ~1e-5
    (bound 1e-4; its FP32 SpMV noise lands partly in small-eigenvalue
    directions; an FP32 SpMV also stalls near the FP64 residual floor, so mixed
    is not asked for 1e-14)."""
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
    vd = []
    for s in systems:
        S = s["S"]
        vd.append((O.solve_direct({**S, "vef": S["voltages"][: S["reserved"]]})[S["reserved"]:], O.grounded_mask(S)))

    def errors(X):
        return np.array([np.max(np.abs(x[m] - v[m])) / np.max(np.abs(v[m])) for x, (v, m) in zip(X, vd)])

    bs = BT.BatchSolver(systems, tol=1e-14, learned=True if precond == "learned" else None)
    bs.set_solver(precond, 0)
    bs.solve()
    it, rel, fl = bs.results()
    # 1e-14 may sit at the FP64 residual floor, where the solve stops after its restarts (flag 0)
    assert np.all(fl >= 0) and np.all(rel <= 1e-12), (fl, rel)
    assert np.all(errors(bs.solutions()) < 1e-9)
    assert np.all(it > 0)
    bs.close()
    err = {}
    for prec in (0, 1):
        bs = BT.BatchSolver(systems, tol=1e-10, learned=True if precond == "learned" else None)
        bs.set_solver(precond, prec)
        bs.solve()
        it, rel, fl = bs.results()
        assert np.all(fl == 1) and np.all(rel <= 1.01e-10), (prec, fl, rel)
        err[prec] = errors(bs.solutions())
        bs.close()
    assert np.all(err[0] <= 5e-7) and np.all(err[1] <= 1e-4), err


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


@pytest.fixture(scope="module")
def mc_batch(mc_systems):
    bs = BT.BatchSolver(mc_systems, tol=1e-8, learned=True, max_iter_factor=20)  # cap: a stalled solve ends in seconds
    yield bs
    bs.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_preconditioners(mc_systems, mc_batch, precision):
    """Every preconditioner reaches 1e-8 on the FP64 true residual (relative to
    |b|); the learned one and the chain blocks take a fraction of Jacobi's iterations."""
    its = {}
    for pk in ("jacobi", "chain", "learned"):
        mc_batch.set_method(0)
        mc_batch.set_solver(pk, precision)
        mc_batch.solve()
        it, rel, fl = mc_batch.results()
        assert np.all(fl == 1), (pk, fl)
        assert np.all(rel <= 1.01e-8), (pk, rel)
        for s, x in zip(mc_systems, mc_batch.solutions()):  # two different 1e-8 solutions of the same system
            ref, m = s["x_ref"], grounded(s["A"])
            assert np.max(np.abs(x[m] - ref[m])) <= 5e-2 * np.max(np.abs(ref[m])), pk
        its[pk] = it.astype(np.float64)
    assert its["learned"].sum() * 4 < its["jacobi"].sum(), its
    assert its["chain"].sum() * 4 < its["jacobi"].sum(), its


def test_batch_sequential_method(mc_systems, mc_batch):
    """Method 2 (one system at a time through the grid-wide kernel) against method 0."""
    out = {}
    for method in (0, 2):
        mc_batch.set_method(method)
        mc_batch.set_solver("jacobi", 0)
        t = mc_batch.solve()
        it, rel, fl = mc_batch.results()
        assert t > 0 and np.all(fl == 1), (method, fl, rel)
        out[method] = (it, mc_batch.solutions())
    # same algorithm (different recurrences, stopping rules and rounding): similar iteration counts, the same voltages at 1e-8
    assert np.all(np.abs(out[0][0] - out[2][0]) <= 0.25 * out[2][0] + 10), (out[0][0], out[2][0])
    for s, a, b in zip(mc_systems, out[0][1], out[2][1]):
        m = grounded(s["A"])
        assert np.max(np.abs(a[m] - b[m])) <= 5e-2 * np.max(np.abs(b[m]))
    # (the per-network mixed path with the chain blocks alone has stalled on one of
    # these systems under this fixture's 20 n iteration cap; not asserted here)
    for pk, prec in (("learned", 0), ("learned", 1), ("chain", 0)):
        mc_batch.set_solver(pk, prec)
        mc_batch.solve()
        it, rel, fl = mc_batch.results()
        assert np.all(fl == 1), (pk, prec, fl)
    mc_batch.set_solver("chain", 0)
    mc_batch.set_method(0)


def test_batch_rejects_malformed_systems(mc_systems):
    """cicy_batch_create checks the CSR and the chain partition on the device
    (reads within the stated sizes only) before any solve can use them."""
    from cicy_geom_b200 import _abi

    good = mc_systems[:3]
    bad_chain = dict(good[1])
    cl = np.array(bad_chain["chain_len"], np.int32).copy()
    cl[0] += 1  # chains overlap: no longer consecutive runs
    bad_chain["chain_len"] = cl
    with pytest.raises(_abi.CicyError, match="system 1: the chains"):
        BT.BatchSolver([good[0], bad_chain, good[2]])
    with pytest.raises(_abi.CicyError, match="cicy_gnn_set_system: the chains"):
        BT.BatchSolver([bad_chain], learned=True)
    bad_col = dict(good[2])
    A = bad_col["A"].copy()
    A.indices = A.indices.copy()
    A.indices[-1] = A.shape[0]  # one column index past the last row
    bad_col["A"] = A
    with pytest.raises(_abi.CicyError, match="system 2: a column index"):
        BT.BatchSolver([good[0], good[1], bad_col])
    bs = BT.BatchSolver(good)  # the valid systems still solve
    bs.solve()
    assert np.all(bs.results()[2] == 1)
    bs.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_cluster_split(mc_systems, mc_batch, precision):
    """Systems on 16-CTA clusters (all of them, then the larger half) reach the
    same tolerance as on one CTA each, with similar iteration counts."""
    sizes = sorted(s["A"].shape[0] for s in mc_systems)
    mc_batch.set_method(0)
    for pk in ("jacobi", "chain", "learned"):
        mc_batch.set_solver(pk, precision)
        mc_batch.set_split(0)
        mc_batch.solve()
        it0, _, _ = mc_batch.results()
        x0 = mc_batch.solutions()
        for rows in (1, sizes[len(sizes) // 2]):
            mc_batch.set_split(rows)
            mc_batch.solve()
            it, rel, fl = mc_batch.results()
            assert np.all(fl == 1) and np.all(rel <= 1.01e-8), (pk, rows, fl, rel)
            # (reduction order differs: Jacobi-CG's iteration count on these systems is the most rounding-sensitive)
            spread = 0.5 if pk == "jacobi" else 0.25
            assert np.all(np.abs(it - it0) <= spread * it0 + 10), (pk, rows, it, it0)
            for s, a, b in zip(mc_systems, mc_batch.solutions(), x0):
                m = grounded(s["A"])
                assert np.max(np.abs(a[m] - b[m])) <= 5e-2 * np.max(np.abs(b[m])), (pk, rows)
    mc_batch.set_split(0)
    mc_batch.set_solver("chain", 0)
