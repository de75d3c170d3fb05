"""The CPU oracle of the learned preconditioner: its analytic gradient against
central finite differences (float64, no BF16 rounding), the BF16 rounding
helper, and the SPD property of the preconditioner it defines."""
import numpy as np
import pytest
from conftest import golden_network

from oracle import learned_oracle as LO


@pytest.fixture(scope="module")
def small_system():
    cfg, net, z = golden_network("c1p_1200_s1")
    S, A = LO.system_from_dump(z, "c0_d0_", net.arrays()["flag"])
    return S, A


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 3.1415926])
    y = LO.bf16(x)
    assert y[0] == 1.0 and y[4] == -2.5  # representable values stay put
    assert LO.bf16(np.array([1.0 + 2 ** -7]))[0] == 1.0 + 2 ** -7
    assert LO.bf16(np.array([1.0 + 2 ** -8]))[0] == 1.0  # tie, rounds to even
    assert LO.bf16(np.array([1.0 + 3 * 2 ** -8]))[0] == 1.0 + 2 ** -6  # tie, rounds to even
    assert np.all((y.astype(np.float32).view(np.uint32) & 0xFFFF) == 0)


def test_analytic_gradient_matches_finite_differences(small_system):
    S, A = small_system
    rng = np.random.default_rng(3)
    theta = LO.init_params(1)
    P = LO.unpack(theta)
    P["v"] = rng.normal(0, 0.3, P["v"].shape)
    theta = LO.pack(P)
    probes = [rng.normal(size=S.n) for _ in range(2)]
    L, g = LO.loss_and_grad(theta, S, probes, rounding=False)
    assert 0 < L < 1
    idx = rng.choice(len(theta), 24, replace=False)
    offs = np.cumsum([0] + [int(np.prod(s)) for _, s in LO.layout()])
    idx = np.unique(np.r_[idx, offs[:-1]])  # the first entry of every tensor too
    for i in idx:
        h = 1e-6 * max(1.0, abs(theta[i]))
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (LO.loss_and_grad(tp, S, probes, rounding=False)[0] - LO.loss_and_grad(tm, S, probes, rounding=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(abs(fd), 1e-3), (i, fd, g[i])


def test_preconditioner_is_symmetric_positive_definite(small_system):
    S, A = small_system
    rng = np.random.default_rng(5)
    w, _ = LO.forward(LO.init_params(2), S)
    assert np.all((w[S.off] > 0) & (w[S.off] < 1))
    a, b = rng.normal(size=S.n), rng.normal(size=S.n)
    za, _ = LO.precond(S, w, a)
    zb, _ = LO.precond(S, w, b)
    assert abs(za @ b - zb @ a) <= 1e-10 * abs(za @ b)
    for _ in range(4):
        r = rng.normal(size=S.n)
        assert LO.precond(S, w, r)[0] @ r > 0


def test_shipped_parameters_match_the_library_layout():
    from cicy_geom_b200 import learned as LG

    p = LG.default_params()
    assert len(p) == LG.param_count() == LO.n_params()
    assert np.all(np.isfinite(p))
    assert len(LG.init_params(0)) == LO.n_params()
    np.testing.assert_allclose(LG.init_params(0)[-2:], [0.0, np.log(4.0)], rtol=1e-6)
