"""Size-independent properties of the device path on the full 25,000-CNT / 6 um network."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components

from cicy_geom_b200.device import Context
from cicy_geom_b200.network import NetworkConfig, generate_cnt_network

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big(cuda_ok):
    cfg = NetworkConfig(side=6.0, n_cnts=25000, seed=2_000_000, tolerance=1e-8, tolerance_unit=1e-12)
    net = generate_cnt_network(cfg).extract_window(cfg)
    ctx = Context(0)
    ctx.upload(net)
    r = ctx.network_to_conductance(cfg.params())
    return cfg, net, ctx, r


def test_contacts_are_unique_and_within_cutoff(big):
    cfg, net, ctx, r = big
    pa, cb, pb, d = ctx.point_contacts()
    a = net.arrays()
    assert len(pa) == r.n_point_contacts > 10000
    key = pa.astype(np.int64) * (1 << 20) + cb
    assert np.all(np.diff(key) > 0)  # sorted and unique (Pa, CNTb)
    assert np.all(d <= cfg.tunnel) and np.all(d >= cfg.vdw)
    assert np.all(a["flag"][pa] < cb) and np.all(a["flag"][pb] == cb)
    p = np.stack([a["x"], a["y"], a["z"]], 1)
    dist = np.linalg.norm(p[pa] - p[pb], axis=1) - 2 * cfg.radius
    np.testing.assert_allclose(np.maximum(dist, cfg.vdw), d, rtol=1e-12)


def test_labels_are_the_connected_components_in_first_contact_order(big):
    cfg, net, ctx, r = big
    pa, cb, pb, d = ctx.point_contacts()
    a = net.arrays()
    lab, nl = ctx.labels()
    n = len(lab)
    ca = a["flag"][pa]
    G = sp.coo_matrix((np.ones(len(ca)), (ca, cb)), shape=(n, n))
    nc, comp = connected_components(G, directed=False)
    m = lab >= 0
    assert m.sum() == len(np.unique(np.concatenate([ca, cb])))
    pairs = set(zip(lab[m].tolist(), comp[m].tolist()))
    assert len(pairs) == nl == len(set(comp[m].tolist()))


def test_solves_reach_the_residual_and_conserve_current(big):
    cfg, net, ctx, r = big
    assert r.n_percolated >= 1 and r.n_solves >= 2
    for s in r.solves[: r.n_solves]:
        assert s.rel_residual <= 1e-7
        assert s.iterations < 300 * s.nodes
    R = r.resistances[0]
    assert 0 < R < 1e6
    # maximum principle on every node connected to a prescribed voltage (nodes of
    # floating islands are undetermined by the system and excluded)
    from oracle import cicy_oracle as O

    S = ctx.system(r.n_solves - 1)
    v = S["voltages"][S["reserved"]:]
    m = O.grounded_mask(S)
    assert m.sum() > 0.9 * len(m)
    assert np.all(v[m] >= -1e-4) and np.all(v[m] <= 1 + 1e-4)
