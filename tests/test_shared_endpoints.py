"""Window trimming can leave two CNT segments sharing an end point (the point
where a CNT was cut at a window face).  Upstream numbers such a point once, for
the CNT earlier in the cluster (LM_matrix_for_cnts, Direct_Electrifying.cpp:
139-215).  Checked on a seeded Monte-Carlo realisation that has such a point
on a face the real-resistor pass does not prescribe, against the upstream
program's resistance and system sizes (tests/golden/mc_3000057.json, made by
tests/golden/make_shared_endpoint_golden.py)."""
import json
import os

import numpy as np
import pytest
from conftest import GOLDEN

from cicy_geom_b200 import batch as BT


def golden():
    with open(os.path.join(GOLDEN, "mc_3000057.json")) as f:
        return json.load(f)


def network():
    from cicy_geom_b200.network import generate_cnt_network

    g = golden()
    cfg = [c for c in BT.monte_carlo_configs(64) if c.seed == g["seed"]][0]
    return cfg, generate_cnt_network(cfg).extract_window(cfg)


def test_window_has_cnts_sharing_an_end_point():
    cfg, net = network()
    a = net.arrays()
    sp, sx = a["structure_ptr"], a["structure_idx"]
    first = sx[sp[:-1][np.diff(sp) > 0]]
    last = sx[sp[1:][np.diff(sp) > 0] - 1]
    ends = np.concatenate([first, last])
    u, cnt = np.unique(ends, return_counts=True)
    assert (cnt > 1).sum() > 0  # some point ends two CNTs


@pytest.mark.gpu
def test_shared_end_points_numbered_once_like_upstream(cuda_ok):
    from cicy_geom_b200.device import Context

    g = golden()
    cfg, net = network()
    cfg.tolerance_unit = 0.0  # upstream: one tolerance for both passes
    ctx = Context(0)
    ctx.set_solver(preconditioner=0)  # the upstream Jacobi-PCG
    ctx.upload(net)
    r = ctx.network_to_conductance(cfg.params())
    real = [s for s in r.solves[: r.n_solves] if s.pass_ >= 0]
    unit = [s for s in r.solves[: r.n_solves] if s.pass_ < 0]
    assert [unit[0].nodes, unit[0].reserved] == g["unit_nodes"]
    assert [real[0].nodes, real[0].reserved] == g["real_nodes"]
    np.testing.assert_allclose(r.resistances[0], g["resistances"][0], rtol=1e-6)
