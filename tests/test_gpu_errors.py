"""Error paths of the C ABI on a GPU context (no fault is provoked on the device)."""
import ctypes as C

import numpy as np
import pytest

from cicy_geom_b200 import _abi
from cicy_geom_b200.device import Context
from cicy_geom_b200.network import HostNetwork, NetworkConfig, generate_cnt_network

pytestmark = pytest.mark.gpu


def test_stage_order_is_enforced(cuda_ok):
    ctx = Context(0)
    p = NetworkConfig().params()
    L = _abi.lib()
    assert L.cicy_contact_grid(ctx.handle, C.byref(p)) == 6  # CICY_E_STATE
    assert b"no network" in L.cicy_last_error(ctx.handle)
    assert L.cicy_clusters(ctx.handle, C.byref(p)) == 6
    r = _abi.Result()
    assert L.cicy_electrical_analysis(ctx.handle, C.byref(p), C.byref(r)) == 6


def test_non_contiguous_structure_is_rejected(cuda_ok):
    cfg = NetworkConfig(side=1.0, n_cnts=3, seed=1)
    a = generate_cnt_network(cfg).extract_window(cfg).arrays()
    a["structure_idx"] = a["structure_idx"].copy()
    a["structure_idx"][[1, 2]] = a["structure_idx"][[2, 1]]
    net = HostNetwork.from_arrays(a)
    ctx = Context(0)
    with pytest.raises(_abi.CicyError) as e:
        ctx.upload(net)
    assert e.value.status == 1 and "consecutive" in str(e.value)


def test_bad_device_and_solver_options(cuda_ok):
    h = C.c_void_p()
    assert _abi.lib().cicy_ctx_create(C.byref(h), 999) == 1
    ctx = Context(0)
    with pytest.raises(_abi.CicyError):
        ctx.set_solver(precision=7)


def test_context_is_reusable_after_an_error(cuda_ok):
    cfg = NetworkConfig(side=1.6, n_cnts=500, seed=3)
    net = generate_cnt_network(cfg).extract_window(cfg)
    ctx = Context(0)
    p = cfg.params()
    with pytest.raises(_abi.CicyError):
        ctx.clusters(p)
    ctx.upload(net)
    r1 = ctx.network_to_conductance(p)
    r2 = ctx.network_to_conductance(p)
    assert list(r1.resistances) == list(r2.resistances)  # deterministic across runs


@pytest.mark.parametrize("precond", [0, 3])
def test_bounded_wait_gives_up_and_the_context_stays_usable(cuda_ok, precond):
    """A grid-barrier wait limited to one poll gives up: the solve returns
    CICY_E_TIMEOUT (every CTA leaves at its next barrier; nothing hangs or faults),
    and the same context then solves the network normally.  Grid-wide kernels only
    (cluster=False): Jacobi-PCG (k_pcg) and the multigrid PCG (k_mg_pcg)."""
    from conftest import golden_network

    cfg, net, z = golden_network("c1p_1200_s1")
    p = cfg.params()
    ref = Context(0)
    ref.set_solver(preconditioner=precond, cluster=False)
    ref.upload(net)
    r0 = list(ref.network_to_conductance(p).resistances)
    ctx = Context(0)
    ctx.set_solver(preconditioner=precond, cluster=False)
    ctx.upload(net)
    ctx.set_spin_limit(1)
    with pytest.raises(_abi.CicyError) as e:
        ctx.network_to_conductance(p)
    assert e.value.status == 4 and "bounded device wait" in str(e.value)  # CICY_E_TIMEOUT
    ctx.set_spin_limit(0)
    assert list(ctx.network_to_conductance(p).resistances) == r0
