"""The allocation-free solve entry point (cicy_jacobi_pcg_static) through the C ABI.

For callers that cannot allocate device memory at solve time (no cudaMalloc /
cudaFree in their loop, or a host that owns all device memory): the caller
passes the system, right-hand side and solution in its own device memory, the
library keeps its scratch in a fixed static device array.  Checked against the
voltages the regular entry point (cicy_electrical_analysis) produced for the
same DEA systems, on two calls in a row, within the voltage tolerance the other
parity tests use.  This file is collected last so a failure here leaves every
other test already run.
"""
import ctypes as C

import numpy as np
import pytest
from conftest import golden_network

from cicy_geom_b200 import _abi
from cicy_geom_b200.device import Context

pytestmark = pytest.mark.gpu


def full_csr(S):
    import scipy.sparse as sp

    n = len(S["diag"])
    L = sp.csr_matrix((S["values"], S["col_ind"], S["row_ptr"]), shape=(n, n))
    A = (L + L.T + sp.diags(S["diag"])).tocsr()
    A.sort_indices()
    return A


def solve_static(A, b, x0, tol):
    import torch

    dev = torch.device("cuda:0")
    rp = torch.tensor(A.indptr.astype(np.int32), device=dev)
    ci = torch.tensor(A.indices.astype(np.int32), device=dev)
    va = torch.tensor(A.data, dtype=torch.float64, device=dev)
    bb = torch.tensor(b, dtype=torch.float64, device=dev)
    xx = torch.tensor(x0, dtype=torch.float64, device=dev)
    it, rel = C.c_int64(), C.c_double()
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = _abi.lib().cicy_jacobi_pcg_static(A.shape[0], A.nnz, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), bb.data_ptr(),
                                           xx.data_ptr(), tol, 300 * A.shape[0], C.c_void_p(stream), C.byref(it), C.byref(rel))
    assert st == 0, _abi.lib().cicy_host_last_error()
    torch.cuda.synchronize()
    return xx.cpu().numpy(), it.value, rel.value


def test_static_solve_matches_the_regular_entry_point_on_two_calls(cuda_ok):
    cfg, net, z = golden_network("c1p_1200_s1")
    p = cfg.params()
    ctx = Context(0)
    ctx.upload(net)
    ctx.contact_grid(p)
    ctx.clusters(p)
    r = ctx.electrical_analysis(p)
    assert r.n_solves >= 2
    for i in range(r.n_solves):
        S = ctx.system(i)
        res = S["reserved"]
        A = full_csr(S)
        v_ref = S["voltages"][res:]
        scale = np.max(np.abs(S["voltages"]))
        runs = [solve_static(A, S["b"], S["x0"], cfg.tolerance) for _ in range(2)]
        for x, it, rel in runs:
            assert it > 0 and rel <= cfg.tolerance * 1.0001
            np.testing.assert_allclose(x, v_ref, rtol=0, atol=1e-5 * scale)
        # the second call starts from the first call's leftover scratch and gives the same answer
        np.testing.assert_array_equal(runs[0][0], runs[1][0])


def test_static_solve_rejects_systems_above_its_limit(cuda_ok):
    it, rel = C.c_int64(), C.c_double()
    st = _abi.lib().cicy_jacobi_pcg_static((1 << 17) + 1, (1 << 17) + 1, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                           C.c_void_p(1), 1e-10, 10, None, C.byref(it), C.byref(rel))
    assert st == 2  # CICY_E_CAPACITY, rejected before any device work
    assert b"static scratch limit" in _abi.lib().cicy_host_last_error()


def _device_csr(A):
    import torch

    dev = torch.device("cuda:0")
    return (torch.tensor(A.indptr.astype(np.int32), device=dev), torch.tensor(A.indices.astype(np.int32), device=dev),
            torch.tensor(A.data, dtype=torch.float64, device=dev))


def _laplacian_1d(n):
    import scipy.sparse as sp

    A = sp.diags([-np.ones(n - 1), 2.0 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1], format="csr")
    A.sort_indices()
    return A


def test_static_solve_rejects_a_malformed_system_before_using_its_indices(cuda_ok):
    import torch

    A = _laplacian_1d(1000)
    rp, ci, va = _device_csr(A)
    ci[17] = A.shape[0] + 5  # a column outside [0, n)
    b = torch.ones(A.shape[0], dtype=torch.float64, device="cuda:0")
    x = torch.zeros_like(b)
    it, rel = C.c_int64(), C.c_double()
    st = _abi.lib().cicy_jacobi_pcg_static(A.shape[0], A.nnz, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), b.data_ptr(), x.data_ptr(),
                                           1e-10, 1000, None, C.byref(it), C.byref(rel))
    assert st == 1  # CICY_E_INPUT
    assert b"column index" in _abi.lib().cicy_host_last_error()
    # the library stays usable: the same call on the well-formed system solves it
    rp, ci, va = _device_csr(A)
    st = _abi.lib().cicy_jacobi_pcg_static(A.shape[0], A.nnz, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), b.data_ptr(), x.data_ptr(),
                                           1e-10, 100000, None, C.byref(it), C.byref(rel))
    assert st == 0 and rel.value <= 1e-10


def test_static_solve_out_of_iterations_returns_ok_with_the_residual_above_tol(cuda_ok):
    import torch

    A = _laplacian_1d(4000)
    rp, ci, va = _device_csr(A)
    b = torch.ones(A.shape[0], dtype=torch.float64, device="cuda:0")
    x = torch.zeros_like(b)
    it, rel = C.c_int64(), C.c_double()
    st = _abi.lib().cicy_jacobi_pcg_static(A.shape[0], A.nnz, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), b.data_ptr(), x.data_ptr(),
                                           1e-10, 1, None, C.byref(it), C.byref(rel))
    assert st == 0
    assert it.value == 1 and rel.value > 1e-10
