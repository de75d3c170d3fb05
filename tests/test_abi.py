"""The C-ABI library loads and exports every symbol include/cicy_b200.h declares (no GPU needed)."""
import ctypes as C

from cicy_geom_b200 import _abi


def test_library_loads_and_exports_all_declared_symbols():
    L = _abi.lib()
    declared = _abi.declared_symbols()
    assert len(declared) >= 25
    missing = [s for s in declared if not hasattr(L, s)]
    assert missing == []


def test_struct_sizes_match_header_layout():
    # the ctypes mirrors must have the C layout: spot-check sizes against the field lists
    assert C.sizeof(_abi.Cuboid) == 9 * 8
    assert C.sizeof(_abi.Params) == 8 * 3 + 8 * 4 + 4 * 6 + 8 * 8
    assert C.sizeof(_abi.SolveInfo) == 4 * 2 + 8 * 6 + 4 * 4
    assert C.sizeof(_abi.Result) == 8 * 6 + 8 * 2 + 4 * 4 + 32 * C.sizeof(_abi.SolveInfo) + 8 * 6
    # cicy_batch_system: n, nnz; 6 pointers; n_chains (+4 padding); 3 pointers (chains, edge weights)
    assert C.sizeof(_abi.BatchSystem) == 4 * 2 + 8 * 6 + 8 + 8 * 3
    # cicy_gnn_system: n, nnz; 3 pointers; n_chains (+4 padding); 2 pointers
    assert C.sizeof(_abi.GnnSystem) == 4 * 2 + 8 * 3 + 8 + 8 * 2
    # cicy_gnps: n (+4 padding); 6 pointers.  cicy_gnp_pair_list: 3 counts; 9 pointers
    assert C.sizeof(_abi.Gnps) == 8 + 8 * 6
    assert C.sizeof(_abi.GnpPairList) == 8 * 3 + 8 * 9
    # cicy_gnp_point_list: count, pointer, n_gnps (+4), 2 pointers, count, 2 pointers, n_boundary (+4), pointer
    assert C.sizeof(_abi.GnpPointList) == 8 * 2 + 8 + 8 * 2 + 8 * 3 + 8 + 8
    # cicy_gnp_window_list: n_inside (+4), 3 pointers, count, 5 pointers, n_gnps (+4), 3 pointers
    assert C.sizeof(_abi.GnpWindowList) == 8 + 8 * 3 + 8 + 8 * 5 + 8 + 8 * 3


def test_context_creation_without_gpu_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        return
    h = C.c_void_p()
    st = _abi.lib().cicy_ctx_create(C.byref(h), 0)
    assert st == 3  # CICY_E_DEVICE
    assert not h.value


def test_host_calls_reject_bad_input():
    L = _abi.lib()
    g = _abi.GenParams()
    g.n_cnts = -1
    out = C.c_void_p()
    assert L.cicy_generate_cnt_network(C.byref(g), C.byref(out)) == 1  # CICY_E_INPUT
    assert L.cicy_extract_window(None, None, C.byref(out)) == 1


def test_device_network_construction_rejects_a_missing_context():
    # the context-bound construction and copy-out calls check their handle before any CUDA call
    L = _abi.lib()
    g, w = _abi.GenParams(), _abi.WindowParams()
    assert L.cicy_ctx_generate_cnt_network(None, C.byref(g)) == 1  # CICY_E_INPUT
    assert L.cicy_ctx_extract_window(None, C.byref(w)) == 1
    n = C.c_int64()
    assert L.cicy_get_network(None, C.byref(n), None, None, None, None, None, None, None, None, None, None, None, None, None, None, None,
                              None, None) == 1
