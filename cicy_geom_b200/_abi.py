"""ctypes mirror of include/cicy_b200.h and the loader of libcicy_b200.so.

The shared library is the product; this module only declares its C types and
signatures.  Loading fails loudly when the library is missing: there is no
Python or CPU fallback for the device path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcicy_b200.so")

CICY_OK = 0
STATUS_NAMES = {
    0: "CICY_OK",
    1: "CICY_E_INPUT",
    2: "CICY_E_CAPACITY",
    3: "CICY_E_DEVICE",
    4: "CICY_E_TIMEOUT",
    5: "CICY_E_ZERO_DIAGONAL",
    6: "CICY_E_STATE",
    7: "CICY_E_INTERNAL",
}

i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
f64p = C.POINTER(C.c_double)


class Cuboid(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("min_x", "min_y", "min_z", "len_x", "len_y", "len_z", "max_x", "max_y", "max_z")]


class Params(C.Structure):
    _fields_ = [
        ("gs_min", C.c_double * 3),
        ("gs_overlap_cnt", C.c_double),
        ("gs_overlap_gnp", C.c_double),
        ("van_der_waals_dist", C.c_double),
        ("tunneling_dist", C.c_double),
        ("min_points", C.c_int32),
        ("simulation_scope", C.c_int32),
        ("resistances", C.c_int32 * 3),
        ("junction_type", C.c_int32),
        ("tolerance", C.c_double),
        ("applied_voltage", C.c_double),
        ("resistivity_cnt", C.c_double),
        ("resistivity_matrix", C.c_double),
        ("junction_resistance", C.c_double),
        ("C1", C.c_double),
        ("C2", C.c_double),
        ("tolerance_unit", C.c_double),
    ]


class Network(C.Structure):
    _fields_ = [
        ("n_points", C.c_int64),
        ("x", f64p),
        ("y", f64p),
        ("z", f64p),
        ("flag", i32p),
        ("n_cnts", C.c_int32),
        ("structure_ptr", i64p),
        ("structure_idx", i64p),
        ("radii", f64p),
        ("n_inside", C.c_int32),
        ("cnts_inside", i32p),
        ("boundary_cnt_ptr", i64p),
        ("boundary_cnt_idx", i32p),
        ("boundary_pts_ptr", i64p),
        ("boundary_pts_idx", i64p),
        ("window", Cuboid),
    ]


SOLVER_NO_CLUSTER = 1
SOLVER_NO_SMOOTHED = 2


class SolverOpts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("preconditioner", C.c_int32), ("max_iter_factor", C.c_int32), ("flags", C.c_int32)]


class SolveInfo(C.Structure):
    _fields_ = [
        ("cluster", C.c_int32),
        ("pass_", C.c_int32),
        ("nodes", C.c_int64),
        ("reserved", C.c_int64),
        ("nnz_lower", C.c_int64),
        ("iterations", C.c_int64),
        ("rel_residual", C.c_double),
        ("seconds", C.c_double),
        ("kernel", C.c_int32),
        ("restarts", C.c_int32),
        ("levels", C.c_int32),
        ("fallback", C.c_int32),
    ]


class Result(C.Structure):
    _fields_ = [
        ("resistances", C.c_double * 3),
        ("resistivities", C.c_double * 3),
        ("n_slots", C.c_int64),
        ("n_point_contacts", C.c_int64),
        ("n_labels", C.c_int32),
        ("n_junctions", C.c_int32),
        ("n_percolated", C.c_int32),
        ("n_solves", C.c_int32),
        ("solves", SolveInfo * 32),
        ("stage_seconds", C.c_double * 6),
    ]


_I64P, _I32P, _F64P = C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_double)


class HybridState(C.Structure):
    """cicy_hybrid_state: a mixed CNT/GNP network after percolation (host arrays)."""
    _fields_ = [
        ("n_clusters", C.c_int32), ("family", _I32P),
        ("clusters_cnt_ptr", _I64P), ("clusters_cnt_idx", _I32P),
        ("clusters_gnp_ptr", _I64P), ("clusters_gnp_idx", _I32P),
        ("cnt_junctions_ptr", _I64P), ("cnt_junctions_idx", _I32P),
        ("gnp_junctions_ptr", _I64P), ("gnp_junctions_idx", _I32P),
        ("mix_junctions_ptr", _I64P), ("mix_junctions_idx", _I32P),
        ("n_junctions_cnt", C.c_int64), ("jc_p1", _I64P), ("jc_n1", _I32P), ("jc_p2", _I64P), ("jc_n2", _I32P), ("jc_dist", _F64P),
        ("n_junctions_gnp", C.c_int64), ("jg_p1", _I64P), ("jg_n1", _I32P), ("jg_p2", _I64P), ("jg_n2", _I32P), ("jg_dist", _F64P),
        ("n_junctions_mixed", C.c_int64), ("jm_p1", _I64P), ("jm_n1", _I32P), ("jm_p2", _I64P), ("jm_n2", _I32P), ("jm_dist", _F64P),
        ("elements_ptr", _I64P), ("elements_idx", _I64P),
        ("n_gnps", C.c_int32), ("n_points_gnp", C.c_int64), ("points_gnp", _F64P),
        ("structure_gnp_ptr", _I64P), ("structure_gnp_idx", _I64P), ("pts_boundary_count", _I32P),
        ("gnp_t", _F64P), ("gnp_volume", _F64P), ("gnp_frame", _F64P),
        ("boundary_gnp_ptr", _I64P), ("boundary_gnp_idx", _I32P),
        ("boundary_gnp_pts_ptr", _I64P), ("boundary_gnp_pts_idx", _I64P),
    ]


class MixedClustersList(C.Structure):
    """cicy_mixed_clusters_list (borrowed view of a cicy_mixed_clusters result)."""
    _fields_ = [("n_percolated", C.c_int32), ("family", _I32P),
                ("clusters_cnt_ptr", _I64P), ("clusters_cnt_idx", _I32P), ("clusters_gnp_ptr", _I64P), ("clusters_gnp_idx", _I32P),
                ("n_isolated_cnt", C.c_int32), ("isolated_cnt_ptr", _I64P), ("isolated_cnt_idx", _I32P),
                ("n_isolated_gnp", C.c_int32), ("isolated_gnp_ptr", _I64P), ("isolated_gnp_idx", _I32P),
                ("cnt_junctions_ptr", _I64P), ("cnt_junctions_idx", _I32P), ("gnp_junctions_ptr", _I64P), ("gnp_junctions_idx", _I32P),
                ("mix_junctions_ptr", _I64P), ("mix_junctions_idx", _I32P),
                ("structure_gnp_ptr", _I64P), ("structure_gnp_idx", _I64P),
                ("pts_boundary_ptr", _I64P), ("pts_boundary_point", _I64P), ("pts_boundary_face", _I32P)]


class MixedState(C.Structure):
    """cicy_mixed_state: a mixed network after Make_mixed_clusters (host arrays)."""
    _fields_ = [("n_labels", C.c_int32), ("n_cnts", C.c_int32), ("labels_cnt", _I32P), ("n_cnts_inside", C.c_int32), ("cnts_inside", _I32P),
                ("n_gnps", C.c_int32), ("labels_gnp", _I32P), ("n_gnps_inside", C.c_int32), ("gnps_inside", _I32P),
                ("boundary_cnt_ptr", _I64P), ("boundary_cnt_idx", _I32P), ("boundary_gnp_ptr", _I64P), ("boundary_gnp_idx", _I32P),
                ("n_junctions_cnt", C.c_int64), ("jc_n1", _I32P), ("jc_n2", _I32P),
                ("n_junctions_gnp", C.c_int64), ("jg_n1", _I32P), ("jg_n2", _I32P),
                ("n_junctions_mixed", C.c_int64), ("jm_n1", _I32P), ("jm_n2", _I32P),
                ("n_points_gnp", C.c_int64), ("structure_gnp_ptr", _I64P), ("structure_gnp_idx", _I64P),
                ("pts_boundary_ptr", _I64P), ("pts_boundary_point", _I64P), ("pts_boundary_face", _I32P), ("bp_flags", _I32P)]


class GnnSystem(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("nnz", C.c_int32),
        ("row_ptr", C.c_void_p),
        ("col_ind", C.c_void_p),
        ("values", C.c_void_p),
        ("n_chains", C.c_int32),
        ("chain_start", C.c_void_p),
        ("chain_len", C.c_void_p),
    ]


class BatchSystem(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("nnz", C.c_int32),
        ("row_ptr", C.c_void_p),
        ("col_ind", C.c_void_p),
        ("values", C.c_void_p),
        ("b", C.c_void_p),
        ("x0", C.c_void_p),
        ("x", C.c_void_p),
        ("n_chains", C.c_int32),
        ("chain_start", C.c_void_p),
        ("chain_len", C.c_void_p),
        ("edge_weights", C.c_void_p),
    ]


class Gnps(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("l", C.c_void_p),
        ("t", C.c_void_p),
        ("center", C.c_void_p),
        ("rotation", C.c_void_p),
        ("vertices", C.c_void_p),
        ("planes", C.c_void_p),
    ]


class GnpPairList(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("n_visits", C.c_int64),
        ("n_pairs", C.c_int64),
        ("a", C.c_void_p),
        ("b", C.c_void_p),
        ("penetrating", C.c_void_p),
        ("dist", C.c_void_p),
        ("direction", C.c_void_p),
        ("displacement", C.c_void_p),
        ("point_a", C.c_void_p),
        ("point_b", C.c_void_p),
        ("outside", C.c_void_p),
    ]


class GnpPointList(C.Structure):
    _fields_ = [
        ("n_points", C.c_int64),
        ("points", C.c_void_p),
        ("n_gnps", C.c_int32),
        ("structure_ptr", C.c_void_p),
        ("structure_idx", C.c_void_p),
        ("n_junctions", C.c_int64),
        ("junctions", C.c_void_p),
        ("junction_dist", C.c_void_p),
        ("n_boundary", C.c_int32),
        ("boundary_used", C.c_void_p),
    ]


class GnpWindowList(C.Structure):
    _fields_ = [
        ("n_inside", C.c_int32),
        ("gnps_inside", C.c_void_p),
        ("boundary_gnp_ptr", C.c_void_p),
        ("boundary_gnp_idx", C.c_void_p),
        ("n_points", C.c_int64),
        ("points", C.c_void_p),
        ("point_gnp", C.c_void_p),
        ("point_boundary", C.c_void_p),
        ("boundary_pts_ptr", C.c_void_p),
        ("boundary_pts_idx", C.c_void_p),
        ("n_gnps", C.c_int32),
        ("structure_ptr", C.c_void_p),
        ("structure_idx", C.c_void_p),
        ("volume", C.c_void_p),
    ]


class GenParams(C.Structure):
    _fields_ = [
        ("sample", Cuboid),
        ("n_cnts", C.c_int32),
        ("n_threads", C.c_int32),
        ("seed", C.c_uint64),
        ("step", C.c_double),
        ("len_min", C.c_double),
        ("len_max", C.c_double),
        ("radius", C.c_double),
        ("max_turn_rad", C.c_double),
    ]


class WindowParams(C.Structure):
    _fields_ = [
        ("sample", Cuboid),
        ("win_max", C.c_double * 3),
        ("win_min", C.c_double * 3),
        ("win_delt", C.c_double * 3),
        ("step_length", C.c_double),
        ("min_points", C.c_int32),
        ("reserved0", C.c_int32),
    ]


_lib = None


def lib() -> C.CDLL:
    """Load libcicy_b200.so (built in-tree by cicy_geom_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m cicy_geom_b200.build` (no CPU fallback exists)")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    sig = {
        "cicy_ctx_create": (C.c_int, [P(C.c_void_p), C.c_int]),
        "cicy_ctx_destroy": (C.c_int, [C.c_void_p]),
        "cicy_ctx_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
        "cicy_ctx_stream": (C.c_void_p, [C.c_void_p]),
        "cicy_ctx_set_solver": (C.c_int, [C.c_void_p, P(SolverOpts)]),
        "cicy_ctx_set_spin_limit": (C.c_int, [C.c_void_p, C.c_int64]),
        "cicy_last_error": (C.c_char_p, [C.c_void_p]),
        "cicy_ctx_kernel_launches": (C.c_int64, [C.c_void_p]),
        "cicy_upload_network": (C.c_int, [C.c_void_p, P(Network)]),
        "cicy_ctx_generate_cnt_network": (C.c_int, [C.c_void_p, P(GenParams)]),
        "cicy_ctx_extract_window": (C.c_int, [C.c_void_p, P(WindowParams)]),
        "cicy_get_network": (C.c_int, [C.c_void_p, i64p, i32p, i32p, i64p, i64p, f64p, f64p, f64p, i32p, i32p, i32p, f64p, i32p, i64p,
                                       i32p, i64p, i32p, P(Cuboid)]),
        "cicy_contact_grid": (C.c_int, [C.c_void_p, P(Params)]),
        "cicy_clusters": (C.c_int, [C.c_void_p, P(Params)]),
        "cicy_electrical_analysis": (C.c_int, [C.c_void_p, P(Params), P(Result)]),
        "cicy_network_to_conductance": (C.c_int, [C.c_void_p, P(Params), P(Result)]),
        "cicy_get_sectioned_domain": (C.c_int, [C.c_void_p, i64p, i64p, i64p, i64p]),
        "cicy_get_point_contacts": (C.c_int, [C.c_void_p, i64p, i64p, i32p, i64p, f64p]),
        "cicy_get_labels": (C.c_int, [C.c_void_p, i32p, i32p, i32p]),
        "cicy_get_junctions": (C.c_int, [C.c_void_p, i64p, i64p, i32p, i64p, i32p, f64p]),
        "cicy_get_volumes": (C.c_int, [C.c_void_p, f64p, f64p, f64p, f64p]),
        "cicy_hybrid_electrical": (C.c_int, [C.c_void_p, P(HybridState), P(Params), C.c_double, C.c_double, P(Result)]),
        "cicy_mixed_percolation": (C.c_int, [C.c_void_p, P(MixedState), P(C.c_void_p)]),
        "cicy_mixed_clusters_view": (C.c_int, [C.c_void_p, P(MixedClustersList)]),
        "cicy_mixed_clusters_free": (None, [C.c_void_p]),
        "cicy_get_hybrid_structure": (C.c_int, [C.c_void_p, i64p, i64p, i64p]),
        "cicy_get_hybrid_volumes": (C.c_int, [C.c_void_p, f64p]),
        "cicy_get_hybrid_junctions": (C.c_int, [C.c_void_p, C.c_int32, i64p, i32p, i64p, i32p]),
        "cicy_get_elements": (C.c_int, [C.c_void_p, C.c_int32, i64p, i64p, i64p, i64p]),
        "cicy_get_clusters": (C.c_int, [C.c_void_p, C.c_int32, i32p, i64p, i64p, i32p, i32p, i64p, i64p, i32p]),
        "cicy_get_system": (C.c_int, [C.c_void_p, C.c_int32, i64p, i64p, i64p, i64p, i64p, f64p, f64p, f64p, f64p, f64p]),
        "cicy_generate_cnt_network": (C.c_int, [P(GenParams), P(C.c_void_p)]),
        "cicy_extract_window": (C.c_int, [C.c_void_p, P(WindowParams), P(C.c_void_p)]),
        "cicy_host_network_from_arrays": (C.c_int, [P(Network), P(C.c_void_p)]),
        "cicy_read_network": (C.c_int, [C.c_char_p, C.c_int32, P(C.c_void_p)]),
        "cicy_read_gnps": (C.c_int, [C.c_char_p, P(C.c_void_p)]),
        "cicy_gnp_set_view": (C.c_int, [C.c_void_p, P(Gnps)]),
        "cicy_gnp_set_free": (None, [C.c_void_p]),
        "cicy_gnp_extract_window": (C.c_int, [C.c_void_p, P(WindowParams), P(C.c_void_p)]),
        "cicy_gnp_window_view": (C.c_int, [C.c_void_p, P(GnpWindowList)]),
        "cicy_gnp_window_free": (None, [C.c_void_p]),
        "cicy_gnp_sectioned_domain": (C.c_int, [C.c_int, C.c_void_p, i32p, C.c_int32, P(Cuboid), f64p, C.c_double, C.c_double,
                                                P(C.c_void_p)]),
        "cicy_gnp_grid_view": (C.c_int, [C.c_void_p, i32p, f64p, P(C.c_void_p), P(C.c_void_p), i64p]),
        "cicy_gnp_grid_free": (None, [C.c_void_p]),
        "cicy_gnp_point_distance": (C.c_int, [C.c_int, C.c_void_p, C.c_int32, f64p, i32p, f64p, f64p, i32p]),
        "cicy_gnp_pair_distance": (C.c_int, [C.c_int, C.c_void_p, C.c_int32, i32p, i32p, C.c_double, f64p, f64p, f64p, i32p]),
        "cicy_gnp_junction_points": (C.c_int, [C.c_int, C.c_void_p, C.c_int32, i32p, i32p, C.c_double, P(Cuboid), C.c_int32, f64p, f64p,
                                               i32p, i32p]),
        "cicy_gnp_contact_pairs": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double, P(Cuboid), C.c_int32,
                                             P(C.c_void_p)]),
        "cicy_gnp_pairs_view": (C.c_int, [C.c_void_p, P(GnpPairList)]),
        "cicy_gnp_pairs_free": (None, [C.c_void_p]),
        "cicy_gnp_labels": (C.c_int, [C.c_int, C.c_void_p, C.c_int32, C.c_int32, i32p, i32p]),
        "cicy_gnp_junction_structures": (C.c_int, [C.c_int, C.c_void_p, C.c_int32, C.c_double, C.c_int32, f64p, i32p, i32p, P(C.c_void_p)]),
        "cicy_gnp_points_view": (C.c_int, [C.c_void_p, P(GnpPointList)]),
        "cicy_gnp_points_free": (None, [C.c_void_p]),
        "cicy_mixed_junctions": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, i64p]),
        "cicy_get_mixed_junctions": (C.c_int, [C.c_void_p, i64p, i64p, i32p, i64p, i32p, f64p, f64p]),
        "cicy_mixed_labels": (C.c_int, [C.c_void_p, i32p, C.c_int32, C.c_int32, i32p, i32p, i32p]),
        "cicy_gnp_cnt_contacts": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, P(Params), C.c_int32, i64p]),
        "cicy_get_gnp_cnt_contacts": (C.c_int, [C.c_void_p, i64p, i64p, i32p, f64p, f64p]),
        "cicy_host_network_view": (C.c_int, [C.c_void_p, P(Network)]),
        "cicy_host_network_free": (None, [C.c_void_p]),
        "cicy_host_last_error": (C.c_char_p, []),
        "cicy_spmv_csr": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "cicy_batch_create": (C.c_int, [P(C.c_void_p), C.c_int, P(BatchSystem), C.c_int32, C.c_double, C.c_int32, C.c_int32]),
        "cicy_batch_destroy": (C.c_int, [C.c_void_p]),
        "cicy_batch_set_shape": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
        "cicy_batch_enable_multigrid": (C.c_int, [C.c_void_p, f64p]),
        "cicy_batch_set_method": (C.c_int, [C.c_void_p, C.c_int32]),
        "cicy_batch_set_solver": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
        "cicy_batch_autotune": (C.c_int, [C.c_void_p, i32p, i32p, i32p, i32p, f64p]),
        "cicy_batch_set_split": (C.c_int, [C.c_void_p, C.c_int32]),
        "cicy_batch_solve": (C.c_int, [C.c_void_p, f64p]),
        "cicy_batch_results": (C.c_int, [C.c_void_p, i64p, f64p, i32p]),
        "cicy_get_chains": (C.c_int, [C.c_void_p, C.c_int32, i32p, i32p, i32p]),
        "cicy_gnn_param_count": (C.c_int32, []),
        "cicy_ctx_set_learned_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int32]),
        "cicy_gnn_create": (C.c_int, [P(C.c_void_p), C.c_int]),
        "cicy_gnn_destroy": (C.c_int, [C.c_void_p]),
        "cicy_gnn_set_system": (C.c_int, [C.c_void_p, P(GnnSystem), C.c_void_p]),
        "cicy_gnn_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "cicy_gnn_loss_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, f64p, C.c_void_p, C.c_void_p]),
        "cicy_gnn_smooth_probes": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p]),
        "cicy_gnn_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_void_p]),
        "cicy_jacobi_pcg_static": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_double, C.c_int64, C.c_void_p, i64p, f64p]),
    }
    for name, (res, args) in sig.items():
        if not hasattr(L, name):  # completeness is asserted by tests/test_abi.py
            continue
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def declared_symbols() -> list[str]:
    """Function names declared in include/cicy_b200.h (parsed from the header)."""
    import re

    hdr = os.path.join(os.path.dirname(HERE), "include", "cicy_b200.h")
    txt = open(hdr).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cicy_[a-z0-9_]+)\s*\(", txt)))


def ptr(a: np.ndarray, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


class CicyError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str = ""):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)} {msg}".strip())
        self.status = status


def check(status: int, where: str, ctx=None):
    if status != CICY_OK:
        msg = ""
        try:
            if ctx is not None:
                m = lib().cicy_last_error(ctx)
                msg = m.decode() if m else ""
            else:
                m = lib().cicy_host_last_error()
                msg = m.decode() if m else ""
        except Exception:  # pragma: no cover - message retrieval is best effort
            pass
        raise CicyError(status, where, msg)
