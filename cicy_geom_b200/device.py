"""Device context: the hot path through the C ABI of libcicy_b200.

`Context` mirrors the upstream call sequence of App_Network_3D for one window
(App_Network_3D.cpp:140-179):

    ctx = Context(0)
    ctx.upload(window_network)           # window-trimmed network (host arrays)
    ctx.contact_grid(params)             # Contact_grid::Generate_contact_grid
    ctx.clusters(params)                 # Hoshen_Kopelman::Determine_clusters_and_percolation
    res = ctx.electrical_analysis(params)  # Electrical_analysis::Perform_analysis_on_clusters

and exposes the public members the upstream classes hand to later stages
(sectioned domain, point contacts, labels, junctions, elements, clusters,
families, each DEA system and its voltages) as numpy arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import check, lib
from .network import HostNetwork


def _p(a, ct):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


class Context:
    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().cicy_ctx_create(C.byref(h), device), "cicy_ctx_create")
        self._h = h
        self._device = device
        self._learned = False

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().cicy_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, st, where):
        check(st, where, self._h)

    # ---- configuration ----
    def set_stream(self, stream_ptr: int):
        self._check(lib().cicy_ctx_set_stream(self._h, C.c_void_p(stream_ptr)), "cicy_ctx_set_stream")

    def stream(self) -> int:
        return lib().cicy_ctx_stream(self._h) or 0

    def set_solver(self, precision: int = 0, preconditioner: int = 0, max_iter_factor: int = 300, cluster: bool = True,
                   smoothed: bool = True):
        """precision: 0 FP64, 1 mixed; preconditioner: 0 Jacobi (upstream), 1 learned, 2 chain blocks, 3 multigrid;
        cluster: allow the cluster-resident solver for systems that fit in shared memory; smoothed: the multigrid
        hierarchy above 20,000 rows smooths its first pairwise prolongator (CICY_SOLVER_NO_SMOOTHED when false)."""
        flags = (0 if cluster else _abi.SOLVER_NO_CLUSTER) | (0 if smoothed else _abi.SOLVER_NO_SMOOTHED)
        o = _abi.SolverOpts(precision, preconditioner, max_iter_factor, flags)
        self._check(lib().cicy_ctx_set_solver(self._h, C.byref(o)), "cicy_ctx_set_solver")
        if preconditioner == 1 and not self._learned:
            from .learned import default_params

            self.set_learned_params(default_params())

    def set_spin_limit(self, polls: int = 0):
        """Polls a grid-barrier wait makes before the solve gives up with CICY_E_TIMEOUT (0: the default)."""
        self._check(lib().cicy_ctx_set_spin_limit(self._h, int(polls)), "cicy_ctx_set_spin_limit")

    def set_learned_params(self, params: np.ndarray):
        """Parameters of the learned preconditioner (flat float32 vector, cicy_gnn_param_count entries)."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(lib().cicy_ctx_set_learned_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), len(p)),
                    "cicy_ctx_set_learned_params")
        self._learned = True

    def kernel_launches(self) -> int:
        return int(lib().cicy_ctx_kernel_launches(self._h))

    # ---- stages ----
    def upload(self, net: HostNetwork):
        v = net.view()
        self._check(lib().cicy_upload_network(self._h, C.byref(v)), "cicy_upload_network")
        self._window = _abi.Cuboid(*[getattr(v.window, f) for f, _ in _abi.Cuboid._fields_])

    def generate_network(self, cfg, trim: bool = True):
        """The seeded network of generate_cnt_network(cfg) generated on the device
        (cicy_ctx_generate_cnt_network), then, with `trim`, its window trimmed on the
        device (cicy_ctx_extract_window): the network the host pipeline
        generate_cnt_network(cfg).extract_window(cfg) uploads, built without the host."""
        from .network import gen_params

        g = gen_params(cfg)
        self._check(lib().cicy_ctx_generate_cnt_network(self._h, C.byref(g)), "cicy_ctx_generate_cnt_network")
        if trim:
            self.extract_window(cfg)

    def extract_window(self, cfg):
        """Window 0 of the context's untrimmed network, trimmed on the device (cicy_ctx_extract_window)."""
        wp = cfg.window_params()
        self._check(lib().cicy_ctx_extract_window(self._h, C.byref(wp)), "cicy_ctx_extract_window")
        w = _abi.Cuboid()
        self._check(lib().cicy_get_network(self._h, None, None, None, None, None, None, None, None, None, None, None, None, None,
                                           None, None, None, None, C.byref(w)), "cicy_get_network")
        self._window = w

    def network(self) -> dict:
        """The context's network (cicy_get_network) in the layout of HostNetwork.arrays()."""
        npt, nc, ni, nb, nq = C.c_int64(), C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64()
        self._check(lib().cicy_get_network(self._h, C.byref(npt), C.byref(nc), C.byref(ni), C.byref(nb), C.byref(nq), None, None, None,
                                           None, None, None, None, None, None, None, None, None, None), "cicy_get_network")
        n, c = npt.value, nc.value
        x, y, z = (np.zeros(max(n, 1)) for _ in range(3))
        flag = np.zeros(max(n, 1), np.int32)
        cs, cl, ins = np.zeros(max(c, 1), np.int32), np.zeros(max(c, 1), np.int32), np.zeros(max(ni.value, 1), np.int32)
        rad = np.zeros(max(c, 1))
        bcp, bpp = np.zeros(7, np.int64), np.zeros(7, np.int64)
        bci, bpi = np.zeros(max(nb.value, 1), np.int32), np.zeros(max(nq.value, 1), np.int32)
        w = _abi.Cuboid()
        self._check(lib().cicy_get_network(self._h, C.byref(npt), C.byref(nc), C.byref(ni), C.byref(nb), C.byref(nq), _p(x, C.c_double),
                                           _p(y, C.c_double), _p(z, C.c_double), _p(flag, C.c_int32), _p(cs, C.c_int32),
                                           _p(cl, C.c_int32), _p(rad, C.c_double), _p(ins, C.c_int32), _p(bcp, C.c_int64),
                                           _p(bci, C.c_int32), _p(bpp, C.c_int64), _p(bpi, C.c_int32), C.byref(w)), "cicy_get_network")
        cl = cl[:c].astype(np.int64)
        sp = np.concatenate([[0], np.cumsum(cl)]).astype(np.int64)
        sidx = np.concatenate([np.arange(s0, s0 + k, dtype=np.int64) for s0, k in zip(cs[:c], cl)]) if c else np.zeros(0, np.int64)
        return {"x": x[:n], "y": y[:n], "z": z[:n], "flag": flag[:n], "structure_ptr": sp, "structure_idx": sidx.astype(np.int64),
                "radii": rad[:c], "cnts_inside": ins[: ni.value], "boundary_cnt_ptr": bcp, "boundary_cnt_idx": bci[: nb.value],
                "boundary_pts_ptr": bpp, "boundary_pts_idx": bpi[: nq.value].astype(np.int64),
                "window": np.array([w.min_x, w.min_y, w.min_z, w.len_x, w.len_y, w.len_z, w.max_x, w.max_y, w.max_z])}

    def contact_grid(self, p: _abi.Params):
        self._check(lib().cicy_contact_grid(self._h, C.byref(p)), "cicy_contact_grid")

    def gnp_cnt_contacts(self, gnp_directory: str, p: _abi.Params, inside_is_error: bool = False, gnps_inside=None):
        """CNT-GNP contacts of the hybrid sample (cicy_gnp_cnt_contacts), after
        contact_grid(p) on the uploaded CNT network: the GNPs of
        gnp_directory/gnp_data.dat listed in `gnps_inside` (Cutoff_Wins::gnps_inside;
        None: all of them) on the same region grid (Generate_contact_grid for
        GNP_CNT_mix, then Find_adjacent_labels).  Returns (point, gnp, junction
        distance, closest GNP point [n, 3]) by contact-point number."""
        h = C.c_void_p()
        check(lib().cicy_read_gnps(gnp_directory.encode(), C.byref(h)), "cicy_read_gnps")
        grid = C.c_void_p()
        try:
            v = _abi.Gnps()
            check(lib().cicy_gnp_set_view(h, C.byref(v)), "cicy_gnp_set_view")
            ins = np.arange(v.n, dtype=np.int32) if gnps_inside is None else np.ascontiguousarray(gnps_inside, dtype=np.int32)
            gs = np.array(list(p.gs_min), dtype=np.float64)
            check(lib().cicy_gnp_sectioned_domain(self._device, h, ins.ctypes.data_as(_abi.i32p), len(ins), C.byref(self._window),
                                                  gs.ctypes.data_as(_abi.f64p), p.gs_overlap_cnt, p.gs_overlap_gnp, C.byref(grid)),
                  "cicy_gnp_sectioned_domain")
            n = C.c_int64()
            self._check(lib().cicy_gnp_cnt_contacts(self._h, h, grid, C.byref(p), int(inside_is_error), C.byref(n)), "cicy_gnp_cnt_contacts")
        finally:
            if grid:
                lib().cicy_gnp_grid_free(grid)
            lib().cicy_gnp_set_free(h)
        N = n.value
        pt, g = np.zeros(max(N, 1), np.int64), np.zeros(max(N, 1), np.int32)
        d, q = np.zeros(max(N, 1)), np.zeros((max(N, 1), 3))
        self._check(lib().cicy_get_gnp_cnt_contacts(self._h, C.byref(n), _p(pt, C.c_int64), _p(g, C.c_int32), _p(d, C.c_double),
                                                    _p(q, C.c_double)), "cicy_get_gnp_cnt_contacts")
        return pt[:N], g[:N], d[:N], q[:N]

    def mixed_labels(self, labels_gnp, n_total_labels: int):
        """Make_mixed_clusters' labels (cicy_mixed_labels) after clusters(p) and
        gnp_cnt_contacts: the GNP labels of the contact pass (numbered after the
        CNT labels, n_total_labels in all) joined to the CNT labels by the CNT-GNP
        contacts.  Returns (labels_cnt, labels_gnp, n_clusters)."""
        g = np.ascontiguousarray(labels_gnp, dtype=np.int32)
        nc = self.labels()[0].shape[0]
        lc, lg, n = np.zeros(max(nc, 1), np.int32), np.zeros(max(len(g), 1), np.int32), C.c_int32()
        self._check(lib().cicy_mixed_labels(self._h, g.ctypes.data_as(_abi.i32p), len(g), int(n_total_labels), _p(lc, C.c_int32),
                                            _p(lg, C.c_int32), C.byref(n)), "cicy_mixed_labels")
        return lc[:nc], lg[:len(g)], int(n.value)

    def mixed_junctions(self, n_points_gnp: int, min_points: int) -> dict:
        """Compress_mixed_contacts on the CNT-GNP contacts (cicy_mixed_junctions):
        junctions (cnt_point, cnt, gnp_point, gnp, dist) and the new GNP points,
        numbered from n_points_gnp."""
        n = C.c_int64()
        self._check(lib().cicy_mixed_junctions(self._h, int(n_points_gnp), int(min_points), C.byref(n)), "cicy_mixed_junctions")
        J = n.value
        cp, gp = np.zeros(max(J, 1), np.int64), np.zeros(max(J, 1), np.int64)
        c, g = np.zeros(max(J, 1), np.int32), np.zeros(max(J, 1), np.int32)
        d, q = np.zeros(max(J, 1)), np.zeros((max(J, 1), 3))
        self._check(lib().cicy_get_mixed_junctions(self._h, C.byref(n), _p(cp, C.c_int64), _p(c, C.c_int32), _p(gp, C.c_int64), _p(g, C.c_int32),
                                                   _p(d, C.c_double), _p(q, C.c_double)), "cicy_get_mixed_junctions")
        return {"cnt_point": cp[:J], "cnt": c[:J], "gnp_point": gp[:J], "gnp": g[:J], "dist": d[:J], "points": q[:J]}

    def clusters(self, p: _abi.Params):
        self._check(lib().cicy_clusters(self._h, C.byref(p)), "cicy_clusters")

    def electrical_analysis(self, p: _abi.Params) -> _abi.Result:
        r = _abi.Result()
        self._check(lib().cicy_electrical_analysis(self._h, C.byref(p), C.byref(r)), "cicy_electrical_analysis")
        return r

    def network_to_conductance(self, p: _abi.Params) -> _abi.Result:
        r = _abi.Result()
        self._check(lib().cicy_network_to_conductance(self._h, C.byref(p), C.byref(r)), "cicy_network_to_conductance")
        return r

    def hybrid_electrical(self, st: dict, p: _abi.Params, rho_gnp_surf: float = 1e-4, rho_gnp_t: float = 1.0) -> _abi.Result:
        """cicy_hybrid_electrical on a mixed CNT/GNP network after percolation.  `st` holds
        numpy arrays named as the fields of cicy_hybrid_state (CSR lists as *_ptr / *_idx;
        gnp_frame 16 values per GNP); the CNT network is the context's uploaded one."""
        types = {f: t for f, t in _abi.HybridState._fields_}
        keep = []
        h = _abi.HybridState()
        for f, t in types.items():
            if t in (C.c_int32, C.c_int64):
                setattr(h, f, int(st[f]))
                continue
            ct = t._type_
            dt = {C.c_int64: np.int64, C.c_int32: np.int32, C.c_double: np.float64}[ct]
            a = np.ascontiguousarray(st[f], dtype=dt)
            if a.size == 0:
                a = np.zeros(1, dt)
            keep.append(a)
            setattr(h, f, a.ctypes.data_as(t))
        self.hybrid_n_gnps = int(st["n_gnps"])
        r = _abi.Result()
        self._check(lib().cicy_hybrid_electrical(self._h, C.byref(h), C.byref(p), rho_gnp_surf, rho_gnp_t, C.byref(r)),
                    "cicy_hybrid_electrical")
        return r

    def hybrid_structure(self):
        """structure_gnp after the hybrid backbone, as (ptr, idx)."""
        n = C.c_int64()
        self._check(lib().cicy_get_hybrid_structure(self._h, C.byref(n), None, None), "cicy_get_hybrid_structure")
        ng = self.hybrid_n_gnps
        ptr, idx = np.zeros(ng + 1, np.int64), np.zeros(max(n.value, 1), np.int64)
        self._check(lib().cicy_get_hybrid_structure(self._h, C.byref(n), _p(ptr, C.c_int64), _p(idx, C.c_int64)), "cicy_get_hybrid_structure")
        return ptr, idx[: n.value]

    def hybrid_volumes(self) -> np.ndarray:
        """volumes_cnt[8], volumes_gnp[8], dead_branches[7], dead_gnps[7] of the hybrid stage."""
        v = np.zeros(30)
        self._check(lib().cicy_get_hybrid_volumes(self._h, _p(v, C.c_double)), "cicy_get_hybrid_volumes")
        return v

    def hybrid_junctions(self, cluster: int):
        """(cluster_gnp_junctions, cluster_mix_junctions) of a cluster after its backbone."""
        ng, nm = C.c_int64(), C.c_int64()
        self._check(lib().cicy_get_hybrid_junctions(self._h, cluster, C.byref(ng), None, C.byref(nm), None), "cicy_get_hybrid_junctions")
        g, m = np.zeros(max(ng.value, 1), np.int32), np.zeros(max(nm.value, 1), np.int32)
        self._check(lib().cicy_get_hybrid_junctions(self._h, cluster, C.byref(ng), _p(g, C.c_int32), C.byref(nm), _p(m, C.c_int32)),
                    "cicy_get_hybrid_junctions")
        return g[: ng.value], m[: nm.value]

    # ---- copy-out ----
    def sectioned_domain(self):
        nr, ns = C.c_int64(), C.c_int64()
        self._check(lib().cicy_get_sectioned_domain(self._h, C.byref(nr), C.byref(ns), None, None), "get_sectioned_domain")
        ptr = np.zeros(nr.value + 1, np.int64)
        idx = np.zeros(max(ns.value, 1), np.int64)
        self._check(lib().cicy_get_sectioned_domain(self._h, C.byref(nr), C.byref(ns), _p(ptr, C.c_int64), _p(idx, C.c_int64)),
                    "get_sectioned_domain")
        return ptr, idx[: ns.value]

    def point_contacts(self):
        n = C.c_int64()
        self._check(lib().cicy_get_point_contacts(self._h, C.byref(n), None, None, None, None), "get_point_contacts")
        N = n.value
        pa, pb = np.zeros(max(N, 1), np.int64), np.zeros(max(N, 1), np.int64)
        cb, d = np.zeros(max(N, 1), np.int32), np.zeros(max(N, 1), np.float64)
        self._check(lib().cicy_get_point_contacts(self._h, C.byref(n), _p(pa, C.c_int64), _p(cb, C.c_int32), _p(pb, C.c_int64),
                                                  _p(d, C.c_double)), "get_point_contacts")
        return pa[:N], cb[:N], pb[:N], d[:N]

    def labels(self):
        nc, nl = C.c_int32(), C.c_int32()
        self._check(lib().cicy_get_labels(self._h, C.byref(nc), C.byref(nl), None), "get_labels")
        lab = np.zeros(max(nc.value, 1), np.int32)
        self._check(lib().cicy_get_labels(self._h, C.byref(nc), C.byref(nl), _p(lab, C.c_int32)), "get_labels")
        return lab[: nc.value], nl.value

    def junctions(self):
        n = C.c_int64()
        self._check(lib().cicy_get_junctions(self._h, C.byref(n), None, None, None, None, None), "get_junctions")
        N = max(n.value, 1)
        p1, p2 = np.zeros(N, np.int64), np.zeros(N, np.int64)
        n1, n2 = np.zeros(N, np.int32), np.zeros(N, np.int32)
        d = np.zeros(N, np.float64)
        self._check(lib().cicy_get_junctions(self._h, C.byref(n), _p(p1, C.c_int64), _p(n1, C.c_int32), _p(p2, C.c_int64),
                                             _p(n2, C.c_int32), _p(d, C.c_double)), "get_junctions")
        k = n.value
        return p1[:k], n1[:k], p2[:k], n2[:k], d[:k]

    def volumes(self) -> dict:
        """Backbone_Network's volume members (cicy_get_volumes): volumes_cnt[8], dead_branches[7],
        total_volumes[8], fractions[8]."""
        v, d, t, f = np.zeros(8), np.zeros(7), np.zeros(8), np.zeros(8)
        self._check(lib().cicy_get_volumes(self._h, *[a.ctypes.data_as(_abi.f64p) for a in (v, d, t, f)]), "cicy_get_volumes")
        return {"volumes_cnt": v, "dead_branches": d, "total_volumes": t, "fractions": f}

    def elements(self, which: int = 0):
        nc, ni = C.c_int64(), C.c_int64()
        self._check(lib().cicy_get_elements(self._h, which, C.byref(nc), C.byref(ni), None, None), "get_elements")
        ptr = np.zeros(nc.value + 1, np.int64)
        idx = np.zeros(max(ni.value, 1), np.int64)
        self._check(lib().cicy_get_elements(self._h, which, C.byref(nc), C.byref(ni), _p(ptr, C.c_int64), _p(idx, C.c_int64)),
                    "get_elements")
        return ptr, idx[: ni.value]

    def percolated_clusters(self, which: int = 0):
        k, ni, nj = C.c_int32(), C.c_int64(), C.c_int64()
        self._check(lib().cicy_get_clusters(self._h, which, C.byref(k), C.byref(ni), None, None, None, C.byref(nj), None, None),
                    "get_clusters")
        K = k.value
        ptr, jptr = np.zeros(K + 1, np.int64), np.zeros(K + 1, np.int64)
        idx, jidx = np.zeros(max(ni.value, 1), np.int32), np.zeros(max(nj.value, 1), np.int32)
        fam = np.zeros(max(K, 1), np.int32)
        self._check(lib().cicy_get_clusters(self._h, which, C.byref(k), C.byref(ni), _p(ptr, C.c_int64), _p(idx, C.c_int32),
                                            _p(fam, C.c_int32), C.byref(nj), _p(jptr, C.c_int64), _p(jidx, C.c_int32)),
                    "get_clusters")
        return {"ptr": ptr, "idx": idx[: ni.value], "family": fam[:K], "junc_ptr": jptr, "junc_idx": jidx[: nj.value]}

    def chains(self, solve: int):
        """(start, len) of the CNT chains of a solve's system."""
        m = C.c_int32()
        self._check(lib().cicy_get_chains(self._h, solve, C.byref(m), None, None), "get_chains")
        st, ln = np.zeros(max(m.value, 1), np.int32), np.zeros(max(m.value, 1), np.int32)
        self._check(lib().cicy_get_chains(self._h, solve, C.byref(m), _p(st, C.c_int32), _p(ln, C.c_int32)), "get_chains")
        return st[: m.value], ln[: m.value]

    def system(self, solve: int) -> dict:
        nodes, res, m = C.c_int64(), C.c_int64(), C.c_int64()
        self._check(lib().cicy_get_system(self._h, solve, C.byref(nodes), C.byref(res), C.byref(m), None, None, None, None, None,
                                          None, None), "get_system")
        n = nodes.value - res.value
        rp = np.zeros(n + 1, np.int64)
        ci = np.zeros(max(m.value, 1), np.int64)
        val = np.zeros(max(m.value, 1), np.float64)
        diag, b, x0 = np.zeros(max(n, 1)), np.zeros(max(n, 1)), np.zeros(max(n, 1))
        volt = np.zeros(max(nodes.value, 1))
        self._check(lib().cicy_get_system(self._h, solve, C.byref(nodes), C.byref(res), C.byref(m), _p(rp, C.c_int64),
                                          _p(ci, C.c_int64), _p(val, C.c_double), _p(diag, C.c_double), _p(b, C.c_double),
                                          _p(x0, C.c_double), _p(volt, C.c_double)), "get_system")
        return {"nodes": nodes.value, "reserved": res.value, "row_ptr": rp, "col_ind": ci[: m.value], "values": val[: m.value],
                "diag": diag[:n], "b": b[:n], "x0": x0[:n], "voltages": volt[: nodes.value]}


def result_dict(r: _abi.Result) -> dict:
    return {
        "resistances": list(r.resistances),
        "resistivities": list(r.resistivities),
        "n_slots": r.n_slots,
        "n_point_contacts": r.n_point_contacts,
        "n_labels": r.n_labels,
        "n_junctions": r.n_junctions,
        "n_percolated": r.n_percolated,
        "solves": [
            {"cluster": s.cluster, "pass": s.pass_, "nodes": s.nodes, "reserved": s.reserved, "nnz_lower": s.nnz_lower,
             "iterations": s.iterations, "rel_residual": s.rel_residual, "seconds": s.seconds, "kernel": s.kernel,
             "restarts": s.restarts, "levels": s.levels, "fallback": s.fallback}
            for s in r.solves[: r.n_solves]
        ],
        "stage_seconds": list(r.stage_seconds),
    }
