"""Host-side networks and parameters (the inputs of the hot path).

`HostNetwork` owns a network in the layout of the upstream `points_cnt`,
`structure_cnt`, `radii` and `Cutoff_Wins` outputs; `generate_cnt_network`
and `HostNetwork.extract_window` call the library's CPU network sources;
`write_read_network_files` writes the binary files `Read_Network` reads
(Read_Network.cpp:154-201, :348-467), so the upstream program and this
library can be run on the very same network.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import check, lib


@dataclass
class NetworkConfig:
    """A seeded synthetic CNT network and the run settings of the hot path."""

    side: float = 2.0            # cube side (um)
    n_cnts: int = 400
    seed: int = 1
    step: float = 0.01           # polyline step (um)
    len_min: float = 0.5
    len_max: float = 1.5
    radius: float = 0.005        # um
    max_turn_deg: float = 10.0
    gs_min: float = 0.05         # background grid cell (um)
    vdw: float = 0.00034         # van der Waals distance (um)
    tunnel: float = 0.0018       # tunnelling cutoff (um)
    min_points: int = 5          # junction compression (Cutoff_dist::min_points)
    cnt_min_points: int = 5      # shortest CNT segment kept by the window trimming (Nanotube_Geo::min_points)
    tolerance: float = 1e-10
    tolerance_unit: float = 0.0  # unit-resistor (backbone) pass; 0: same as `tolerance`
    applied_voltage: float = 1.0
    resistivity_cnt: float = 1e-3
    resistivity_matrix: float = 1.03e20
    junction: str = "exponential"
    junction_resistance: float = 1e7
    h_planck: float = 6.62606957
    e_charge: float = 1.60217662
    e_mass: float = 9.10938291
    barrier: float = 0.5
    resistances: tuple = (1, 0, 0)
    simulation_scope: int = 0
    gen_threads: int = 0

    def sample(self) -> _abi.Cuboid:
        s = self.side
        return _abi.Cuboid(0.0, 0.0, 0.0, s, s, s, s, s, s)

    def c1_c2(self):
        """Electric_para::C1, C2 exactly as Input_Reader.cpp:1450-1456 forms them."""
        sq = math.sqrt(2.0 * self.e_mass * self.barrier * self.e_charge)
        c1 = 10.0 * self.h_planck * self.h_planck / (self.e_mass * self.e_mass * sq)
        c2 = 4000.0 * 3.1415926535897932384626433832795 * sq / self.h_planck
        return c1, c2

    def params(self) -> _abi.Params:
        p = _abi.Params()
        for a in range(3):
            p.gs_min[a] = self.gs_min
        p.gs_overlap_cnt = 2 * self.radius + self.tunnel
        p.gs_overlap_gnp = 0.0
        p.van_der_waals_dist = self.vdw
        p.tunneling_dist = self.tunnel
        p.min_points = self.min_points
        p.simulation_scope = self.simulation_scope
        for a in range(3):
            p.resistances[a] = int(self.resistances[a])
        p.junction_type = 1 if self.junction == "exponential" else 0
        p.tolerance = self.tolerance
        p.applied_voltage = self.applied_voltage
        p.resistivity_cnt = self.resistivity_cnt
        p.resistivity_matrix = self.resistivity_matrix
        p.junction_resistance = self.junction_resistance
        p.C1, p.C2 = self.c1_c2()
        p.tolerance_unit = self.tolerance_unit
        return p

    def window_params(self) -> _abi.WindowParams:
        w = _abi.WindowParams()
        w.sample = self.sample()
        for a in range(3):
            w.win_max[a] = self.side
            w.win_min[a] = self.side
            w.win_delt[a] = 0.25
        w.step_length = self.step
        w.min_points = self.cnt_min_points
        return w


class HostNetwork:
    """A CNT network in host memory owned by libcicy_b200."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().cicy_host_network_free(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    def view(self) -> _abi.Network:
        v = _abi.Network()
        check(lib().cicy_host_network_view(self._h, C.byref(v)), "cicy_host_network_view")
        return v

    def arrays(self) -> dict:
        """Copies of the network arrays as numpy arrays."""
        v = self.view()
        n, c = v.n_points, v.n_cnts

        def arr(p, count, dt):
            if count == 0 or not p:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(p, shape=(count,)).astype(dt, copy=True)

        sp = arr(v.structure_ptr, c + 1, np.int64)
        bcp = arr(v.boundary_cnt_ptr, 7, np.int64)
        bpp = arr(v.boundary_pts_ptr, 7, np.int64)
        w = v.window
        return {
            "x": arr(v.x, n, np.float64),
            "y": arr(v.y, n, np.float64),
            "z": arr(v.z, n, np.float64),
            "flag": arr(v.flag, n, np.int32),
            "structure_ptr": sp,
            "structure_idx": arr(v.structure_idx, int(sp[-1]) if c >= 0 else 0, np.int64),
            "radii": arr(v.radii, c, np.float64),
            "cnts_inside": arr(v.cnts_inside, v.n_inside, np.int32),
            "boundary_cnt_ptr": bcp,
            "boundary_cnt_idx": arr(v.boundary_cnt_idx, int(bcp[6]), np.int32),
            "boundary_pts_ptr": bpp,
            "boundary_pts_idx": arr(v.boundary_pts_idx, int(bpp[6]), np.int64),
            "window": np.array([w.min_x, w.min_y, w.min_z, w.len_x, w.len_y, w.len_z, w.max_x, w.max_y, w.max_z]),
        }

    @property
    def n_points(self) -> int:
        return int(self.view().n_points)

    @property
    def n_cnts(self) -> int:
        return int(self.view().n_cnts)

    def extract_window(self, cfg: NetworkConfig) -> "HostNetwork":
        """Shells + Cutoff_Wins for window 0 (cicy_extract_window)."""
        out = C.c_void_p()
        wp = cfg.window_params()
        check(lib().cicy_extract_window(self._h, C.byref(wp), C.byref(out)), "cicy_extract_window")
        return HostNetwork(out.value)

    @staticmethod
    def from_arrays(a: dict) -> "HostNetwork":
        keep = {}

        def p(name, ct, dt):
            x = np.ascontiguousarray(a[name], dtype=dt)
            keep[name] = x
            return x.ctypes.data_as(C.POINTER(ct))

        v = _abi.Network()
        v.n_points = len(a["x"])
        v.x, v.y, v.z = p("x", C.c_double, np.float64), p("y", C.c_double, np.float64), p("z", C.c_double, np.float64)
        v.flag = p("flag", C.c_int32, np.int32)
        v.n_cnts = len(a["radii"])
        v.structure_ptr = p("structure_ptr", C.c_int64, np.int64)
        v.structure_idx = p("structure_idx", C.c_int64, np.int64)
        v.radii = p("radii", C.c_double, np.float64)
        v.n_inside = len(a.get("cnts_inside", []))
        if v.n_inside:
            v.cnts_inside = p("cnts_inside", C.c_int32, np.int32)
        if "boundary_cnt_ptr" in a:
            v.boundary_cnt_ptr = p("boundary_cnt_ptr", C.c_int64, np.int64)
            v.boundary_cnt_idx = p("boundary_cnt_idx", C.c_int32, np.int32)
            v.boundary_pts_ptr = p("boundary_pts_ptr", C.c_int64, np.int64)
            v.boundary_pts_idx = p("boundary_pts_idx", C.c_int64, np.int64)
        w = np.asarray(a["window"], dtype=np.float64)
        v.window = _abi.Cuboid(*[float(t) for t in w])
        out = C.c_void_p()
        check(lib().cicy_host_network_from_arrays(C.byref(v), C.byref(out)), "cicy_host_network_from_arrays")
        return HostNetwork(out.value)


def read_network_files(directory: str, file_type: str = "dat") -> HostNetwork:
    """The network Read_Network reads from `directory` (cicy_read_network): sample_geom.csv
    and cnt_struct/cnt_coordinates in the binary ("dat") or CSV ("csv") format."""
    ft = {"dat": 0, "csv": 1}[file_type]
    out = C.c_void_p()
    check(lib().cicy_read_network(directory.encode(), ft, C.byref(out)), "cicy_read_network")
    return HostNetwork(out.value)


def gen_params(cfg: NetworkConfig) -> _abi.GenParams:
    """Generator parameters of a configuration (cicy_gen_params)."""
    g = _abi.GenParams()
    g.sample = cfg.sample()
    g.n_cnts = cfg.n_cnts
    g.n_threads = cfg.gen_threads
    g.seed = cfg.seed
    g.step = cfg.step
    g.len_min = cfg.len_min
    g.len_max = cfg.len_max
    g.radius = cfg.radius
    g.max_turn_rad = math.radians(cfg.max_turn_deg)
    return g


def generate_cnt_network(cfg: NetworkConfig) -> HostNetwork:
    """Seeded synthetic CNT network (cicy_generate_cnt_network)."""
    g = gen_params(cfg)
    out = C.c_void_p()
    check(lib().cicy_generate_cnt_network(C.byref(g), C.byref(out)), "cicy_generate_cnt_network")
    return HostNetwork(out.value)


def write_read_network_files(directory: str, net: HostNetwork, cfg: NetworkConfig, file_type: str = "dat") -> None:
    """Write input.dat, sample_geom.csv and the CNT files Read_Network reads.

    file_type "dat": binary layout of Read_Network::Read_cnt_data_from_dat
    (Read_Network.cpp:348-467): cnt_struct.dat = int n_cnts, then per CNT
    {int n_points; double radius}; cnt_coordinates.dat = x, y, z doubles per
    point in CNT order.  "csv": Read_cnt_data_from_csv (:203-346):
    cnt_struct.csv = "n_cnts,n_cnts", then "n_points,radius" per CNT;
    cnt_coordinates.csv = "x,y,z" per point (shortest round-trip decimals).
    """
    os.makedirs(directory, exist_ok=True)
    a = net.arrays()
    sp = a["structure_ptr"]
    counts = np.diff(sp).astype(np.int32)
    idx = a["structure_idx"]
    xyz = np.stack([a["x"][idx], a["y"][idx], a["z"][idx]], axis=1).astype("<f8")
    if file_type == "dat":
        rec = np.zeros(len(counts), dtype=np.dtype([("np", "<i4"), ("r", "<f8")], align=False))
        rec["np"] = counts
        rec["r"] = a["radii"]
        with open(os.path.join(directory, "cnt_struct.dat"), "wb") as f:
            f.write(np.int32(len(counts)).tobytes())
            f.write(rec.tobytes())
        with open(os.path.join(directory, "cnt_coordinates.dat"), "wb") as f:
            f.write(xyz.tobytes())
    elif file_type == "csv":
        with open(os.path.join(directory, "cnt_struct.csv"), "w") as f:
            f.write(f"{len(counts)},{len(counts)}\n")
            f.write("".join(f"{int(c)},{float(r)!r}\n" for c, r in zip(counts, a["radii"])))
        with open(os.path.join(directory, "cnt_coordinates.csv"), "w") as f:
            f.write("".join(f"{float(x)!r},{float(y)!r},{float(z)!r}\n" for x, y, z in xyz))
    else:
        raise ValueError("file_type: 'dat' or 'csv'")
    s = cfg.side
    with open(os.path.join(directory, "sample_geom.csv"), "w") as f:
        f.write(f"0,0,0\n{s!r},{s!r},{s!r}\n")
    with open(os.path.join(directory, "input.dat"), "w") as f:
        f.write(input_dat(cfg, file_type))


def input_dat(cfg: NetworkConfig, file_type: str = "dat") -> str:
    """An upstream input.dat for a single-window Read_Network run of `cfg` (CNT files in `file_type`)."""
    s = repr(float(cfg.side))
    r = cfg.resistances
    if cfg.junction == "exponential":
        junc = f"exponential {cfg.h_planck!r} {cfg.e_charge!r} {cfg.e_mass!r} {cfg.barrier!r}"
    else:
        junc = f"constant {cfg.junction_resistance!r}"
    scope = f"{cfg.simulation_scope} {r[0]} {r[1]} {r[2]}" if cfg.simulation_scope == 0 else f"{cfg.simulation_scope}"
    return f"""Application
3D_Electrical_Network
Simulation_Parameters
Synthetic
1
CNT_wires
Read_Network
{file_type}
vol 0.01
1
{scope}
{cfg.tolerance!r}
5
Sample_Geometry
0 0 0 {s} {s} {s}
{s} {s} {s}
0.25 0.25 0.25
{s} {s} {s}
{cfg.gs_min!r} {cfg.gs_min!r} {cfg.gs_min!r}
1.03
Cutoff_Distances
{cfg.vdw!r} {cfg.tunnel!r} {cfg.min_points}
CNT_Geometry
random
-1.5707963267948966 1.5707963267948966
{cfg.step!r}
uniform {cfg.len_min!r} {cfg.len_max!r}
points {cfg.cnt_min_points}
uniform {cfg.radius!r} {cfg.radius!r}
1.78
Electrical_Parameters
{cfg.applied_voltage!r}
{cfg.resistivity_cnt!r}
1.0 1e-4
{cfg.resistivity_matrix!r}
{junc}
Visualization_Flags
0
0
0
0
0
Output_Data_Flags
0
0
0
"""


# ---------------------------------------------------------------------------
# GNPs (graphene nanoplatelets): seeded generation and the Read_Network file


def generate_gnps(n: int, side: float, seed: int, l_range=(0.5, 1.0), thickness: float = 0.01) -> dict:
    """Seeded GNPs for a cube of `side` um (the hybrid configuration's distribution):
    square side U[l_range], thickness `thickness`, centre uniform in the cube,
    normal uniform on the sphere, stored as the (theta, phi) of the normal that
    gnp_data.dat holds (Read_Network.cpp:576-679: the rotation matrix's third
    column is the normal)."""
    rng = np.random.default_rng(seed)
    return {"l": rng.uniform(*l_range, n), "t": np.full(n, float(thickness)),
            "theta": np.arccos(rng.uniform(-1.0, 1.0, n)), "phi": rng.uniform(0.0, 2 * math.pi, n),
            "center": rng.uniform(0.0, side, (n, 3))}


def write_gnp_file(directory: str, gnps: dict) -> None:
    """gnp_data.dat as Read_Network::Read_gnp_data_from_dat reads it: int n, then per
    GNP the doubles l, t, theta, phi, centre x, y, z."""
    os.makedirs(directory, exist_ok=True)
    n = len(gnps["l"])
    rec = np.zeros((n, 7), "<f8")
    rec[:, 0], rec[:, 1], rec[:, 2], rec[:, 3] = gnps["l"], gnps["t"], gnps["theta"], gnps["phi"]
    rec[:, 4:7] = gnps["center"]
    with open(os.path.join(directory, "gnp_data.dat"), "wb") as f:
        f.write(np.int32(n).tobytes())
        f.write(rec.tobytes())


def read_gnps(directory: str) -> dict:
    """GNPs of `directory`/gnp_data.dat as upstream's Read_Network builds them
    (cicy_read_gnps): l, t [n]; center [n, 3]; rotation [n, 3, 3]; vertices
    [n, 8, 3]; planes [n, 6, 4] (normal, offset)."""
    h = C.c_void_p()
    check(lib().cicy_read_gnps(directory.encode(), C.byref(h)), "cicy_read_gnps")
    try:
        v = _abi.Gnps()
        check(lib().cicy_gnp_set_view(h, C.byref(v)), "cicy_gnp_set_view")
        n = v.n

        def arr(ptr, count, shape):
            if count == 0:
                return np.zeros(shape)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_double)), shape=(count,)).copy().reshape(shape)

        return {"l": arr(v.l, n, (n,)), "t": arr(v.t, n, (n,)), "center": arr(v.center, 3 * n, (n, 3)),
                "rotation": arr(v.rotation, 9 * n, (n, 3, 3)), "vertices": arr(v.vertices, 24 * n, (n, 8, 3)),
                "planes": arr(v.planes, 24 * n, (n, 6, 4))}
    finally:
        lib().cicy_gnp_set_free(h)


def gnp_sectioned_domain(directory: str, inside, window, gs_min, overlap_cnt: float, overlap_gnp: float, device: int = 0):
    """Upstream's GNP part of the contact grid on the device (cicy_gnp_sectioned_domain) for
    the GNPs of `directory`/gnp_data.dat: returns (n_regions[3], l_regions[3], ptr, idx),
    region t's GNPs being idx[ptr[t]:ptr[t + 1]].  window = (min xyz, len xyz, max xyz)."""
    h = C.c_void_p()
    check(lib().cicy_read_gnps(directory.encode(), C.byref(h)), "cicy_read_gnps")
    grid = C.c_void_p()
    try:
        ins = np.ascontiguousarray(inside, dtype=np.int32)
        gs = np.ascontiguousarray(gs_min, dtype=np.float64)
        w = _abi.Cuboid(*[float(x) for x in window])
        check(lib().cicy_gnp_sectioned_domain(device, h, ins.ctypes.data_as(_abi.i32p), len(ins), C.byref(w), gs.ctypes.data_as(_abi.f64p),
                                              float(overlap_cnt), float(overlap_gnp), C.byref(grid)), "cicy_gnp_sectioned_domain")
        n = np.zeros(3, np.int32)
        l = np.zeros(3)
        pp, ip = C.c_void_p(), C.c_void_p()
        ne = C.c_int64()
        check(lib().cicy_gnp_grid_view(grid, n.ctypes.data_as(_abi.i32p), l.ctypes.data_as(_abi.f64p), C.byref(pp), C.byref(ip),
                                       C.byref(ne)), "cicy_gnp_grid_view")
        tot = int(n[0]) * int(n[1]) * int(n[2])
        ptr = np.ctypeslib.as_array(C.cast(pp, C.POINTER(C.c_int32)), shape=(tot + 1,)).copy()
        idx = (np.ctypeslib.as_array(C.cast(ip, C.POINTER(C.c_int32)), shape=(ne.value,)).copy() if ne.value else np.zeros(0, np.int32))
        return n, l, ptr, idx
    finally:
        if grid:
            lib().cicy_gnp_grid_free(grid)
        lib().cicy_gnp_set_free(h)


def gnp_closest_points(directory: str, xyz, gnp, device: int = 0):
    """Closest point of GNP gnp[i] (of `directory`/gnp_data.dat) to xyz[i] on the device
    (cicy_gnp_point_distance): returns (distance[n], closest[n, 3], flag[n]; -1 inside)."""
    h = C.c_void_p()
    check(lib().cicy_read_gnps(directory.encode(), C.byref(h)), "cicy_read_gnps")
    try:
        p = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        g = np.ascontiguousarray(gnp, dtype=np.int32)
        n = len(g)
        dist, q, fl = np.zeros(n), np.zeros((n, 3)), np.zeros(n, np.int32)
        check(lib().cicy_gnp_point_distance(device, h, n, p.ctypes.data_as(_abi.f64p), g.ctypes.data_as(_abi.i32p),
                                            dist.ctypes.data_as(_abi.f64p), q.ctypes.data_as(_abi.f64p), fl.ctypes.data_as(_abi.i32p)),
              "cicy_gnp_point_distance")
        return dist, q, fl
    finally:
        lib().cicy_gnp_set_free(h)


def gnp_pair_distance(directory: str, a, b, vdw: float, device: int = 0):
    """Upstream's GNP-GNP distance step (Get_distance_between_GNPs: GJK, EPA when
    the GNPs interpenetrate) on the device for pairs (a[i], b[i]) of the GNPs of
    `directory`/gnp_data.dat (cicy_gnp_pair_distance): returns (dist[n],
    direction[n, 3], displacement of b [n, 3], penetrating[n])."""
    h = C.c_void_p()
    check(lib().cicy_read_gnps(directory.encode(), C.byref(h)), "cicy_read_gnps")
    try:
        a = np.ascontiguousarray(a, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.int32)
        n = len(a)
        if len(b) != n:
            raise ValueError("a and b differ in length")
        d, N, m, p = np.zeros(n), np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n, np.int32)
        check(lib().cicy_gnp_pair_distance(device, h, n, a.ctypes.data_as(_abi.i32p), b.ctypes.data_as(_abi.i32p), float(vdw),
                                           d.ctypes.data_as(_abi.f64p), N.ctypes.data_as(_abi.f64p), m.ctypes.data_as(_abi.f64p),
                                           p.ctypes.data_as(_abi.i32p)), "cicy_gnp_pair_distance")
        return d, N, m, p
    finally:
        lib().cicy_gnp_set_free(h)


def gnp_junction_points(directory: str, a, b, vdw: float, sample, allow_simplex3: bool = False, device: int = 0):
    """Upstream's junction step of Label_gnps_in_window on the device for pairs
    (a[i], b[i]) (cicy_gnp_junction_points): returns (point_a [n, 3], point_b
    [n, 3], outside[n] (1: point_a outside `sample`, 2: point_b), status[n]
    (0, or the step upstream fails in))."""
    h = C.c_void_p()
    check(lib().cicy_read_gnps(directory.encode(), C.byref(h)), "cicy_read_gnps")
    try:
        a = np.ascontiguousarray(a, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.int32)
        n = len(a)
        if len(b) != n:
            raise ValueError("a and b differ in length")
        w = _abi.Cuboid(*[float(x) for x in sample])
        pa, pb, out, st = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n, np.int32), np.zeros(n, np.int32)
        check(lib().cicy_gnp_junction_points(device, h, n, a.ctypes.data_as(_abi.i32p), b.ctypes.data_as(_abi.i32p), float(vdw), C.byref(w),
                                             int(allow_simplex3), pa.ctypes.data_as(_abi.f64p), pb.ctypes.data_as(_abi.f64p),
                                             out.ctypes.data_as(_abi.i32p), st.ctypes.data_as(_abi.i32p)), "cicy_gnp_junction_points")
        return pa, pb, out, st
    finally:
        lib().cicy_gnp_set_free(h)


def gnp_contact_pairs(directory: str, inside, window, gs_min, overlap_cnt: float, overlap_gnp: float, vdw: float, tunnel: float,
                      sample=None, allow_simplex3: bool = False, n_labels_cnt=None, tol_gnp2=None, device: int = 0, init=None) -> dict:
    """GNP-GNP contact pass of Label_gnps_in_window on the device: the GNP region
    lists (cicy_gnp_sectioned_domain of `inside`) and every pair sharing a region,
    measured once, with the junction points of each contact
    (cicy_gnp_contact_pairs).  Returns the pairs within the tunnelling cutoff in
    upstream's visiting order: a, b, penetrating, dist, direction [n, 3],
    displacement [n, 3], point_a, point_b [n, 3], outside [n] (against `sample`,
    default the window), and the visit and pair counts; with `n_labels_cnt`, also
    the GNP labels of Make_gnp_clusters (cicy_gnp_labels): labels_gnp and
    n_total_labels; with `tol_gnp2`, also the GNP point structures of
    Add_gnp_junction (cicy_gnp_junction_structures, no initial points):
    gnp_points [m, 3], structure_ptr, structure_idx, junctions [k, 4] (Pa, GNPa,
    Pb, GNPb), junction_dist; `init` = (points [m, 3], structure_ptr, structure_idx)
    gives the initial points and lists (the window's boundary points) and adds
    boundary_used (bp_flags)."""
    h = C.c_void_p()
    check(lib().cicy_read_gnps(directory.encode(), C.byref(h)), "cicy_read_gnps")
    grid, pairs = C.c_void_p(), C.c_void_p()
    try:
        ins = np.ascontiguousarray(inside, dtype=np.int32)
        gs = np.ascontiguousarray(gs_min, dtype=np.float64)
        w = _abi.Cuboid(*[float(x) for x in window])
        check(lib().cicy_gnp_sectioned_domain(device, h, ins.ctypes.data_as(_abi.i32p), len(ins), C.byref(w), gs.ctypes.data_as(_abi.f64p),
                                              float(overlap_cnt), float(overlap_gnp), C.byref(grid)), "cicy_gnp_sectioned_domain")
        smp = _abi.Cuboid(*[float(x) for x in (window if sample is None else sample)])
        check(lib().cicy_gnp_contact_pairs(device, h, grid, float(vdw), float(tunnel), C.byref(smp), int(allow_simplex3), C.byref(pairs)),
              "cicy_gnp_contact_pairs")
        v = _abi.GnpPairList()
        check(lib().cicy_gnp_pairs_view(pairs, C.byref(v)), "cicy_gnp_pairs_view")
        n = int(v.n)

        def arr(ptr, ct, count, dt):
            if count == 0:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(count,)).copy()

        res = {}
        if n_labels_cnt is not None:
            gv = _abi.Gnps()
            check(lib().cicy_gnp_set_view(h, C.byref(gv)), "cicy_gnp_set_view")
            lab = np.zeros(max(gv.n, 1), np.int32)
            tot = C.c_int32()
            check(lib().cicy_gnp_labels(device, pairs, gv.n, int(n_labels_cnt), lab.ctypes.data_as(_abi.i32p), C.byref(tot)), "cicy_gnp_labels")
            res = {"labels_gnp": lab[:gv.n], "n_total_labels": int(tot.value)}
        if tol_gnp2 is not None:
            gv = _abi.Gnps()
            check(lib().cicy_gnp_set_view(h, C.byref(gv)), "cicy_gnp_set_view")
            pts = C.c_void_p()
            if init is None:
                check(lib().cicy_gnp_junction_structures(device, pairs, gv.n, float(tol_gnp2), 0, None, None, None, C.byref(pts)),
                      "cicy_gnp_junction_structures")
            else:
                ip = np.ascontiguousarray(init[0], dtype=np.float64)
                iptr = np.ascontiguousarray(init[1], dtype=np.int32)
                iidx = np.ascontiguousarray(init[2], dtype=np.int32)
                if iidx.size == 0:
                    iidx = np.zeros(1, np.int32)
                check(lib().cicy_gnp_junction_structures(device, pairs, gv.n, float(tol_gnp2), len(ip), ip.ctypes.data_as(_abi.f64p),
                                                         iptr.ctypes.data_as(_abi.i32p), iidx.ctypes.data_as(_abi.i32p), C.byref(pts)),
                      "cicy_gnp_junction_structures")
            try:
                pv = _abi.GnpPointList()
                check(lib().cicy_gnp_points_view(pts, C.byref(pv)), "cicy_gnp_points_view")
                npt, nj = int(pv.n_points), int(pv.n_junctions)
                res.update({"gnp_points": arr(pv.points, C.c_double, 3 * npt, np.float64).reshape(npt, 3),
                            "structure_ptr": arr(pv.structure_ptr, C.c_int32, pv.n_gnps + 1, np.int32),
                            "junctions": arr(pv.junctions, C.c_int32, 4 * nj, np.int32).reshape(nj, 4),
                            "junction_dist": arr(pv.junction_dist, C.c_double, nj, np.float64)})
                res["structure_idx"] = arr(pv.structure_idx, C.c_int32, int(res["structure_ptr"][-1]), np.int32)
                res["boundary_used"] = arr(pv.boundary_used, C.c_int32, int(pv.n_boundary), np.int32)
            finally:
                lib().cicy_gnp_points_free(pts)
        return {**res, "a": arr(v.a, C.c_int32, n, np.int32), "b": arr(v.b, C.c_int32, n, np.int32),
                "penetrating": arr(v.penetrating, C.c_int32, n, np.int32), "dist": arr(v.dist, C.c_double, n, np.float64),
                "direction": arr(v.direction, C.c_double, 3 * n, np.float64).reshape(n, 3),
                "displacement": arr(v.displacement, C.c_double, 3 * n, np.float64).reshape(n, 3),
                "point_a": arr(v.point_a, C.c_double, 3 * n, np.float64).reshape(n, 3),
                "point_b": arr(v.point_b, C.c_double, 3 * n, np.float64).reshape(n, 3),
                "outside": arr(v.outside, C.c_int32, n, np.int32),
                "n_visits": int(v.n_visits), "n_pairs": int(v.n_pairs)}
    finally:
        if pairs:
            lib().cicy_gnp_pairs_free(pairs)
        if grid:
            lib().cicy_gnp_grid_free(grid)
        lib().cicy_gnp_set_free(h)


def gnp_extract_window(directory: str, side: float, window_side=None) -> dict:
    """GNP part of the window extraction for window 0 (cicy_gnp_extract_window)
    for the GNPs of `directory`/gnp_data.dat in a cube of `side` um, the window
    being the sample or a centred cube of `window_side` um: gnps_inside, the
    GNPs and boundary points of each face (CSR, 7 offsets), the boundary points
    [m, 3] with their GNP and face, and each GNP's boundary points (CSR)."""
    h = C.c_void_p()
    check(lib().cicy_read_gnps(directory.encode(), C.byref(h)), "cicy_read_gnps")
    win = C.c_void_p()
    try:
        w = _abi.WindowParams()
        w.sample = _abi.Cuboid(0.0, 0.0, 0.0, side, side, side, side, side, side)
        ws = float(side if window_side is None else window_side)
        for a in range(3):
            w.win_max[a] = w.win_min[a] = ws
            w.win_delt[a] = 0.25
        check(lib().cicy_gnp_extract_window(h, C.byref(w), C.byref(win)), "cicy_gnp_extract_window")
        v = _abi.GnpWindowList()
        check(lib().cicy_gnp_window_view(win, C.byref(v)), "cicy_gnp_window_view")

        def arr(ptr, ct, count, dt):
            if count == 0:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(count,)).copy()

        n = int(v.n_points)
        bg_ptr = arr(v.boundary_gnp_ptr, C.c_int32, 7, np.int32)
        bp_ptr = arr(v.boundary_pts_ptr, C.c_int32, 7, np.int32)
        st_ptr = arr(v.structure_ptr, C.c_int32, v.n_gnps + 1, np.int32)
        return {"gnps_inside": arr(v.gnps_inside, C.c_int32, v.n_inside, np.int32),
                "boundary_gnp_ptr": bg_ptr, "boundary_gnp_idx": arr(v.boundary_gnp_idx, C.c_int32, int(bg_ptr[-1]), np.int32),
                "boundary_pts_ptr": bp_ptr, "boundary_pts_idx": arr(v.boundary_pts_idx, C.c_int32, int(bp_ptr[-1]), np.int32),
                "points": arr(v.points, C.c_double, 3 * n, np.float64).reshape(n, 3),
                "point_gnp": arr(v.point_gnp, C.c_int32, n, np.int32), "point_boundary": arr(v.point_boundary, C.c_int32, n, np.int32),
                "structure_ptr": st_ptr, "structure_idx": arr(v.structure_idx, C.c_int32, int(st_ptr[-1]), np.int32),
                "volume": arr(v.volume, C.c_double, v.n_gnps, np.float64)}
    finally:
        if win:
            lib().cicy_gnp_window_free(win)
        lib().cicy_gnp_set_free(h)
