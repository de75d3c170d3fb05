"""GNP input of the hybrid CNT/GNP configuration: cicy_read_gnps builds the GNPs
(rotation, vertices, face planes) bit for bit as upstream's Read_Network does,
checked against the golden fixture made by the upstream program
(tests/golden/make_gnp_golden.py) and, when oracle/_ref/gnp_dump is built, live
on another seed.  The fixture's GNP-GNP distances (upstream GJK / EPA) and GNP
region lists are the oracle of the GNP contact search; the distances' upstream
invariants and the CPU restatement of the region filling are checked here, and
so is the CPU restatement of the CNT-GNP contact pass (Find_adjacent_labels)
against upstream's contacts on the fixture's hybrid sample and live."""
import os
import subprocess

import numpy as np
import pytest

from cicy_geom_b200 import _abi
from cicy_geom_b200.network import generate_gnps, read_gnps, write_gnp_file

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "gnp_120_s4000000.npz")
REF = os.path.join(ROOT, "oracle", "_ref", "gnp_dump")


def golden():
    return dict(np.load(GOLDEN))


def check_against(z, ours, prefix):
    n = len(ours["l"])
    assert np.array_equal(z[prefix + "gnp_lt"].reshape(n, 2), np.stack([ours["l"], ours["t"]], 1))
    assert np.array_equal(z[prefix + "gnp_center"].reshape(n, 3), ours["center"])
    assert np.array_equal(z[prefix + "gnp_rotation"].reshape(n, 3, 3), ours["rotation"])
    assert np.array_equal(z[prefix + "gnp_vertices"].reshape(n, 8, 3), ours["vertices"])
    assert np.array_equal(z[prefix + "gnp_planes"].reshape(n, 6, 4), ours["planes"])


def test_gnp_geometry_matches_upstream_golden(tmp_path):
    z = golden()
    g = {"l": z["in_l"], "t": z["in_t"], "theta": z["in_theta"], "phi": z["in_phi"], "center": z["in_center"]}
    write_gnp_file(str(tmp_path), g)
    check_against(z, read_gnps(str(tmp_path)), "ref_")


def test_golden_gnp_distances_keep_upstream_invariants():
    z = golden()
    vdw, tunnel = float(z["meta"][3]), float(z["meta"][4])
    a, b = z["ref_pair_a"], z["ref_pair_b"]
    pen = z["ref_pair_penetrating"].astype(bool)
    d = z["ref_pair_dist"]
    n_dir = z["ref_pair_direction"].reshape(-1, 3)
    disp = z["ref_pair_displacement"].reshape(-1, 3)
    assert np.all(a < b) and len(a) > 1000
    assert pen.sum() > 100 and (~pen).sum() > 100  # both GJK-only and EPA cases
    assert np.all(d[pen] == vdw)  # interpenetrating: moved apart to the van der Waals distance
    assert np.all(d[~pen] > 0) and np.all(disp[~pen] == 0)
    assert np.allclose(np.linalg.norm(n_dir, axis=1), 1.0, atol=1e-15)
    # the move of GNP b is along the direction, by the penetration depth plus the van der Waals distance
    mag = np.linalg.norm(disp[pen], axis=1)
    assert np.all(mag > vdw)
    np.testing.assert_allclose(disp[pen] / mag[:, None], n_dir[pen], atol=1e-12)
    assert ((d <= tunnel) & ~pen).sum() > 0  # separated pairs within the tunnelling cutoff


@pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref/gnp_dump not built")
def test_gnp_geometry_matches_upstream_live(tmp_path):
    from oracle.dumpio import read_dump

    d = str(tmp_path)
    g = generate_gnps(60, 3.0, 4_000_123)
    write_gnp_file(d, g)
    with open(os.path.join(d, "sample_geom.csv"), "w") as f:
        f.write("0,0,0\n3.0,3.0,3.0\n")
    subprocess.run([REF, d, os.path.join(d, "g.bin"), "0.00034", "0.0018"], check=True, capture_output=True, timeout=600)
    check_against(read_dump(os.path.join(d, "g.bin")), read_gnps(d), "")


def test_gnp_file_errors(tmp_path):
    d = str(tmp_path)
    with pytest.raises(_abi.CicyError, match="gnp_data.dat"):
        read_gnps(d)
    write_gnp_file(d, generate_gnps(5, 2.0, 1))
    path = os.path.join(d, "gnp_data.dat")
    data = open(path, "rb").read()
    open(path, "wb").write(data[:-8])
    with pytest.raises(_abi.CicyError, match="end-of-file of gnp_data.dat"):
        read_gnps(d)


def test_gnp_contact_grid_oracle_matches_upstream_golden():
    """The CPU restatement of upstream's GNP region filling (oracle/gnp_oracle.py)
    gives upstream's region lists on the fixture."""
    from oracle import gnp_oracle as G

    z = golden()
    side, gs, ov_cnt, ov_gnp = float(z["meta"][1]), float(z["meta"][5]), float(z["meta"][6]), float(z["meta"][7])
    win = [0.0, 0.0, 0.0, side, side, side, side, side, side]
    n, l = G.region_grid(win, [gs] * 3, ov_cnt, ov_gnp)
    assert list(n) == list(z["ref_sd_n_regions"]) and np.array_equal(l, z["ref_sd_l_regions"])
    N = len(z["in_l"])
    regs = G.fill_sectioned_domain_gnps(win, z["ref_gnp_vertices"].reshape(N, 8, 3), z["in_l"], z["in_t"], range(N), n, l, ov_gnp)
    ptr, idx = z["ref_sd_ptr"], z["ref_sd_idx"]
    assert len(regs) == len(ptr) - 1
    assert all(list(idx[ptr[k]:ptr[k + 1]]) == regs[k] for k in range(len(regs)))
    assert len(idx) > 10000


def test_golden_gnp_closest_points_keep_upstream_invariants():
    """Upstream's closest GNP points: inside points flagged -1 at distance 0, the
    others at the returned distance from the query, every branch represented."""
    z = golden()
    q = z["in_queries"]
    fl, d, c = z["ref_query_flag"], z["ref_query_dist"], z["ref_query_point"].reshape(-1, 3)
    assert set(np.unique(fl)) == {-1, 0}
    assert np.all(d[fl == -1] == 0)
    out = fl == 0
    assert out.sum() > 500 and (~out).sum() > 500
    np.testing.assert_allclose(np.linalg.norm(q[out, :3] - c[out], axis=1), d[out], rtol=1e-9, atol=1e-12)


def hybrid_inputs(z, directory):
    """The fixture's CNT network as upstream reads it (regenerated from its seed,
    checked against the stored hash), its CNT region lists from the CPU
    restatement, and the fixture's GNP region lists, vertices and planes."""
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_gnp_golden as M
    from oracle import cicy_oracle as O

    net = dict(M.hybrid_network(directory))
    assert M.net_hash(net) == str(z["cnt_sha256"])
    side, gs, ov_cnt, ov_gnp = float(z["meta"][1]), float(z["meta"][5]), float(z["meta"][6]), float(z["meta"][7])
    net["cnts_inside"] = np.arange(len(net["radii"]))
    net["window"] = np.array([0.0, 0.0, 0.0, side, side, side, side, side, side])
    _, _, regs = O.contact_grid(net, {"gs_min": (gs,) * 3, "gs_overlap_cnt": ov_cnt, "gs_overlap_gnp": ov_gnp})
    ptr = np.cumsum([0] + [len(r) for r in regs])
    idx = np.concatenate([np.asarray(r, dtype=np.int64) for r in regs])
    assert M.arr_hash(ptr, idx) == str(z["mix_sd_sha256"])  # upstream's CNT region lists of the hybrid grid
    sp, si = z["ref_sd_ptr"], z["ref_sd_idx"]
    sd_gnp = [si[sp[k]:sp[k + 1]].tolist() for k in range(len(sp) - 1)]
    n = len(z["in_l"])
    return net, regs, sd_gnp, z["ref_gnp_vertices"].reshape(n, 8, 3), z["ref_gnp_planes"].reshape(n, 6, 4)


def test_mixed_contacts_oracle_matches_upstream_golden(tmp_path):
    """The CPU restatement of upstream's CNT-GNP contact pass
    (oracle/gnp_oracle.py find_adjacent_labels) gives upstream's contacts on the
    fixture: the same (point, GNP) pairs, contact-point numbers, junction
    distances and closest GNP points, bit for bit."""
    from oracle import gnp_oracle as G

    z = golden()
    net, regs, sd_gnp, V, F = hybrid_inputs(z, str(tmp_path))
    xyz = np.stack([net["x"], net["y"], net["z"]], 1)
    out = G.find_adjacent_labels(xyz.tolist(), net["flag"], net["radii"], regs, sd_gnp, V.tolist(), F.tolist(),
                                 float(z["meta"][3]), float(z["meta"][4]))
    P, g, i, d = z["ref_mix_point"], z["ref_mix_gnp"], z["ref_mix_index"], z["ref_mix_dist"]
    cp = z["ref_mix_contact_points"].reshape(-1, 3)
    assert len(out) == len(P) > 1000
    for k in range(len(P)):
        num, dj, q = out[(int(P[k]), int(g[k]))]
        assert num == i[k] and dj == d[k] and tuple(q) == tuple(cp[num])


def test_golden_mixed_contacts_keep_upstream_invariants():
    z = golden()
    vdw, tunnel = float(z["meta"][3]), float(z["meta"][4])
    P, g, i, d = z["ref_mix_point"], z["ref_mix_gnp"], z["ref_mix_index"], z["ref_mix_dist"]
    assert np.array_equal(np.sort(i), np.arange(len(i)))  # one contact point per (point, GNP) pair
    assert len(set(zip(P.tolist(), g.tolist()))) == len(P)
    assert np.all(d >= vdw) and np.all(d <= tunnel)
    assert (d == vdw).sum() > 100 and (d > vdw).sum() > 100  # clamped and tunnelling junctions


@pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref/gnp_dump not built")
def test_mixed_contacts_oracle_matches_upstream_live(tmp_path):
    """Another seed and sample: the restatement against the upstream program run here."""
    from cicy_geom_b200.network import NetworkConfig, generate_cnt_network, read_network_files, write_read_network_files
    from oracle import cicy_oracle as O, gnp_oracle as G
    from oracle.dumpio import read_dump

    d, side, vdw, tunnel, gs = str(tmp_path), 1.5, 0.00034, 0.0018, 0.05
    cfg = NetworkConfig(side=side, n_cnts=250, seed=4_000_321)
    write_read_network_files(d, generate_cnt_network(cfg), cfg)
    write_gnp_file(d, generate_gnps(50, side, 4_000_322))
    ov_cnt, ov_gnp = 2 * cfg.radius + tunnel, gs / np.sqrt(8.0)
    subprocess.run([REF, d, os.path.join(d, "g.bin"), repr(vdw), repr(tunnel), repr(gs), repr(ov_cnt), repr(float(ov_gnp))],
                   check=True, capture_output=True, timeout=600)
    z = read_dump(os.path.join(d, "g.bin"))
    net = dict(read_network_files(d).arrays())
    net["cnts_inside"] = np.arange(len(net["radii"]))
    net["window"] = np.array([0.0, 0.0, 0.0, side, side, side, side, side, side])
    _, _, regs = O.contact_grid(net, {"gs_min": (gs,) * 3, "gs_overlap_cnt": ov_cnt, "gs_overlap_gnp": float(ov_gnp)})
    assert np.array_equal(np.cumsum([0] + [len(r) for r in regs]), z["mix_sd_cnt_ptr"])
    sp, si = z["sd_ptr"], z["sd_idx"]
    n = len(z["gnp_lt"]) // 2
    out = G.find_adjacent_labels(np.stack([net["x"], net["y"], net["z"]], 1).tolist(), net["flag"], net["radii"], regs,
                                 [si[sp[k]:sp[k + 1]].tolist() for k in range(len(sp) - 1)],
                                 z["gnp_vertices"].reshape(n, 8, 3).tolist(), z["gnp_planes"].reshape(n, 6, 4).tolist(), vdw, tunnel)
    ref = {(int(a), int(b)): (int(c), float(e)) for a, b, c, e in zip(z["mix_point"], z["mix_gnp"], z["mix_index"], z["mix_dist"])}
    assert len(ref) > 200 and {k: v[:2] for k, v in out.items()} == ref
    cp = z["mix_contact_points"].reshape(-1, 3)
    assert all(tuple(v[2]) == tuple(cp[v[0]]) for v in out.values())


def test_gnp_distance_oracle_matches_upstream_golden():
    """The CPU restatement of upstream's GNP-GNP distance step (GJK, EPA for the
    interpenetrating pairs, the move apart) gives upstream's doubles on every
    candidate pair of the fixture."""
    from oracle import gnp_oracle as G

    z = golden()
    V = z["ref_gnp_vertices"].reshape(-1, 8, 3).tolist()
    vdw = float(z["meta"][3])
    for i, (a, b) in enumerate(zip(z["ref_pair_a"], z["ref_pair_b"])):
        d, N, m, p = G.pair_distance(V[a], V[b], vdw)
        assert int(p) == z["ref_pair_penetrating"][i] and d == z["ref_pair_dist"][i]
        assert tuple(N) == tuple(z["ref_pair_direction"][3 * i:3 * i + 3])
        assert tuple(m) == tuple(z["ref_pair_displacement"][3 * i:3 * i + 3])


def test_gnp_contact_pairs_oracle_agrees_with_upstream_golden():
    """The restated GNP-GNP contact pass of Label_gnps_in_window over upstream's
    region lists: exactly the fixture's pairs within the tunnelling cutoff that
    share a region, each once, with upstream's distances."""
    from oracle import gnp_oracle as G

    z = golden()
    V = z["ref_gnp_vertices"].reshape(-1, 8, 3).tolist()
    sp, si = z["ref_sd_ptr"], z["ref_sd_idx"]
    sd = [si[sp[k]:sp[k + 1]].tolist() for k in range(len(sp) - 1)]
    vdw, tunnel = float(z["meta"][3]), float(z["meta"][4])
    out = G.contact_pairs(sd, V, vdw, tunnel)
    ref = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(z["ref_pair_a"], z["ref_pair_b"]))}
    shared = {(min(g[j], g[k]), max(g[j], g[k])) for g in sd for j in range(len(g)) for k in range(j + 1, len(g))}
    within = {k for k, i in ref.items() if z["ref_pair_dist"][i] <= tunnel}
    assert {(a, b) for a, b, *_ in out} == within & shared and len(out) == len(within & shared) > 500
    for a, b, d, N, m, p in out:
        i = ref[(a, b)]
        assert d == z["ref_pair_dist"][i] and int(p) == z["ref_pair_penetrating"][i]
        assert tuple(N) == tuple(z["ref_pair_direction"][3 * i:3 * i + 3])


KAT = os.path.join(ROOT, "tests", "golden", "gnp_junction_cases.npz")


@pytest.mark.parametrize("path,side", [(GOLDEN, 2.0), (KAT, 12.0)])
def test_junction_oracle_matches_upstream_golden(path, side):
    """The CPU restatement of upstream's junction step (Find_junction_points_for_gnps
    on the moved GNP, the point moved back, the outside test) against upstream on
    the random fixture's 555 contacts (vertex-face, crossing edges) and the 10
    hand-placed cases (face-face, edge-face, parallel edges with upstream's NaN,
    vertex-vertex, vertex-edge, and a face-face case upstream fails on); points
    compared as bit patterns."""
    from oracle import gnp_oracle as G

    z = dict(np.load(path))
    V, F = z["ref_gnp_vertices"].reshape(-1, 8, 3).tolist(), z["ref_gnp_planes"].reshape(-1, 6, 4).tolist()
    vdw = 0.00034
    for i, p in enumerate(z["ref_junc_pair"]):
        a, b = z["ref_pair_a"][p], z["ref_pair_b"][p]
        r = G.pair_junction(V[a], F[a], V[b], F[b], vdw, (0.0, 0.0, 0.0), (side, side, side))
        assert (r is not None) == bool(z["ref_junc_ok"][i])
        if r is not None:
            mine = np.array(list(r[0]) + list(r[1]))
            assert np.array_equal(mine.view(np.int64), z["ref_junc_points"][6 * i:6 * i + 6].view(np.int64))
            assert r[2] == z["ref_junc_outside"][i]


LABELS = os.path.join(ROOT, "tests", "golden", "gnp_hybrid_labels.npz")


def hybrid_oracle_labels(z, directory, network):
    """The labels of a hybrid sample from the CPU restatements alone: CNT region
    lists and CNT labels (oracle/cicy_oracle.py), GNP region lists, GNP-GNP
    contacts and junction points, CNT-GNP contacts, then the GNP and mixed HK76
    passes (oracle/gnp_oracle.py), on upstream's GNPs."""
    from oracle import cicy_oracle as O, gnp_oracle as G

    side, gs, ov_cnt, ov_gnp = float(z["meta"][1]), float(z["meta"][5]), float(z["meta"][6]), float(z["meta"][7])
    vdw, tunnel = float(z["meta"][3]), float(z["meta"][4])
    net = dict(network(directory))
    net["cnts_inside"] = np.arange(len(net["radii"]))
    win = [0.0, 0.0, 0.0, side, side, side, side, side, side]
    net["window"] = np.array(win)
    p = {"gs_min": (gs,) * 3, "gs_overlap_cnt": ov_cnt, "gs_overlap_gnp": ov_gnp, "vdw": vdw, "tunnel": tunnel}
    n, l, regs = O.contact_grid(net, p)
    lab_cnt, n_cnt, _, _ = O.label_cnts(net, p, regs)
    N = len(z["in_l"])
    V, F = z["ref_gnp_vertices"].reshape(N, 8, 3), z["ref_gnp_planes"].reshape(N, 6, 4).tolist()
    sd_gnp = G.fill_sectioned_domain_gnps(win, V, z["in_l"], z["in_t"], range(N), n, l, ov_gnp)
    V = V.tolist()
    pairs = G.contact_pairs(sd_gnp, V, vdw, tunnel)
    outside = [G.pair_junction(V[a], F[a], V[b], F[b], vdw, win[0:3], win[6:9])[2] for a, b, *_ in pairs]
    lab_gnp, n_total = G.gnp_labels(N, [(a, b) for a, b, *_ in pairs], outside, n_cnt)
    mix = G.find_adjacent_labels(np.stack([net["x"], net["y"], net["z"]], 1).tolist(), net["flag"], net["radii"], regs, sd_gnp, V, F, vdw,
                                 tunnel)
    contacts = [(int(net["flag"][P]), g) for (P, g), _ in sorted(mix.items(), key=lambda kv: kv[1][0])]
    hybrid_oracle_labels.last = {"pairs": pairs, "outside": outside, "mix": mix, "flag": net["flag"], "V": V, "F": F, "win": win}
    return (lab_cnt, n_cnt), (lab_gnp, n_total), G.mixed_labels(lab_cnt, lab_gnp, n_total, contacts)


@pytest.mark.parametrize("path", [GOLDEN, LABELS])
def test_hybrid_labels_oracle_matches_upstream_golden(tmp_path, path):
    """CNT, GNP and mixed labels of a hybrid sample restated on the CPU against
    upstream's Make_cnt_clusters, Make_gnp_clusters and Make_mixed_clusters: the
    120-GNP fixture (one mixed cluster) and the sparse one (28 CNT and 4 GNP
    labels into 25 mixed clusters)."""
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_gnp_golden as M

    z = dict(np.load(path))
    network = M.hybrid_network if path == GOLDEN else M.sparse_network
    assert M.net_hash(network(str(tmp_path))) == str(z["cnt_sha256"])
    (lc, nc), (lg, nt), (mc, mg, nm) = hybrid_oracle_labels(z, str(tmp_path), network)
    assert list(lc) == list(z["ref_lab_cnt"]) and nc == z["ref_lab_counts"][0]
    assert list(lg) == list(z["ref_lab_gnp"]) and nt == z["ref_lab_counts"][1]
    assert list(mc) == list(z["ref_mixlab_cnt"]) and list(mg) == list(z["ref_mixlab_gnp"]) and nm == z["ref_mixlab_count"][0]


@pytest.mark.parametrize("path", [GOLDEN, LABELS])
def test_gnp_structures_oracle_matches_upstream_golden(tmp_path, path):
    """Add_gnp_junction (GNP point lists with the interpenetrating pairs' points
    merged within tol_gnp) and Compress_mixed_contacts (one junction per run of
    CNT points per GNP) restated on the CPU against upstream's points_gnp,
    structure_gnp, junctions_gnp and junctions_mixed."""
    import sys

    from oracle import gnp_oracle as G

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_gnp_golden as M

    z = dict(np.load(path))
    hybrid_oracle_labels(z, str(tmp_path), M.hybrid_network if path == GOLDEN else M.sparse_network)
    r = hybrid_oracle_labels.last
    V, F, win, vdw = r["V"], r["F"], r["win"], float(z["meta"][3])
    contacts = []
    for (a, b, d, N, m, pen), o in zip(r["pairs"], r["outside"]):
        PA, PB, _ = G.pair_junction(V[a], F[a], V[b], F[b], vdw, win[0:3], win[6:9])
        contacts.append((a, b, d, pen, PA, PB, o))
    tol = 1.5 * float(np.max(z["in_t"]))  # Input_Reader.cpp:1161
    pts, st, jn, _ = G.add_gnp_junctions(contacts, len(V), tol * tol)
    assert np.array_equal(np.array(pts), z["ref_gnpjn_points"].reshape(-1, 3))
    assert np.array_equal(np.cumsum([0] + [len(x) for x in st]), z["ref_gnpjn_structure_ptr"])
    assert np.array_equal(np.array([x for y in st for x in y]), z["ref_gnpjn_structure_idx"])
    assert np.array_equal(np.array([j[:4] for j in jn]), z["ref_junctions_gnp"].reshape(-1, 4))
    assert [j[4] for j in jn] == list(z["ref_junctions_gnp_dist"])
    pts2, st2, jm, _ = G.compress_mixed_contacts(r["mix"], r["flag"], 5, pts, st)
    assert np.array_equal(np.array(pts2), z["ref_mixjn_points"].reshape(-1, 3))
    assert np.array_equal(np.array([x for y in st2 for x in y]), z["ref_mixjn_structure_idx"])
    assert np.array_equal(np.array([j[:4] for j in jm]), z["ref_junctions_mixed"].reshape(-1, 4)) and len(jm) > 10
    assert [j[4] for j in jm] == list(z["ref_junctions_mixed_dist"])


@pytest.mark.parametrize("path", [GOLDEN, LABELS])
def test_triangulation_oracle_matches_upstream_golden(path):
    """Triangulation::Generate_3d_trangulation restated on the CPU (points onto
    the mid-plane, Bowyer-Watson from the supertriangle, first-occurrence edges;
    all pairs for four points or fewer) against upstream's edges for every GNP's
    final point list (after the GNP and mixed junctions)."""
    from oracle import gnp_oracle as G

    z = dict(np.load(path))
    N = len(z["in_l"])
    pts = z["ref_mixjn_points"].reshape(-1, 3)
    sp, si = z["ref_mixjn_structure_ptr"], z["ref_mixjn_structure_idx"]
    rot, cen = z["ref_gnp_rotation"].reshape(N, 3, 3), z["ref_gnp_center"].reshape(N, 3)
    F, lt = z["ref_gnp_planes"].reshape(N, 6, 4), z["ref_gnp_lt"].reshape(N, 2)
    tp, te = z["ref_tri_ptr"], z["ref_tri_edges"].reshape(-1, 2)
    assert tp[-1] > 100
    for g in range(N):
        e = G.triangulate_gnp(pts, si[sp[g]:sp[g + 1]], lt[g, 0], cen[g], rot[g], F[g, 0, :3])
        assert e == [tuple(x) for x in te[tp[g]:tp[g + 1]].tolist()]


WINDOWS = os.path.join(ROOT, "tests", "golden", "gnp_windows.npz")


def _window_case(tmp_path, k):
    """(GNP inputs written to tmp_path, sample side, window side, upstream arrays) of a window case;
    k = -1: the 120-GNP fixture with the sample as the window."""
    if k < 0:
        z = golden()
        g = {"l": z["in_l"], "t": z["in_t"], "theta": z["in_theta"], "phi": z["in_phi"], "center": z["in_center"]}
        ref = {key[len("ref_"):]: v for key, v in z.items() if key.startswith("ref_win_")}
        side, ws = float(z["meta"][1]), None
    else:
        z = dict(np.load(WINDOWS))
        g = {key: z[f"c{k}_in_{key}"] for key in ("l", "t", "theta", "phi", "center")}
        ref = {key[len(f"c{k}_ref_"):]: v for key, v in z.items() if key.startswith(f"c{k}_ref_")}
        side, ws = float(z[f"c{k}_meta"][1]), float(z[f"c{k}_meta"][3])
    write_gnp_file(str(tmp_path), g)
    return side, ws, ref


@pytest.mark.parametrize("k", [-1, 0, 1])
def test_gnp_window_extraction_matches_upstream_golden(tmp_path, k):
    """cicy_gnp_extract_window (host) against upstream's Fill_gnps_inside:
    gnps_inside, boundary_gnp, boundary_gnp_pts, structure_gnp, the boundary
    points and the volumes inside the window bit for bit, for the whole sample
    and two centred smaller windows."""
    from cicy_geom_b200.network import gnp_extract_window

    side, ws, ref = _window_case(tmp_path, k)
    w = gnp_extract_window(str(tmp_path), side, ws)
    assert np.array_equal(w["gnps_inside"], ref["win_inside"])
    for mine, theirs in (("boundary_gnp", "win_bgnp"), ("boundary_pts", "win_bpts"), ("structure", "win_structure")):
        assert np.array_equal(w[mine + "_ptr"], ref[theirs + "_ptr"]) and np.array_equal(w[mine + "_idx"], ref[theirs + "_idx"])
    assert np.array_equal(w["points"].ravel().view(np.int64), ref["win_points"].view(np.int64)) and len(w["points"]) > 100
    vol = w["volume"]
    set_ = ~np.isnan(vol)  # the GNPs whose volume the extraction sets (Approximate_gnp_volume_inside_sample)
    assert np.array_equal(set_, ~np.isnan(ref["win_volume"])) and set_.sum() > 50
    assert np.array_equal(vol[set_].view(np.int64), ref["win_volume"][set_].view(np.int64))


def test_gnp_entry_points_reject_bad_input(tmp_path):
    """Argument checks of the GNP entry points that run before any device work:
    null handles, out-of-range GNP indices, malformed initial structures and
    multi-window parameters fail with CICY_E_INPUT and a message."""
    import ctypes as C

    from cicy_geom_b200.network import gnp_extract_window

    L = _abi.lib()
    d = str(tmp_path)
    write_gnp_file(d, generate_gnps(6, 2.0, 11))
    h = C.c_void_p()
    assert L.cicy_read_gnps(d.encode(), C.byref(h)) == 0
    try:
        out = C.c_void_p()
        assert L.cicy_gnp_labels(0, None, 6, 0, None, None) == 1
        assert L.cicy_gnp_junction_structures(0, None, 6, 0.1, 0, None, None, None, C.byref(out)) == 1
        assert L.cicy_gnp_contact_pairs(0, h, None, 0.00034, 0.0018, None, 0, C.byref(out)) == 1
        assert L.cicy_gnp_extract_window(None, None, C.byref(out)) == 1
        a = np.array([0, 7], np.int32)  # GNP 7 of 6
        b = np.array([1, 2], np.int32)
        r = np.zeros(8)
        i = np.zeros(2, np.int32)
        assert L.cicy_gnp_pair_distance(0, h, 2, a.ctypes.data_as(_abi.i32p), b.ctypes.data_as(_abi.i32p), 0.00034,
                                        r.ctypes.data_as(_abi.f64p), r.ctypes.data_as(_abi.f64p), r.ctypes.data_as(_abi.f64p),
                                        i.ctypes.data_as(_abi.i32p)) == 1
        assert b"out of range" in L.cicy_host_last_error()
        q = np.zeros(3)
        g = np.array([9], np.int32)
        assert L.cicy_gnp_point_distance(0, h, 1, q.ctypes.data_as(_abi.f64p), g.ctypes.data_as(_abi.i32p), r.ctypes.data_as(_abi.f64p),
                                         r.ctypes.data_as(_abi.f64p), i.ctypes.data_as(_abi.i32p)) == 1
    finally:
        L.cicy_gnp_set_free(h)
    with pytest.raises(_abi.CicyError, match="single-window"):
        w = _abi.WindowParams()
        w.sample = _abi.Cuboid(0.0, 0.0, 0.0, 2.0, 2.0, 2.0, 2.0, 2.0, 2.0)
        for k in range(3):
            w.win_max[k], w.win_min[k], w.win_delt[k] = 2.0, 1.0, 0.25
        h2, out2 = C.c_void_p(), C.c_void_p()
        assert L.cicy_read_gnps(d.encode(), C.byref(h2)) == 0
        try:
            _abi.check(L.cicy_gnp_extract_window(h2, C.byref(w), C.byref(out2)), "cicy_gnp_extract_window")
        finally:
            L.cicy_gnp_set_free(h2)
    assert len(gnp_extract_window(d, 2.0)["gnps_inside"]) > 0


FLOW = os.path.join(ROOT, "tests", "golden", "gnp_hybrid_flow.npz")


@pytest.mark.parametrize("tag", ["s", "m"])
def test_hybrid_chain_matches_upstream_flow(tmp_path, tag):
    """The whole hybrid chain against upstream's own stage sequence for
    GNP_CNT_mix (window extraction, contact grid, Determine_clusters_and_
    percolation): the window extraction of CNTs and GNPs on the host
    (cicy_extract_window, cicy_gnp_extract_window), then the CPU restatements of
    the CNT contacts, labels and junctions, the GNP contact pass, junction
    points and labels, the GNP point lists with the boundary points, the CNT-GNP
    contacts, mixed labels and junctions, and the percolation with junction
    groups: equal to upstream's clusters, isolated particles, families and
    junction groups on both hybrid samples."""
    import sys

    from cicy_geom_b200.network import gnp_extract_window, read_network_files
    from oracle import cicy_oracle as O, gnp_oracle as G
    from oracle.dumpio import csr

    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_gnp_golden as M

    fz = dict(np.load(FLOW))
    z = {k[len(tag) + 1:]: v for k, v in fz.items() if k.startswith(tag + "_")}
    d = str(tmp_path)
    if tag == "m":
        M.hybrid_network(d)
        write_gnp_file(d, generate_gnps(M.N, M.SIDE, M.SEED))
        cfg = M.cnt_config()
    else:
        M.sparse_network(d)
        write_gnp_file(d, generate_gnps(M.SPARSE_N, M.SIDE, M.SPARSE_SEED, l_range=(0.3, 0.5)))
        cfg = M.sparse_config()
    side = M.SIDE
    a = dict(read_network_files(d).extract_window(cfg).arrays())
    bc = [a["boundary_cnt_idx"][a["boundary_cnt_ptr"][f]:a["boundary_cnt_ptr"][f + 1]].tolist() for f in range(6)]
    assert np.array_equal(a["cnts_inside"], z["flow_cnts_inside"]) and [list(x) for x in csr(z, "flow_boundary_cnt")] == bc
    gw = gnp_extract_window(d, side)
    bg = [gw["boundary_gnp_idx"][gw["boundary_gnp_ptr"][f]:gw["boundary_gnp_ptr"][f + 1]].tolist() for f in range(6)]
    assert np.array_equal(gw["gnps_inside"], z["flow_gnps_inside"]) and [list(x) for x in csr(z, "flow_boundary_gnp")] == bg
    vdw, tun, ovg = M.VDW, M.TUNNEL, float(M.OVERLAP_GNP)
    p = {"gs_min": (M.GS_MIN,) * 3, "gs_overlap_cnt": M.OVERLAP_CNT, "gs_overlap_gnp": ovg, "vdw": vdw, "tunnel": tun, "min_points": 5}
    n, l, regs = O.contact_grid(a, p)
    lab_cnt, n_cnt, pc, ce = O.label_cnts(a, p, regs)
    jc, el_cnt = O.compress_junctions(a, p, pc, ce)
    Vg = read_gnps(d)
    sd_gnp = G.fill_sectioned_domain_gnps(a["window"], Vg["vertices"], Vg["l"], Vg["t"], gw["gnps_inside"], n, l, ovg)
    V, F = Vg["vertices"].tolist(), Vg["planes"].tolist()
    cts = []
    for pa, pb, dd, _, _, pen in G.contact_pairs(sd_gnp, V, vdw, tun):
        PA, PB, o = G.pair_junction(V[pa], F[pa], V[pb], F[pb], vdw, (0.0, 0.0, 0.0), (side, side, side))
        cts.append((pa, pb, dd, pen, PA, PB, o))
    NG = len(V)
    lab_gnp, n_total = G.gnp_labels(NG, [(x[0], x[1]) for x in cts], [x[6] for x in cts], n_cnt)
    sp = gw["structure_ptr"]
    tol = 1.5 * float(np.max(Vg["t"]))
    pts, st, jg, _ = G.add_gnp_junctions(cts, NG, tol * tol, [tuple(q) for q in gw["points"]],
                                         [gw["structure_idx"][sp[g]:sp[g + 1]].tolist() for g in range(NG)])
    mix = G.find_adjacent_labels(np.stack([a["x"], a["y"], a["z"]], 1).tolist(), a["flag"], a["radii"], regs, sd_gnp, V, F, vdw, tun)
    order = sorted(mix.items(), key=lambda kv: kv[1][0])
    mc, mg, nm = G.mixed_labels(lab_cnt, lab_gnp, n_total, [(int(a["flag"][P]), g) for (P, g), _ in order])
    _, st_mix, jm, el_mix = G.compress_mixed_contacts(mix, a["flag"], 5, pts, st)
    res = G.mixed_percolation(nm, a["cnts_inside"], gw["gnps_inside"], mc, mg, bc, bg, [(j[1], j[3]) for j in jc], [(j[1], j[3]) for j in jg],
                              [(j[1], j[3]) for j in jm])
    assert res["family"] == list(z["flow_family"]) and len(res["family"]) >= 1
    for key in ("clusters_cnt", "clusters_gnp", "isolated_cnt", "isolated_gnp", "cluster_cnt_junctions", "cluster_gnp_junctions",
                "cluster_mix_junctions"):
        assert res[key] == [list(x) for x in csr(z, "flow_" + key)], key
    # Remove_gnp_points_in_non_relevant_boundaries: the point lists and boundary points the
    # electrical stage starts from (upstream's, tests/golden/gnp_hybrid_electrical.npz)
    _, _, _, bp = G.add_gnp_junctions(cts, NG, tol * tol, [tuple(q) for q in gw["points"]],
                                      [gw["structure_idx"][sp[g]:sp[g + 1]].tolist() for g in range(NG)])
    bpp, bpi = gw["boundary_pts_ptr"], gw["boundary_pts_idx"]
    pb = [[] for _ in range(NG)]
    for P, g, b in zip(range(len(gw["point_gnp"])), gw["point_gnp"], gw["point_boundary"]):
        if b >= 0:
            pb[int(g)].append((P, int(b)))
    st2 = [list(x) for x in st_mix]
    G.remove_nonrelevant_boundary_points(res["clusters_gnp"], res["family"], pb, st2, bp)
    ez = {k[2:]: v for k, v in np.load(os.path.join(ROOT, "tests", "golden", "gnp_hybrid_electrical.npz")).items() if k.startswith(tag + "_")}
    assert st2 == [list(x) for x in csr(ez, "e_structure_gnp_start")]
    epb = csr(ez, "e_pts_boundary")
    assert [[v for q in x for v in q] for x in pb] == [list(x) for x in epb]
    # elements_cnt: the CNT junctions' points, every mixed junction's CNT point, then
    # Complete_cnt_elements (after Make_mixed_clusters for GNP_CNT_mix) adds the end points
    elems = [set(el_cnt.get(c, ())) for c in range(len(a["radii"]))]
    for c, P in el_mix:
        elems[c].add(P)
    sp_c, si_c = a["structure_ptr"], a["structure_idx"]
    for c in range(len(elems)):
        if elems[c]:
            elems[c] |= {int(si_c[sp_c[c]]), int(si_c[sp_c[c + 1] - 1])}
    assert [sorted(e) for e in elems] == [list(x) for x in csr(ez, "e_elements_start")]


def test_hybrid_flow_golden_carries_upstream_resistances():
    """The end-to-end target of the hybrid path: upstream's Electrical_analysis
    on both hybrid samples gives a finite resistance along x (the percolating
    direction of both) and the matrix resistance rho_m L / A along y and z,
    which were not requested."""
    z = dict(np.load(FLOW))
    for tag in ("s", "m"):
        r = z[f"{tag}_flow_resistances"]
        assert len(r) == 3 and 0 < r[0] < 1e6
        assert np.allclose(r[1:], 1.03e20 * 2.0 / 4.0)


def test_gnp_resistance_oracle_matches_upstream_golden():
    """The GNP resistor of a triangulation edge restated on the CPU against
    upstream's Calculate_resistance_gnp on the 120-GNP fixture's edges (radii as
    Fill_2d_matrices_gnp takes them), bit for bit, and upstream's failure on
    coincident points."""
    from oracle import gnp_oracle as G

    z = dict(np.load(os.path.join(ROOT, "tests", "golden", "gnp_resistors.npz")))
    cases, ref = z["cases"], z["ref_resistance"]
    assert len(cases) > 1000
    for c, r in zip(cases, ref):
        R = G.gnp_resistance(c[0:3], c[3:6], c[6], c[7], c[8], c[9])
        if r == -1.0:
            assert R is None
        else:
            assert np.float64(R).view(np.int64) == np.float64(r).view(np.int64)
