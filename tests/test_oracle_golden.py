"""Pins the CPU oracle against the reference's own known-answer tests and
against brute force under the reference's floating-point formula
(test/build.jl:13-28, test/edges_cpu.jl:14-79).  CPU only."""
import numpy as np
import pytest

from conftest import clustered, lattice, uniform
from kats import coords_of, f32, load_kats

K = load_kats()


def test_morton3_roundtrip_and_codes(oracle_mod):
    for c in K["morton3_roundtrip"]["cases"]:
        x, y, z = c["xyz"]
        code = oracle_mod.morton_encode3(x, y, z)
        assert code == c["code"]
        assert oracle_mod.morton_decode3(code) == (x, y, z)


def test_morton3_monotone_along_x(oracle_mod):
    k = K["morton3_monotone_x"]
    prev = oracle_mod.morton_encode3(0, k["y"], k["z"])
    for x in range(1, k["x_max"] + 1):
        cur = oracle_mod.morton_encode3(x, k["y"], k["z"])
        assert cur > prev
        prev = cur


def test_morton2_roundtrip_codes_topbits(oracle_mod):
    for c in K["morton2_roundtrip"]["cases"]:
        x, y = c["xy"]
        code = oracle_mod.morton_encode2(x, y)
        assert code == c["code"]
        assert oracle_mod.morton_decode2(code) == (x, y)
    for x, y in K["morton2_top_bits_zero"]["cases"]:
        assert oracle_mod.morton_encode2(x, y) >> 62 == 0
    k = K["morton2_monotone_x"]
    prev = oracle_mod.morton_encode2(0, k["y"])
    for x in range(1, k["x_max"] + 1):
        cur = oracle_mod.morton_encode2(x, k["y"])
        assert cur > prev
        prev = cur


@pytest.mark.parametrize("name", ["bin_point3", "bin_point2"])
def test_bin_point(oracle_mod, name):
    for c in K[name]["cases"]:
        cell = oracle_mod.bin_point_f32([f32(v) for v in c["p"]], [f32(v) for v in c["o"]], f32(c["inv_cs"]))
        assert list(cell) == c["cell"]


def test_bin_point_inexact(oracle_mod):
    # floor(Int32, x) throws InexactError out of range (src/morton.jl:84).
    with pytest.raises(OverflowError):
        oracle_mod.bin_point_f32([np.float32(3e9)], [np.float32(0)], np.float32(1))
    with pytest.raises(OverflowError):
        oracle_mod.bin_point_f32([np.float32(np.nan)], [np.float32(0)], np.float32(1))


def _neighbors(oracle_mod, x, r, i, exclude_self=True):
    t = oracle_mod.build_tree(x, r)
    e = oracle_mod.build_edges(t, x, exclude_self=exclude_self)
    return sorted(int(s) for s, rc in zip(e["senders"], e["receivers"]) if rc == i)


@pytest.mark.parametrize("name", ["exact_radius_included_3d", "just_past_radius_excluded_3d",
                                  "exact_radius_included_2d", "docstring_example", "single_point"])
def test_edge_case_neighbors(oracle_mod, name):
    c = K[name]
    x = coords_of(c)
    for i, want in c["neighbors"].items():
        assert _neighbors(oracle_mod, x, f32(c["r"]), int(i)) == want
    if "n_nodes" in c:
        assert oracle_mod.build_tree(x, f32(c["r"])).n_nodes == c["n_nodes"]


@pytest.mark.parametrize("name", ["coincident_3d", "coincident_2d"])
def test_coincident(oracle_mod, name):
    c = K[name]
    x = np.zeros((c["n"], c["ndims"]), np.float32)
    t = oracle_mod.build_tree(x, f32(c["r"]))
    # bit exhaustion: one leaf at max level below a single-child chain
    assert sorted(t.perm.tolist()) == list(range(1, c["n"] + 1))
    e = oracle_mod.build_edges(t, x, exclude_self=True)
    cnt = np.bincount(e["receivers"], minlength=c["n"] + 1)[1:]
    assert (cnt == c["n"] - 1).all()


def test_empty_sets(oracle_mod):
    for d in K["empty_set"]["ndims"]:
        x = np.zeros((0, d), np.float32)
        t = oracle_mod.build_tree(x, f32(K["empty_set"]["r"]))
        assert t.n_nodes == 0
        e = oracle_mod.build_edges(t, x, exclude_self=True)
        assert len(e["senders"]) == 0 and e["rel_displacement"].shape == (0, d)


def test_tiny_and_huge_radius(oracle_mod):
    c = K["tiny_radius"]
    x = uniform(c["n"], c["ndims"], 3002)
    e = oracle_mod.build_edges(oracle_mod.build_tree(x, f32(c["r"])), x, exclude_self=True)
    assert len(e["senders"]) == 0
    c = K["huge_radius"]
    x = uniform(c["n"], c["ndims"], 3003)
    e = oracle_mod.build_edges(oracle_mod.build_tree(x, f32(c["r"])), x, exclude_self=True)
    assert len(e["senders"]) == c["n"] * (c["n"] - 1)


def _tree_invariants(t, x):
    """test/build.jl:30-81."""
    n = x.shape[0]
    nch = 1 << x.shape[1]
    assert t.n_nodes >= 1
    assert t.node_first[0] == 1 and t.node_last[0] == n
    assert sorted(t.perm.tolist()) == list(range(1, n + 1))
    for nid in range(t.n_nodes):
        kids = t.children[nid]
        if kids[0] == -1 and (kids == -1).all():
            assert t.node_last[nid] - t.node_first[nid] + 1 >= 1
        else:
            tot = 0
            for cid in kids:
                if cid == -1:
                    continue
                assert cid > nid + 1
                assert t.node_first[cid - 1] >= t.node_first[nid] and t.node_last[cid - 1] <= t.node_last[nid]
                tot += t.node_last[cid - 1] - t.node_first[cid - 1] + 1
            assert tot == t.node_last[nid] - t.node_first[nid] + 1
        pts = x[t.perm[t.node_first[nid] - 1:t.node_last[nid]] - 1]
        assert (pts >= t.bmin[nid]).all() and (pts <= t.bmax[nid]).all()
        assert (pts.min(0) == t.bmin[nid]).all() and (pts.max(0) == t.bmax[nid]).all()


@pytest.mark.parametrize("gen", ["uniform500", "clustered2000", "uniform2d", "clustered2d"])
def test_tree_invariants(oracle_mod, gen):
    x, r = {
        "uniform500": (uniform(500, 3, 1), 0.08),
        "clustered2000": (clustered(2000, 3, 2), 0.05),
        "uniform2d": (uniform(800, 2, 5), 0.05),
        "clustered2d": (clustered(1500, 2, 6), 0.03),
    }[gen]
    _tree_invariants(oracle_mod.build_tree(x, np.float32(r)), x)


CASES = [
    ("u200_r15", lambda: uniform(200, 3, 11), 0.15, True),
    ("u1000_r05", lambda: uniform(1000, 3, 21), 0.05, True),
    ("clustered2000", lambda: (0.1 * np.random.default_rng(31).standard_normal((2000, 3))).astype(np.float32), 0.03, True),
    ("neg_coords", lambda: uniform(200, 3, 3001, -1.0, 1.0), 0.1, True),
    ("u2d", lambda: uniform(1500, 2, 41), 0.04, True),
    ("lattice", lambda: lattice(10, 3, 0.01, 0.001, 7), 0.02, True),
    ("f64", lambda: uniform(600, 3, 51, dtype=np.float64), 0.1, True),
    ("f64_2d", lambda: uniform(600, 2, 52, dtype=np.float64), 0.06, True),
]


@pytest.mark.parametrize("name,gen,r,self_pair", CASES, ids=[c[0] for c in CASES])
def test_edges_match_brute_force(oracle_mod, name, gen, r, self_pair):
    x = gen()
    rr = x.dtype.type(r)
    t = oracle_mod.build_tree(x, rr)
    e = oracle_mod.build_edges(t, x, exclude_self=self_pair)
    bs, br = oracle_mod.brute_force(x, x, rr, self_pair)
    got = sorted(zip(e["receivers"].tolist(), e["senders"].tolist()))
    want = sorted(zip(br.tolist(), bs.tolist()))
    assert got == want
    # features: (x_i - x_j) * inv(r) and sqrt(d2) * inv(r), same rounding
    inv_r = x.dtype.type(1) / rr
    i, j = e["receivers"] - 1, e["senders"] - 1
    diff = (x[j] - x[i]).astype(x.dtype)
    assert np.array_equal(e["rel_displacement"], (-diff * inv_r).astype(x.dtype))
    d2 = diff[:, 0] * diff[:, 0] + diff[:, 1] * diff[:, 1]
    if x.shape[1] == 3:
        d2 = d2 + diff[:, 2] * diff[:, 2]
    assert np.array_equal(e["rel_dist_norm"], (np.sqrt(d2) * inv_r).astype(x.dtype))
    # receivers ascending, segments from the offsets
    assert (np.diff(e["receivers"]) >= 0).all()


def test_asymmetric_pair(oracle_mod):
    """test/edges_cpu.jl:99-124: query A against target B, no self exclusion."""
    a = uniform(150, 3, 41)
    b = uniform(250, 3, 42)
    r = np.float32(0.12)
    t = oracle_mod.build_tree(b, r)
    e = oracle_mod.build_edges(t, a, exclude_self=False)
    bs, br = oracle_mod.brute_force(a, b, r, False)
    assert sorted(zip(e["receivers"].tolist(), e["senders"].tolist())) == sorted(zip(br.tolist(), bs.tolist()))


def test_rrule_matches_central_differences(oracle_mod):
    """ext/OctopusChainRulesCoreExt.jl rrule vs FP64 4-point central
    differences on a frozen edge set (test/chainrules.jl:23-78 shape)."""
    x = uniform(40, 3, 8002, dtype=np.float64)
    r = 0.25
    t = oracle_mod.build_tree(x, r)
    e = oracle_mod.build_edges(t, x, exclude_self=True)
    s, rc = e["senders"] - 1, e["receivers"] - 1

    def loss(c):
        d = (c[rc] - c[s]) / r
        return (d * d).sum() + 0.5 * (np.sqrt((d * d).sum(1)) ** 2).sum()

    g = oracle_mod.diff_backward(x.shape[0], e["senders"], e["receivers"], e["rel_displacement"],
                                 e["rel_dist_norm"], 2 * e["rel_displacement"], e["rel_dist_norm"], r)
    eps = 1e-4
    fd = np.zeros_like(x)
    for k in range(x.size):
        def f(delta):
            c = x.copy()
            c.flat[k] += delta
            return loss(c)
        fd.flat[k] = (-f(2 * eps) + 8 * f(eps) - 8 * f(-eps) + f(-2 * eps)) / (12 * eps)
    np.testing.assert_allclose(g, fd, rtol=1e-4, atol=1e-7)


@pytest.mark.parametrize("ndims,r", [(3, 0.06), (2, 0.02)])
def test_query_range_is_the_slice_of_the_full_coo(oracle_mod, ndims, r):
    """The oracle's query-range COO (used to compare COOs too large for host
    memory slice by slice) equals the slice of the whole COO those queries
    own, offsets included."""
    rng = np.random.default_rng(500 + ndims)
    x = rng.random((6000, ndims)).astype(np.float32)
    r = np.float32(r)
    t = oracle_mod.build_tree(x, r)
    full = oracle_mod.build_edges(t, x, exclude_self=True)
    off = full["offsets"]
    for lo, hi in [(0, 6000), (0, 1), (17, 1033), (2500, 2500), (5999, 6000), (1234, 5000)]:
        part = oracle_mod.build_edges(t, x, exclude_self=True, query_range=(lo, hi))
        a, b = off[lo], off[hi]
        for k in ("senders", "receivers", "rel_displacement", "rel_dist_norm"):
            assert np.array_equal(part[k], full[k][a:b]), (lo, hi, k)
        assert np.array_equal(part["offsets"], off[lo:hi + 1] - a)
    with pytest.raises(ValueError):
        oracle_mod.build_edges(t, x, query_range=(10, 6001))
