"""API contracts of the TNS mirror on the GPU (test/contracts.jl,
test/edge_cases.jl, test/refit.jl, test/api.jl, test/edges_cuda.jl)."""
import numpy as np
import pytest
import torch

from conftest import uniform
from kats import coords_of, f32, load_kats

pytestmark = pytest.mark.gpu
K = load_kats()


def make(ob, x, r, ndims=None):
    tns = ob.TNS(torch.float32 if x.dtype == np.float32 else torch.float64, ndims=ndims or x.shape[1])
    ob.set_search_radius_(tns, r)
    sid = ob.add_point_set_(tns, torch.from_numpy(np.ascontiguousarray(x)).cuda().t())
    ob.set_active_search_(tns, sid, sid)
    return tns, sid


@pytest.mark.parametrize("name", ["exact_radius_included_3d", "just_past_radius_excluded_3d",
                                  "exact_radius_included_2d", "docstring_example", "single_point"])
def test_reference_kats(ob, name):
    c = K[name]
    x = coords_of(c)
    tns, sid = make(ob, x, f32(c["r"]))
    ob.run_(tns)
    for i, want in c["neighbors"].items():
        assert sorted(ob.get_neighborlist(tns, sid, sid, int(i)).tolist()) == want
    if "n_nodes" in c:
        assert tns.trees[sid - 1].n_nodes == c["n_nodes"]


@pytest.mark.parametrize("name", ["coincident_3d", "coincident_2d"])
def test_coincident_points(ob, name):
    c = K[name]
    x = np.zeros((c["n"], c["ndims"]), np.float32)
    tns, sid = make(ob, x, f32(c["r"]))
    ob.run_(tns)
    for i in range(1, c["n"] + 1):
        assert len(ob.get_neighborlist(tns, sid, sid, i)) == c["n"] - 1
    perm = tns.permutation[sid - 1].cpu().numpy()
    assert sorted(perm.tolist()) == list(range(1, c["n"] + 1))


@pytest.mark.parametrize("d", [3, 2])
def test_empty_point_set(ob, d):
    x = np.zeros((0, d), np.float32)
    tns, sid = make(ob, x, np.float32(0.1), ndims=d)
    ob.run_(tns)
    assert tns.trees[sid - 1].n_nodes == 0
    e = ob.build_edges(tns, sid, sid)
    assert e.senders.numel() == 0 and e.receivers.numel() == 0
    assert tuple(e.rel_displacement.shape) == (d, 0)
    assert tuple(e.rel_dist_norm.shape) == (1, 0)


def test_build_edges_before_run_is_empty(ob):
    """test/backend_errors_cpu.jl:40-57."""
    x = uniform(100, 3, 5003)
    tns, sid = make(ob, x, np.float32(0.1))
    e0 = ob.build_edges(tns, sid, sid)
    assert e0.senders.numel() == 0
    ob.run_(tns)
    assert ob.build_edges(tns, sid, sid).senders.numel() > 0


def test_output_types_shapes_alignment(ob):
    """test/edges_cuda.jl:92-145: dtypes, shapes and that row k of every
    array describes the same edge."""
    x = uniform(800, 3, 202)
    r = np.float32(0.1)
    tns, sid = make(ob, x, r)
    ob.run_(tns)
    e = ob.build_edges(tns, sid, sid)
    n = e.senders.numel()
    assert e.senders.dtype == torch.int32 and e.receivers.dtype == torch.int32
    assert tuple(e.rel_displacement.shape) == (3, n) and tuple(e.rel_dist_norm.shape) == (1, n)
    assert e.rel_displacement.stride() == (1, 3)  # column-major like a Julia matrix
    s = e.senders.cpu().numpy() - 1
    rc = e.receivers.cpu().numpy() - 1
    assert (s != rc).all()
    d = x[rc] - x[s]
    nd = np.sqrt((d.astype(np.float64) ** 2).sum(1))
    assert (nd <= r * (1 + 1e-4)).all()
    assert np.abs(e.rel_displacement.t().cpu().numpy() - d / r).max() < 1e-4
    assert np.abs(e.rel_dist_norm.reshape(-1).cpu().numpy() - nd / r).max() < 1e-4


def test_build_edges_aliases_edge_buffer(ob):
    """test/contracts.jl:223-240."""
    tns, sid = make(ob, uniform(150, 3, 1010), np.float32(0.1))
    ob.run_(tns)
    e = ob.build_edges(tns, sid, sid)
    buf = tns.edge_buffers[tns.active_pairs.index((sid, sid))]
    assert e.senders is buf.senders and e.receivers is buf.receivers
    assert e.rel_displacement is buf.rel_displacement and e.rel_dist_norm is buf.rel_dist_norm
    assert buf.materialized
    ob.run_(tns)  # nothing dirty, but buffers are invalidated (src/api.jl:243-248)
    assert not buf.materialized


def test_set_active_search_idempotent_and_unregistered_pair(ob):
    a = uniform(30, 3, 1014)
    b = uniform(40, 3, 1015)
    tns = ob.TNS()
    ob.set_search_radius_(tns, 0.15)
    ia = ob.add_point_set_(tns, torch.from_numpy(a).cuda().t())
    ib = ob.add_point_set_(tns, torch.from_numpy(b).cuda().t())
    ob.set_active_search_(tns, ia, ib)
    ob.set_active_search_(tns, ia, ib)
    assert tns.active_pairs == [(ia, ib)] and len(tns.edge_buffers) == 1
    ob.run_(tns)
    with pytest.raises(ob.OctopusError):
        ob.build_edges_(tns, ib, ia)


def test_update_point_set_and_dirty(ob, oracle_mod):
    """test/contracts.jl:170-198 and test/api.jl:35-42."""
    x = uniform(500, 3, 1008)
    tns, sid = make(ob, x, np.float32(0.1))
    ob.run_(tns)
    e1 = ob.build_edges(tns, sid, sid).senders.clone()
    with pytest.raises(ob.DimensionMismatch):
        ob.update_point_set_(tns, sid, torch.rand(3, 499, device="cuda"))
    x2 = (x + np.float32(0.01)).astype(np.float32) * np.float32(1.3)
    ob.update_point_set_(tns, sid, torch.from_numpy(x2).cuda().t())
    assert tns.dirty[sid - 1]
    ob.run_(tns)
    e2 = ob.build_edges(tns, sid, sid)
    oe = oracle_mod.build_edges(oracle_mod.build_tree(x2, np.float32(0.1)), x2, exclude_self=True)
    assert np.array_equal(e2.senders.cpu().numpy(), oe["senders"])
    assert e2.senders.numel() != e1.numel() or not torch.equal(e2.senders, e1)


def test_resize_point_set(ob, oracle_mod):
    x = uniform(300, 3, 77)
    tns, sid = make(ob, x, np.float32(0.1))
    ob.run_(tns)
    y = uniform(700, 3, 78)
    ob.resize_point_set_(tns, sid, torch.from_numpy(y).cuda().t())
    ob.run_(tns)
    e = ob.build_edges(tns, sid, sid)
    oe = oracle_mod.build_edges(oracle_mod.build_tree(y, np.float32(0.1)), y, exclude_self=True)
    assert np.array_equal(e.senders.cpu().numpy(), oe["senders"])


def test_refit_mode_keeps_morton_codes(ob, oracle_mod):
    """test/refit.jl:15-86: morton codes kept only in refit mode; results
    identical either way."""
    x = uniform(300, 3, 2002)
    tns, sid = make(ob, x, np.float32(0.1))
    ob.run_(tns)
    assert tns.morton_codes[sid - 1].numel() == 0
    assert tns.permutation[sid - 1].numel() == 300
    e_plain = ob.build_edges(tns, sid, sid).senders.clone()
    ob.set_refit_mode_(tns, True)
    assert tns.dirty[sid - 1]
    ob.run_(tns)
    m = tns.morton_codes[sid - 1].cpu().numpy().view(np.uint64)
    ot = oracle_mod.build_tree(x, np.float32(0.1))
    assert np.array_equal(m, ot.morton)
    assert torch.equal(ob.build_edges(tns, sid, sid).senders, e_plain)


def test_for_each_neighbor_order_and_self(ob, oracle_mod):
    """test/api.jl:44-62, test/contracts.jl:200-221: the callback sees self
    when q == t; get_neighborlist filters it."""
    x = uniform(200, 3, 2)
    r = np.float32(0.1)
    tns, sid = make(ob, x, r)
    ob.run_(tns)
    e = oracle_mod.build_edges(oracle_mod.build_tree(x, r), x, exclude_self=True)
    for i in (1, 7, 50, 200):
        seen = []
        ob.for_each_neighbor(seen.append, tns, sid, sid, i)
        assert i in seen
        lst = ob.get_neighborlist(tns, sid, sid, i)
        assert i not in lst.tolist()
        seg = e["senders"][e["offsets"][i - 1]:e["offsets"][i]]
        assert lst.tolist() == seg.tolist()  # the reference's traversal order
        assert sorted(j for j in seen if j != i) == sorted(lst.tolist())


def test_device_view_contract(ob, oracle_mod):
    x = uniform(2000, 3, 3)
    r = np.float32(0.07)
    tns, sid = make(ob, x, r)
    ob.run_(tns)
    dv = ob.device_view(tns, sid, sid)
    assert dv.n_nodes == tns.trees[sid - 1].n_nodes
    assert dv.radius_sq == float(np.float32(r) * np.float32(r))
    assert tuple(dv.node_children.shape) == (8, dv.n_nodes)
    assert tuple(dv.bounds_min.shape) == (3, dv.n_nodes)
    ot = oracle_mod.build_tree(x, r)
    assert np.array_equal(dv.perm.cpu().numpy(), ot.perm)


@pytest.mark.parametrize("bad", [np.nan, np.inf, 3.0e9])
def test_inexact_error(ob, bad):
    """floor(Int32, ...) throws InexactError in the reference (src/morton.jl:84)."""
    x = uniform(100, 3, 4)
    x[17, 1] = bad
    tns, sid = make(ob, x, np.float32(0.1))
    with pytest.raises(ob.InexactError):
        ob.run_(tns)


def test_two_tns_independent(ob):
    a = uniform(80, 3, 1013)
    b = uniform(120, 3, 1016)
    t1, i1 = make(ob, a, np.float32(0.1))
    t2, i2 = make(ob, b, np.float32(0.2))
    ob.run_(t1)
    ob.run_(t2)
    assert t1.point_sets[0].n == 80 and t2.point_sets[0].n == 120
    assert t1.radius == float(np.float32(0.1)) and t2.radius == float(np.float32(0.2))


def test_traversal_statistics_are_consistent(ob):
    """oct_edges_traversal_stats: the diagnostic count pass counts exactly the
    edges of build_edges, and every hit is one of the pair tests issued."""
    import ctypes as C
    rng = np.random.default_rng(401)
    x = rng.random((30000, 3)).astype(np.float32)
    tns = ob.TNS(torch.float32)
    ob.set_search_radius_(tns, 0.05)
    sid = ob.add_point_set_(tns, torch.from_numpy(x).cuda().t())
    ob.set_active_search_(tns, sid, sid)
    ob.run_(tns)
    e = ob.build_edges(tns, sid, sid)
    snd = e.senders.clone()
    names = ob._lib.TRAVERSAL_STATS
    buf = (C.c_uint64 * len(names))()
    ctx = tns._ctx
    h = tns.trees[sid - 1].handle
    ctx.check(ctx.lib.oct_edges_traversal_stats(ctx.handle, h, h, 1, buf, len(names)), "stats")
    st = dict(zip(names, (int(v) for v in buf)))
    assert st["hits"] == snd.numel()
    assert st["queries"] == len(x)
    assert st["pair_tests"] >= st["hits"] > 0
    assert st["cycles_total"] >= st["cycles_leaf"] >= st["cycles_pairs"] > 0
    # the counts buffer was reused: a fill needs a new count
    e2 = ob.build_edges(tns, sid, sid)
    assert torch.equal(e2.senders, snd)
