"""Failure paths, driven from the host without faulting the GPU.

Models the reference's one fault-injection test (test/edges_cuda.jl:147-265:
the build kernels run with a node capacity below what they need, a canary
region past it must stay intact, and the public API must retry into a correct
tree) and extends it to the library's other recovery paths:

* a look-back wait of the key sort that runs out: a tile made to withhold its
  counts is a flag that nothing sets, the waits after it give up after a short
  polling limit, the build returns OCT_ERR_TIMEOUT with every canary intact,
  and the next build on the same context is exact again;
* the node-capacity overflow and its retry, with canaries after every node
  array;
* hit records that run out, so the fill walks those query groups again.

Every wait involved is bounded; nothing here traps, hangs or reads out of
bounds."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import lattice, uniform
from test_gpu_parity import assert_edges_equal, assert_tree_equal, gpu_run

pytestmark = pytest.mark.gpu


def set_opt(ctx, opt, value):
    ctx.check(ctx.lib.oct_ctx_set_option(ctx.handle, opt, value), "oct_ctx_set_option")


def get_opt(ctx, opt):
    v = C.c_int64(-99)
    ctx.check(ctx.lib.oct_ctx_get_option(ctx.handle, opt, C.byref(v)), "oct_ctx_get_option")
    return int(v.value)


@pytest.fixture
def ctx(ob):
    """The shared device context, with every option back at its default
    after the test."""
    c = ob.api._Context.get(torch.cuda.current_device())
    L = ob._lib
    saved = {o: get_opt(c, o) for o in (L.OPT_WAIT_LIMIT, L.OPT_NODE_CAPACITY, L.OPT_RECORD_CAP,
                                        L.OPT_GUARD_CHECK, L.OPT_WITHHOLD_TILE)}
    yield c
    for o, v in saved.items():
        set_opt(c, o, v)


def test_option_values_are_checked(ob, ctx):
    L = ob._lib
    assert get_opt(ctx, L.OPT_WAIT_LIMIT) == 1 << 22
    assert get_opt(ctx, L.OPT_WITHHOLD_TILE) == -1
    assert ctx.lib.oct_ctx_set_option(ctx.handle, L.OPT_WAIT_LIMIT, -1) == L.ERR_ARGUMENT
    assert ctx.lib.oct_ctx_set_option(ctx.handle, L.OPT_NODE_CAPACITY, 1 << 40) == L.ERR_ARGUMENT
    assert ctx.lib.oct_ctx_set_option(ctx.handle, L.STAT_BUILD_ATTEMPTS, 3) == L.ERR_ARGUMENT
    assert ctx.lib.oct_ctx_set_option(ctx.handle, 12345, 0) == L.ERR_ARGUMENT


def _raw_build(ctx, tree, x_dev, n, r):
    ctx.bind_stream()
    return ctx.lib.oct_tree_build(ctx.handle, tree.handle, C.c_void_p(x_dev.data_ptr()), n, float(r), 0)


def test_sort_wait_that_runs_out_is_reported_and_the_context_recovers(ob, oracle_mod, ctx):
    """200,000 points: 98 tiles of 2048 keys on the look-back sort path.  Tile
    5 withholds its counts in the first pass; the tiles after it give up
    after 2,000 polling rounds."""
    L = ob._lib
    x = uniform(200_000, 3, 71)
    r = np.float32(0.01)
    xd = torch.from_numpy(x).cuda()  # (n, 3) row-major: the (3, n) column-major layout of the C ABI
    tree = ob.api.Octree(ctx, 3, 0)
    set_opt(ctx, L.OPT_GUARD_CHECK, 1)
    set_opt(ctx, L.OPT_WAIT_LIMIT, 2000)
    set_opt(ctx, L.OPT_WITHHOLD_TILE, 5)
    st = _raw_build(ctx, tree, xd, len(x), r)
    # OCT_ERR_TIMEOUT, not OCT_ERR_STATE: the canaries after the sort buffers
    # and node arrays were checked first and found intact.
    assert st == L.ERR_TIMEOUT, ctx.lib.oct_ctx_last_error(ctx.handle)
    assert b"look-back" in ctx.lib.oct_ctx_last_error(ctx.handle)
    torch.cuda.synchronize()  # the context is still usable
    # The same tree again, waits restored: exact.
    set_opt(ctx, L.OPT_WITHHOLD_TILE, -1)
    set_opt(ctx, L.OPT_WAIT_LIMIT, 1 << 22)
    assert _raw_build(ctx, tree, xd, len(x), r) == L.OK
    tree.built = True
    assert_tree_equal(tree, oracle_mod.build_tree(x, r))
    # And through the public API on the same context.
    set_opt(ctx, L.OPT_GUARD_CHECK, 0)
    tns, sid = gpu_run(ob, x, r)
    e = ob.build_edges(tns, sid, sid)
    assert_edges_equal(e, oracle_mod.build_edges(oracle_mod.build_tree(x, r), x, exclude_self=True))


def _jittered_lattice_2d(n, r, seed):
    """The reference test's input shape (test/edges_cuda.jl:170-181): a 2D
    lattice of spacing r / 1.6 with +-0.125 spacing jitter, first n points."""
    rng = np.random.default_rng(seed)
    s = r / 1.6
    per = int(np.ceil(n ** 0.5))
    g = np.stack(np.meshgrid(np.arange(per), np.arange(per), indexing="ij"), -1).reshape(-1, 2).astype(np.float64)
    pts = (g + 0.25 * (rng.random(g.shape) - 0.5)) * s
    return pts[:n].astype(np.float32)


@pytest.mark.parametrize("cap", [16, 1000])
def test_node_capacity_overflow_retries_into_the_exact_tree(ob, oracle_mod, ctx, cap):
    """D = 2, N = 40,000, r = 0.072 (the reference test's configuration) with
    a first-attempt capacity far below the node count: the attempt overflows
    without writing a node (every canary intact), the retry builds the tree
    the oracle builds."""
    L = ob._lib
    x = _jittered_lattice_2d(40_000, np.float32(0.072), 81)
    r = np.float32(0.072)
    ot = oracle_mod.build_tree(x, r)
    assert ot.n_nodes > cap
    set_opt(ctx, L.OPT_GUARD_CHECK, 1)
    set_opt(ctx, L.OPT_NODE_CAPACITY, cap)
    tns, sid = gpu_run(ob, x, r)
    assert get_opt(ctx, L.STAT_BUILD_ATTEMPTS) == 2
    assert_tree_equal(tns.trees[sid - 1], ot)
    e = ob.build_edges(tns, sid, sid)
    assert_edges_equal(e, oracle_mod.build_edges(ot, x, exclude_self=True))
    # A capacity that fits: one attempt.
    set_opt(ctx, L.OPT_NODE_CAPACITY, ot.n_nodes)
    ob.update_point_set_(tns, sid, torch.from_numpy(x).cuda().t())
    ob.run_(tns)
    assert get_opt(ctx, L.STAT_BUILD_ATTEMPTS) == 1
    assert_tree_equal(tns.trees[sid - 1], ot)


def test_node_capacity_overflow_in_refit_mode_and_3d(ob, oracle_mod, ctx):
    L = ob._lib
    x = lattice(30, 3, 0.01, 0.001, 82)
    r = np.float32(0.02)
    ot = oracle_mod.build_tree(x, r)
    set_opt(ctx, L.OPT_GUARD_CHECK, 1)
    set_opt(ctx, L.OPT_NODE_CAPACITY, 100)
    tns = ob.TNS(torch.float32, ndims=3)
    ob.set_search_radius_(tns, r)
    ob.set_refit_mode_(tns, True)
    sid = ob.add_point_set_(tns, torch.from_numpy(x).cuda().t())
    ob.set_active_search_(tns, sid, sid)
    ob.run_(tns)
    assert get_opt(ctx, L.STAT_BUILD_ATTEMPTS) == 2
    assert_tree_equal(tns.trees[sid - 1], ot)
    y = (x + np.float32(0.002)).astype(np.float32)  # every key may move: the merge or a full sort
    ob.update_point_set_(tns, sid, torch.from_numpy(y).cuda().t())
    ob.run_(tns)
    assert_tree_equal(tns.trees[sid - 1], oracle_mod.build_tree(y, r))


def test_hit_records_that_run_out_take_the_walking_fill(ob, oracle_mod, ctx):
    """Too few hit records per query point: the groups whose records run out
    are written by a second walk of the tree, the rest expanded from their
    records, and the COO is exact at every record count."""
    L = ob._lib
    x = uniform(30_000, 3, 91)
    r = np.float32(0.05)
    want = oracle_mod.build_edges(oracle_mod.build_tree(x, r), x, exclude_self=True)
    tns, sid = gpu_run(ob, x, r)
    overflowed = {}
    for cap in (1, 2, 4, 8, 16, 64):
        set_opt(ctx, L.OPT_RECORD_CAP, cap)
        e = ob.build_edges(tns, sid, sid)
        assert get_opt(ctx, L.STAT_RECORD_CAP) == cap
        overflowed[cap] = get_opt(ctx, L.STAT_RECORD_OVERFLOW)
        assert_edges_equal(e, want)
    ov = [overflowed[c] for c in sorted(overflowed)]
    assert ov[0] > 0, overflowed
    assert all(a >= b for a, b in zip(ov, ov[1:])), overflowed
    assert any(0 < v < ov[0] for v in ov), overflowed  # a count where both fills ran
    set_opt(ctx, L.OPT_RECORD_CAP, 0)
    e = ob.build_edges(tns, sid, sid)
    assert get_opt(ctx, L.STAT_RECORD_OVERFLOW) == 0
    assert_edges_equal(e, want)
