"""oct_edges_count_noalloc: the allocation-free edge count, for callers that
cannot let a library call cudaMalloc (their device memory belongs to their
own pool allocator, or their loop cannot absorb cudaMalloc's device
synchronization).  It must give exactly what the regular entry point gives:
the per-query counts and offsets implied by build_edges' COO, and the same
edge total -- on consecutive calls, since every call reuses one fixed scratch
array.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import uniform

pytestmark = pytest.mark.gpu


def _tns(ob, x, r):
    tns = ob.TNS(torch.float32, ndims=x.shape[1])
    ob.set_search_radius_(tns, r)
    sid = ob.add_point_set_(tns, torch.from_numpy(x).cuda().t())
    ob.set_active_search_(tns, sid, sid)
    ob.run_(tns)
    return tns, sid


def _noalloc_count(tns, qid, tid, exclude_self):
    ctx = tns._ctx
    n = tns.point_sets[qid - 1].n
    counts = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
    offsets = torch.full((n + 1,), -7, dtype=torch.int64, device="cuda")
    ne = C.c_int64(-1)
    ctx.bind_stream()
    st = ctx.lib.oct_edges_count_noalloc(ctx.handle, tns.trees[qid - 1].handle, tns.trees[tid - 1].handle,
                                         exclude_self, C.c_void_p(counts.data_ptr()),
                                         C.c_void_p(offsets.data_ptr()), C.byref(ne))
    ctx.check(st, "oct_edges_count_noalloc")
    return counts[:n], offsets, int(ne.value)


def test_noalloc_count_matches_regular_entry_point_on_consecutive_calls(ob):
    cases = [(uniform(20000, 3, 11), np.float32(0.05)),   # first call on this device: sets up
             (uniform(50000, 3, 12), np.float32(0.03)),   # second call reuses the scratch
             (uniform(30000, 2, 13), np.float32(0.01))]
    for x, r in cases:
        tns, sid = _tns(ob, x, r)
        e = ob.build_edges(tns, sid, sid)  # regular entry points: oct_edges_count + oct_edges_fill
        n = x.shape[0]
        want_counts = torch.bincount(e.receivers.long() - 1, minlength=n).to(torch.int32)
        want_offsets = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
        want_offsets[1:] = torch.cumsum(want_counts.long(), 0)
        for _ in range(2):
            counts, offsets, ne = _noalloc_count(tns, sid, sid, 1)
            assert ne == e.senders.numel()
            assert torch.equal(counts, want_counts)
            assert torch.equal(offsets, want_offsets)


def test_noalloc_count_cross_pair_and_empty_target(ob):
    a = uniform(3000, 3, 21)
    b = uniform(5000, 3, 22)
    tns = ob.TNS(torch.float32)
    ob.set_search_radius_(tns, 0.08)
    ia = ob.add_point_set_(tns, torch.from_numpy(a).cuda().t())
    ib = ob.add_point_set_(tns, torch.from_numpy(b).cuda().t())
    ie = ob.add_point_set_(tns, torch.zeros((3, 0), device="cuda"))
    ob.set_active_search_(tns, ia, ib)
    ob.run_(tns)
    e = ob.build_edges(tns, ia, ib)
    counts, offsets, ne = _noalloc_count(tns, ia, ib, 0)
    assert ne == e.senders.numel()
    assert torch.equal(counts, torch.bincount(e.receivers.long() - 1, minlength=3000).to(torch.int32))
    counts, offsets, ne = _noalloc_count(tns, ia, ie, 0)
    assert ne == 0 and int(counts.abs().sum()) == 0 and int(offsets.abs().sum()) == 0


def test_noalloc_count_allocates_no_device_memory(ob):
    """The property the entry point exists for: once a first call has set up
    (and the kernels it launches are loaded), further calls leave the
    device's free memory unchanged."""
    x = uniform(40000, 3, 31)
    tns, sid = _tns(ob, x, np.float32(0.04))
    n = x.shape[0]
    counts = torch.empty((n,), dtype=torch.int32, device="cuda")
    offsets = torch.empty((n + 1,), dtype=torch.int64, device="cuda")
    ctx = tns._ctx
    ctx.bind_stream()
    args = (ctx.handle, tns.trees[sid - 1].handle, tns.trees[sid - 1].handle, 1, C.c_void_p(counts.data_ptr()),
            C.c_void_p(offsets.data_ptr()))
    ne = C.c_int64(-1)
    ctx.check(ctx.lib.oct_edges_count_noalloc(*args, C.byref(ne)), "warm-up call")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        ctx.check(ctx.lib.oct_edges_count_noalloc(*args, C.byref(ne)), "oct_edges_count_noalloc")
        ctx.check(ctx.lib.oct_edges_count_noalloc(*args, None), "oct_edges_count_noalloc without the total")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert int(offsets[n]) == ne.value > 0


def test_noalloc_count_follows_the_batched_tree_rules(ob):
    """A batched tree is counted against itself with self pairs excluded, as
    oct_edges_count does; the other combinations are argument errors."""
    rng = np.random.default_rng(41)
    sizes = np.array([700, 0, 1, 2500, 1200], np.int64)
    radii = [0.05, 0.04, 0.06, 0.03, 0.07]
    cat = rng.random((int(sizes.sum()), 3)).astype(np.float32)
    bs = ob.BatchedSearch(torch.float32, 3)
    bs.run_(torch.from_numpy(cat).cuda().t(), sizes, radii)
    e = bs.build_edges()
    n = int(sizes.sum())
    coff = np.concatenate([[0], np.cumsum(sizes)])
    cloud_of_edge = np.repeat(np.arange(len(sizes)), np.diff(e.edge_offsets))
    rcv_global = e.receivers.cpu().numpy().astype(np.int64) - 1 + coff[cloud_of_edge]
    want = np.bincount(rcv_global, minlength=n).astype(np.int32)
    ctx = bs._ctx
    ctx.bind_stream()
    counts = torch.empty((n,), dtype=torch.int32, device="cuda")
    offsets = torch.empty((n + 1,), dtype=torch.int64, device="cuda")
    h = bs.tree.handle
    for _ in range(2):
        ne = C.c_int64(-1)
        ctx.check(ctx.lib.oct_edges_count_noalloc(ctx.handle, h, h, 1, C.c_void_p(counts.data_ptr()),
                                                  C.c_void_p(offsets.data_ptr()), C.byref(ne)), "batched count")
        assert ne.value == e.senders.numel()
        assert np.array_equal(counts.cpu().numpy(), want)
    # self pairs kept, and a batched target searched by another tree: rejected
    st = ctx.lib.oct_edges_count_noalloc(ctx.handle, h, h, 0, C.c_void_p(counts.data_ptr()),
                                         C.c_void_p(offsets.data_ptr()), None)
    assert st == ob._lib.ERR_ARGUMENT
    tns, sid = _tns(ob, uniform(500, 3, 42), np.float32(0.05))
    st = ctx.lib.oct_edges_count_noalloc(ctx.handle, tns.trees[sid - 1].handle, h, 0,
                                         C.c_void_p(counts.data_ptr()), C.c_void_p(offsets.data_ptr()), None)
    assert st == ob._lib.ERR_ARGUMENT
    assert b"batched" in ctx.lib.oct_ctx_last_error(ctx.handle)


def test_noalloc_count_total_is_refused_while_capturing(ob):
    """Reading the total back needs a synchronize, which a stream under
    capture forbids: the call refuses before it issues any work."""
    x = uniform(5000, 3, 51)
    tns, sid = _tns(ob, x, np.float32(0.06))
    n = x.shape[0]
    counts = torch.empty((n,), dtype=torch.int32, device="cuda")
    offsets = torch.empty((n + 1,), dtype=torch.int64, device="cuda")
    ctx = tns._ctx
    h = tns.trees[sid - 1].handle
    y = torch.zeros(16, device="cuda")
    g = torch.cuda.CUDAGraph()
    ne = C.c_int64(-1)
    with torch.cuda.graph(g):
        y.add_(1.0)
        ctx.bind_stream()
        st = ctx.lib.oct_edges_count_noalloc(ctx.handle, h, h, 1, C.c_void_p(counts.data_ptr()),
                                             C.c_void_p(offsets.data_ptr()), C.byref(ne))
    del g
    ctx.bind_stream()
    assert st == ob._lib.ERR_STATE
    assert b"captured" in ctx.lib.oct_ctx_last_error(ctx.handle)
    assert ne.value == 0


def test_noalloc_count_replays_in_a_cuda_graph(ob):
    """Without the total (n_edges NULL) the call may be captured: the count and
    its scan (kernels that start early on their predecessor, programmatic
    dependent launch) replay from a CUDA graph with the regular entry point's
    counts and offsets."""
    x = uniform(20000, 3, 71)
    tns, sid = _tns(ob, x, np.float32(0.05))
    n = x.shape[0]
    e = ob.build_edges(tns, sid, sid)
    want_counts = torch.bincount(e.receivers.long() - 1, minlength=n).to(torch.int32)
    want_offsets = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    want_offsets[1:] = torch.cumsum(want_counts.long(), 0)
    _noalloc_count(tns, sid, sid, 1)  # set-up call, outside the capture
    counts = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    offsets = torch.full((n + 1,), -7, dtype=torch.int64, device="cuda")
    ctx = tns._ctx
    h = tns.trees[sid - 1].handle
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        ctx.bind_stream()
        st = ctx.lib.oct_edges_count_noalloc(ctx.handle, h, h, 1, C.c_void_p(counts.data_ptr()),
                                             C.c_void_p(offsets.data_ptr()), None)
    ctx.bind_stream()
    ctx.check(st, "oct_edges_count_noalloc (captured)")
    for _ in range(2):
        counts.fill_(-7)
        offsets.fill_(-7)
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(counts, want_counts)
        assert torch.equal(offsets, want_offsets)
    del g


def test_noalloc_count_at_its_exact_limit(ob):
    """16,777,216 query points: the largest set, every tile of the fixed
    scratch in use."""
    n = 1 << 24
    gen = torch.Generator(device="cuda").manual_seed(61)
    x = torch.rand((n, 3), device="cuda", generator=gen)
    tns = ob.TNS(torch.float32)
    ob.set_search_radius_(tns, 0.002)
    sid = ob.add_point_set_(tns, x.t())
    ob.set_active_search_(tns, sid, sid)
    ob.run_(tns)
    e = ob.build_edges(tns, sid, sid)
    want_counts = torch.bincount(e.receivers.long() - 1, minlength=n).to(torch.int32)
    for _ in range(2):
        counts, offsets, ne = _noalloc_count(tns, sid, sid, 1)
        assert ne == e.senders.numel() > 0
        assert torch.equal(counts, want_counts)
        assert torch.equal(offsets[1:], torch.cumsum(want_counts.long(), 0))
        assert int(offsets[0]) == 0


def test_noalloc_count_rejects_sets_beyond_its_scratch(ob):
    n = (1 << 24) + 1
    x = torch.rand((n, 3), device="cuda")
    tns = ob.TNS(torch.float32)
    ob.set_search_radius_(tns, 0.01)
    sid = ob.add_point_set_(tns, x.t())
    ob.run_(tns)
    ctx = tns._ctx
    ne = C.c_int64(-1)
    st = ctx.lib.oct_edges_count_noalloc(ctx.handle, tns.trees[0].handle, tns.trees[0].handle, 1,
                                         C.c_void_p(0), C.c_void_p(0), C.byref(ne))
    assert st == ob._lib.ERR_CAPACITY
    assert b"16,777,216" in ctx.lib.oct_ctx_last_error(ctx.handle)
