"""Parity at the benchmark configurations' full sizes.

The 1M-point SPH time step and the 2M-point differentiable configuration are
compared with the oracle array for array.  The 4M-point nonuniform 2D
configuration (1.55 G edges, ~31 GB of COO) is compared with the oracle in
slices of queries, each slice the part of the COO those queries own; the
same shape at a larger radius runs past 2^31 edges."""
import os
import sys

import numpy as np
import pytest
import torch

from test_gpu_parity import assert_edges_equal, assert_tree_equal

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "octopus.jl_b200"))
import workloads as wl  # noqa: E402


def test_sph_time_step_1m(ob, oracle_mod):
    xs = wl.sph_snapshots(100, 3, 12345)
    r = np.float32(0.02)
    tns = ob.TNS(torch.float32, ndims=3)
    ob.set_search_radius_(tns, r)
    ob.set_refit_mode_(tns, True)
    sid = ob.add_point_set_(tns, torch.from_numpy(xs[0]).cuda().t())
    ob.set_active_search_(tns, sid, sid)
    for x in xs:
        ob.update_point_set_(tns, sid, torch.from_numpy(x).cuda().t())
        ob.run_(tns)
    assert tns.trees[sid - 1].last_build()[0] in (1, 2)  # refit-mode path
    e = ob.build_edges(tns, sid, sid)
    ot = oracle_mod.build_tree(xs[-1], r)
    assert_tree_equal(tns.trees[sid - 1], ot)
    assert_edges_equal(e, oracle_mod.build_edges(ot, xs[-1], exclude_self=True), tns)


def test_uniform_2m(ob, oracle_mod):
    x = wl.uniform(2_000_000, 3, 2025)
    r = np.float32(0.012)
    tns = ob.TNS(torch.float32, ndims=3)
    ob.set_search_radius_(tns, r)
    sid = ob.add_point_set_(tns, torch.from_numpy(x).cuda().t())
    ob.set_active_search_(tns, sid, sid)
    ob.run_(tns)
    e = ob.build_edges(tns, sid, sid)
    assert_edges_equal(e, oracle_mod.build_edges(oracle_mod.build_tree(x, r), x, exclude_self=True), tns)


def _assert_slices_equal(e, ot, x, lo, hi, oracle_mod, nthreads=0):
    """Queries lo..hi-1 (0-based) own one contiguous slice of the GPU COO; it
    must equal the oracle's COO for those queries, array for array."""
    part = oracle_mod.build_edges(ot, x, exclude_self=True, query_range=(lo, hi), nthreads=nthreads)
    q = torch.tensor([lo + 1, hi + 1], dtype=torch.int32, device="cuda")
    a, b = (int(v) for v in torch.searchsorted(e.receivers, q))
    assert b - a == len(part["senders"]), f"queries [{lo}, {hi}): {b - a} edges, oracle {len(part['senders'])}"
    assert np.array_equal(e.senders[a:b].cpu().numpy(), part["senders"]), f"senders of queries [{lo}, {hi})"
    assert np.array_equal(e.receivers[a:b].cpu().numpy(), part["receivers"]), f"receivers of queries [{lo}, {hi})"
    assert np.array_equal(e.rel_displacement[:, a:b].t().cpu().numpy(), part["rel_displacement"]), \
        f"rel_displacement of queries [{lo}, {hi})"
    assert np.array_equal(e.rel_dist_norm[0, a:b].cpu().numpy(), part["rel_dist_norm"]), \
        f"rel_dist_norm of queries [{lo}, {hi})"
    return a, b


def _nonuniform_2d_run(ob, x, r):
    """run! and the COO through the C ABI (int64 edge count and capacity: the
    TNS mirror's EdgeBuffer keeps the reference's Int32 edge count)."""
    import ctypes as C
    from collections import namedtuple
    tns = ob.TNS(torch.float32, ndims=2)
    ob.set_search_radius_(tns, r)
    sid = ob.add_point_set_(tns, torch.from_numpy(x).cuda().t())
    ob.set_active_search_(tns, sid, sid)
    ob.run_(tns)
    ctx = tns._ctx
    ctx.bind_stream()
    h = tns.trees[sid - 1].handle
    ne = C.c_int64()
    ctx.check(ctx.lib.oct_edges_count(ctx.handle, h, h, 1, C.byref(ne)), "count")
    m = int(ne.value)
    snd = torch.empty(m, dtype=torch.int32, device="cuda")
    rcv = torch.empty(m, dtype=torch.int32, device="cuda")
    disp = torch.empty((m, 2), dtype=torch.float32, device="cuda")
    dist = torch.empty((1, m), dtype=torch.float32, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    ctx.check(ctx.lib.oct_edges_fill(ctx.handle, h, h, 1, p(snd), p(rcv), p(disp), p(dist), m), "fill")
    ob.synchronize(tns)
    E = namedtuple("E", "senders receivers rel_displacement rel_dist_norm")
    return tns, sid, E(snd, rcv, disp.t(), dist)


def test_nonuniform_2d_4m_bit_exact(ob, oracle_mod):
    """The 4M-point nonuniform 2D configuration (seed 2026, r = 0.002): the
    tree and all 1,547,624,876 edges -- senders, receivers, rel_displacement
    and rel_dist_norm, in order -- equal the oracle's.  The COO (~31 GB) is
    compared in slices of 250,000 queries, which the oracle emits one at a
    time against the same tree."""
    x = wl.gaussian_mixture_2d(4_000_000, 64, 2026)
    r = np.float32(0.002)
    tns, sid, e = _nonuniform_2d_run(ob, x, r)
    E = e.senders.numel()
    assert E == 1_547_624_876
    ot = oracle_mod.build_tree(x, r)
    assert_tree_equal(tns.trees[sid - 1], ot)
    covered = 0
    for lo in range(0, len(x), 250_000):
        a, b = _assert_slices_equal(e, ot, x, lo, min(len(x), lo + 250_000), oracle_mod)
        assert a == covered
        covered = b
    assert covered == E
    del e, tns
    torch.cuda.empty_cache()


def test_nonuniform_2d_above_2_31_edges(ob, oracle_mod):
    """The same 4M-point shape at r = 0.0025: more than 2^31 - 1 edges, which
    the reference's Int32 edge count and scan cannot represent
    (src/types.jl:89, src/cpu/edges_cpu.jl:209-212).  The int64 offsets must
    place every query's edges contiguously and in query order across edge
    index 2^31; the slices at the start, around edge 2^31 and at the end equal
    the oracle's."""
    x = wl.gaussian_mixture_2d(4_000_000, 64, 2026)
    r = np.float32(0.0025)
    tns, sid, e = _nonuniform_2d_run(ob, x, r)
    E = e.senders.numel()
    assert E > 2**31
    rcv = e.receivers
    n = len(x)
    # receivers never decrease: each query's edges contiguous, in query order
    step = 1 << 28
    for a in range(0, E - 1, step):
        b = min(E, a + step + 1)
        assert bool((rcv[a + 1:b] >= rcv[a:b - 1]).all()), f"receivers decrease in [{a}, {b})"
    assert int(rcv[0]) >= 1 and int(rcv[-1]) <= n
    ot = oracle_mod.build_tree(x, r)
    q_mid = int(rcv[2**31]) - 1  # the query owning edge 2^31
    spans = [(0, 100_000), (max(0, q_mid - 50_000), min(n, q_mid + 50_000)), (n - 100_000, n)]
    for lo, hi in spans:
        a, b = _assert_slices_equal(e, ot, x, lo, hi, oracle_mod)
        if lo == spans[1][0]:
            assert a < 2**31 < b
        if hi == n:
            assert b == E
    del e, tns
    torch.cuda.empty_cache()
