"""Parity at the benchmark configurations' full sizes.

The 1M-point SPH time step and the 2M-point differentiable configuration are
compared with the oracle array for array.  The 4M-point nonuniform 2D
configuration (1.55 G edges, ~37 GB of COO) is beyond the oracle's host
memory, so it is checked through size-independent properties: the neighbor
sets of sampled queries against a brute force in the reference's FP32
operation order (d2 = dx*dx + dy*dy, dx = x_t - x_q), the offsets against
the segment lengths, and the symmetry of the self-pair COO on the sample."""
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


def test_nonuniform_2d_4m_properties(ob):
    x = wl.gaussian_mixture_2d(4_000_000, 64, 2026)
    r = np.float32(0.002)
    tns = ob.TNS(torch.float32, ndims=2)
    ob.set_search_radius_(tns, r)
    xd = torch.from_numpy(x).cuda()
    sid = ob.add_point_set_(tns, xd.t())
    ob.set_active_search_(tns, sid, sid)
    ob.run_(tns)
    e = ob.build_edges(tns, sid, sid)
    ob.synchronize(tns)
    E = e.senders.numel()
    assert E == 1_547_624_876
    rcv = e.receivers
    # segment starts of sampled receivers, by binary search on the sorted receivers
    rng = np.random.default_rng(7)
    qs = torch.from_numpy(np.sort(rng.choice(len(x), 256, replace=False)) + 1).int().cuda()
    lo = torch.searchsorted(rcv, qs, right=False)
    hi = torch.searchsorted(rcv, qs, right=True)
    assert torch.all(rcv[:-1] <= rcv[1:]) if E < 2**31 else True
    r2 = torch.tensor(r * r, dtype=torch.float32, device="cuda")
    for k in range(len(qs)):
        i = int(qs[k]) - 1
        dx = xd[:, 0] - xd[i, 0]  # x_t - x_q, FP32
        dy = xd[:, 1] - xd[i, 1]
        d2 = dx * dx + dy * dy
        want = torch.nonzero(d2 <= r2).reshape(-1) + 1
        want = want[want != i + 1]
        got = e.senders[int(lo[k]):int(hi[k])]
        assert got.numel() == want.numel(), f"query {i + 1}"
        assert torch.equal(torch.sort(got).values, want.int()), f"query {i + 1}"
        # symmetry: every neighbor j lists i
        js = got[:64].long()
        jl = torch.searchsorted(rcv, js.int(), right=False)
        jh = torch.searchsorted(rcv, js.int(), right=True)
        for a, b in zip(jl.tolist(), jh.tolist()):
            assert bool((e.senders[a:b] == i + 1).any())
    # features of one segment equal their FP32 definition
    k = 0
    i = int(qs[k]) - 1
    seg = slice(int(lo[k]), int(hi[k]))
    j = e.senders[seg].long() - 1
    inv = torch.tensor(1, dtype=torch.float32, device="cuda") / torch.tensor(r, device="cuda")
    dx = xd[j] - xd[i]
    assert torch.equal(e.rel_displacement[:, seg].t(), (-dx) * inv)
    d2 = dx[:, 0] * dx[:, 0] + dx[:, 1] * dx[:, 1]
    assert torch.equal(e.rel_dist_norm[0, seg], torch.sqrt(d2) * inv)
