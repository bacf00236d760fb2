"""build_edges_diff: the GPU adjoint against the oracle's restatement of the
reference rrule and against FP64 central differences on a frozen edge set
(test/chainrules.jl)."""
import numpy as np
import pytest
import torch

from conftest import uniform

pytestmark = pytest.mark.gpu


def setup(ob, x, r):
    T = torch.float32 if x.dtype == np.float32 else torch.float64
    tns = ob.TNS(T, ndims=x.shape[1])
    ob.set_search_radius_(tns, r)
    c = torch.from_numpy(x).cuda().t().requires_grad_(True)
    sid = ob.add_point_set_(tns, c.detach())
    ob.set_active_search_(tns, sid, sid)
    ob.run_(tns)
    return tns, sid, c


@pytest.mark.parametrize("d,dtype,mode", [(3, np.float64, "full"), (2, np.float64, "full"),
                                          (3, np.float64, "disp"), (3, np.float64, "dist"),
                                          (3, np.float32, "full"), (2, np.float32, "full")])
def test_adjoint_matches_reference_rrule(ob, oracle_mod, d, dtype, mode):
    x = uniform(3000, d, 8100 + d, dtype=dtype)
    r = dtype(0.08 if d == 3 else 0.03)
    tns, sid, c = setup(ob, x, r)
    e = ob.build_edges_diff(c, tns, sid, r)
    loss = 0
    if mode in ("full", "disp"):
        loss = loss + (e.rel_displacement ** 2).sum()
    if mode in ("full", "dist"):
        loss = loss + 0.5 * (e.rel_dist_norm ** 2).sum()
    loss.backward()
    g = c.grad.t().cpu().numpy()
    rd = e.rel_displacement.detach().t().cpu().numpy()
    rn = e.rel_dist_norm.detach().reshape(-1).cpu().numpy()
    go = oracle_mod.diff_backward(x.shape[0], e.senders.cpu().numpy(), e.receivers.cpu().numpy(), rd, rn,
                                  2 * rd if mode in ("full", "disp") else None,
                                  rn if mode in ("full", "dist") else None, r)
    tol = 1e-12 if dtype == np.float64 else 2e-5
    scale = np.abs(go).max()
    assert np.abs(g - go).max() <= tol * scale


def test_adjoint_matches_fp64_central_differences(ob, oracle_mod):
    x = uniform(400, 3, 8002, dtype=np.float64)
    r = 0.25
    tns, sid, c = setup(ob, x, r)
    e = ob.build_edges_diff(c, tns, sid, r)
    loss = (e.rel_displacement ** 2).sum() + 0.5 * (e.rel_dist_norm ** 2).sum()
    loss.backward()
    g = c.grad.t().cpu().numpy()
    s = e.senders.cpu().numpy() - 1
    rc = e.receivers.cpu().numpy() - 1

    def f(cc):
        dd = (cc[rc] - cc[s]) / r
        return (dd * dd).sum() + 0.5 * (dd * dd).sum()

    rng = np.random.default_rng(0)
    eps = 1e-4
    for k in rng.choice(x.size, 60, replace=False):
        def fk(delta):
            cc = x.copy()
            cc.flat[k] += delta
            return f(cc)
        fd = (-fk(2 * eps) + 8 * fk(eps) - 8 * fk(-eps) + fk(-2 * eps)) / (12 * eps)
        assert abs(g.flat[k] - fd) <= 1e-5 * max(1.0, abs(fd))


def test_adjoint_is_deterministic(ob):
    x = uniform(20000, 3, 99)
    r = np.float32(0.05)
    tns, sid, c = setup(ob, x, r)
    grads = []
    for _ in range(2):
        c.grad = None
        e = ob.build_edges_diff(c, tns, sid, r)
        ((e.rel_displacement ** 2).sum() + 0.5 * (e.rel_dist_norm ** 2).sum()).backward()
        grads.append(c.grad.clone())
    assert torch.equal(grads[0], grads[1])


def test_index_only_loss_gives_zero_gradient(ob):
    """test/chainrules.jl:149-168."""
    x = uniform(300, 3, 5, dtype=np.float64)
    tns, sid, c = setup(ob, x, 0.2)
    e = ob.build_edges_diff(c, tns, sid, 0.2)
    (e.rel_displacement.sum() * 0).backward()
    assert torch.count_nonzero(c.grad) == 0


def test_recompute_mode_gives_identical_gradient(ob):
    """recompute=True keeps no feature arrays and recomputes them from the
    coordinates with the forward's arithmetic: same gradient bits."""
    x = uniform(30000, 3, 77)
    r = np.float32(0.04)
    grads = []
    for recompute in (False, True):
        tns, sid, c = setup(ob, x, r)
        e = ob.build_edges_diff(c, tns, sid, r, recompute=recompute)
        ((e.rel_displacement ** 2).sum() + 0.5 * (e.rel_dist_norm ** 2).sum()).backward()
        grads.append(c.grad.clone())
    assert torch.equal(grads[0], grads[1])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_general_coo_uses_sorted_adjoint(ob, oracle_mod, dtype):
    """Edges without their mirrors (a subset of a self-pair COO) take the
    sender-sorted adjoint; it must still match the reference rrule."""
    import ctypes as C
    x = uniform(4000, 3, 31, dtype=dtype)
    r = dtype(0.06)
    tns, sid, _ = setup(ob, x, r)
    e = ob.build_edges(tns, sid, sid)
    keep = torch.arange(e.senders.numel(), device="cuda") % 10 != 3
    snd = e.senders[keep].contiguous()
    rcv = e.receivers[keep].contiguous()
    rd = e.rel_displacement.t()[keep].contiguous()
    rn = e.rel_dist_norm.reshape(-1)[keep].contiguous()
    gd = 2 * rd
    gn = rn.clone()
    grad = torch.empty_like(torch.from_numpy(x)).cuda()
    lc = tns._ctx
    lc.bind_stream()
    lc.check(lc.lib.oct_edges_diff_backward(
        lc.handle, 3, 0 if dtype == np.float32 else 1, x.shape[0], snd.numel(), C.c_void_p(snd.data_ptr()),
        C.c_void_p(rcv.data_ptr()), C.c_void_p(rd.data_ptr()), C.c_void_p(rn.data_ptr()),
        C.c_void_p(gd.data_ptr()), C.c_void_p(gn.data_ptr()), float(r), C.c_void_p(grad.data_ptr())), "adjoint")
    go = oracle_mod.diff_backward(x.shape[0], snd.cpu().numpy(), rcv.cpu().numpy(), rd.cpu().numpy(),
                                  rn.cpu().numpy(), gd.cpu().numpy(), gn.cpu().numpy(), r)
    tol = 1e-12 if dtype == np.float64 else 2e-5
    assert np.abs(grad.cpu().numpy() - go).max() <= tol * np.abs(go).max()


def _pair_rrule_f64(nq, nt, s, q, rd, rn, gd, gn, r):
    """The rrule's per-edge term (ext/OctopusChainRulesCoreExt.jl:150-189)
    added to the receiver and subtracted from the sender, in float64."""
    rd = rd.astype(np.float64)
    rn = rn.astype(np.float64)
    term = gd.astype(np.float64) / r
    mask = rn > 1e-8
    term[mask] += rd[mask] * (gn.astype(np.float64)[mask] / (rn[mask] * r))[:, None]
    g_q = np.zeros((nq, rd.shape[1]))
    g_t = np.zeros((nt, rd.shape[1]))
    np.add.at(g_q, q, term)
    np.subtract.at(g_t, s, term)
    return g_q, g_t


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_cross_pair_adjoint(ob, dtype):
    """Query set A, target set B: gradients reach both coordinate sets."""
    T = torch.float32 if dtype == np.float32 else torch.float64
    a = uniform(2500, 3, 8201, dtype=dtype)
    b = uniform(3500, 3, 8202, dtype=dtype)
    r = dtype(0.09)
    tns = ob.TNS(T, ndims=3)
    ob.set_search_radius_(tns, r)
    ca = torch.from_numpy(a).cuda().t().requires_grad_(True)
    cb = torch.from_numpy(b).cuda().t().requires_grad_(True)
    ia = ob.add_point_set_(tns, ca.detach())
    ib = ob.add_point_set_(tns, cb.detach())
    ob.set_active_search_(tns, ia, ib)
    ob.run_(tns)
    e = ob.build_edges_diff_pair(ca, cb, tns, ia, ib, r)
    ((e.rel_displacement ** 2).sum() + 0.5 * (e.rel_dist_norm ** 2).sum()).backward()
    s = e.senders.cpu().numpy().astype(np.int64) - 1
    q = e.receivers.cpu().numpy().astype(np.int64) - 1
    rd = e.rel_displacement.detach().t().cpu().numpy()
    rn = e.rel_dist_norm.detach().reshape(-1).cpu().numpy()
    gq, gt = _pair_rrule_f64(len(a), len(b), s, q, rd, rn, 2 * rd, rn, float(r))
    tol = 1e-12 if dtype == np.float64 else 2e-5
    assert np.abs(ca.grad.t().cpu().numpy() - gq).max() <= tol * np.abs(gq).max()
    assert np.abs(cb.grad.t().cpu().numpy() - gt).max() <= tol * np.abs(gt).max()
    with pytest.raises(ob.ArgumentError):
        ob.build_edges_diff_pair(ca, ca, tns, ia, ia, r)


def test_cross_pair_adjoint_fp64_central_differences(ob):
    a = uniform(300, 3, 8203, dtype=np.float64)
    b = uniform(350, 3, 8204, dtype=np.float64)
    r = 0.25
    tns = ob.TNS(torch.float64, ndims=3)
    ob.set_search_radius_(tns, r)
    ca = torch.from_numpy(a).cuda().t().requires_grad_(True)
    cb = torch.from_numpy(b).cuda().t().requires_grad_(True)
    ia = ob.add_point_set_(tns, ca.detach())
    ib = ob.add_point_set_(tns, cb.detach())
    ob.set_active_search_(tns, ia, ib)
    ob.run_(tns)
    e = ob.build_edges_diff_pair(ca, cb, tns, ia, ib, r)
    ((e.rel_displacement ** 2).sum() + 0.5 * (e.rel_dist_norm ** 2).sum()).backward()
    s = e.senders.cpu().numpy() - 1
    q = e.receivers.cpu().numpy() - 1

    def f(xa, xb):
        dd = (xa[q] - xb[s]) / r
        return 1.5 * (dd * dd).sum()

    rng = np.random.default_rng(1)
    eps = 1e-4
    for which, x, g in ((0, a, ca.grad.t().cpu().numpy()), (1, b, cb.grad.t().cpu().numpy())):
        for k in rng.choice(x.size, 30, replace=False):
            def fk(delta):
                xx = x.copy()
                xx.flat[k] += delta
                return f(xx, b) if which == 0 else f(a, xx)
            fd = (-fk(2 * eps) + 8 * fk(eps) - 8 * fk(-eps) + fk(-2 * eps)) / (12 * eps)
            assert abs(g.flat[k] - fd) <= 1e-5 * max(1.0, abs(fd))


def _backward_raw(ob, tns, n, snd, rcv, rd, rn, gd, gn, r, dtype, order=None, coords=None):
    """The C-ABI pullback on raw device arrays; returns (status, grad)."""
    import ctypes as C
    lc = tns._ctx
    lc.bind_stream()
    T = torch.float32 if dtype == np.float32 else torch.float64
    grad = torch.full((n, 3), float("nan"), dtype=T, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)
    if order is None and coords is None:
        st = lc.lib.oct_edges_diff_backward(lc.handle, 3, 0 if dtype == np.float32 else 1, n, snd.numel(), p(snd),
                                            p(rcv), p(rd), p(rn), p(gd), p(gn), float(r), p(grad))
    else:
        st = lc.lib.oct_edges_diff_backward_ordered(lc.handle, 3, 0 if dtype == np.float32 else 1, n, snd.numel(),
                                                    p(snd), p(rcv), p(rd), p(rn), p(coords), p(gd), p(gn), float(r),
                                                    p(grad), p(order))
    return st, grad


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_adjoint_order_changes_nothing(ob, dtype):
    """The processing order (tree perm, a random permutation, none) picks
    which warp handles a point, never a point's sum: bit-identical grads."""
    x = uniform(6000, 3, 8301, dtype=dtype)
    r = dtype(0.07)
    tns, sid, c = setup(ob, x, r)
    e = ob.build_edges(tns, sid, sid)
    snd, rcv = e.senders.clone(), e.receivers.clone()
    rd = e.rel_displacement.t().contiguous()
    rn = e.rel_dist_norm.reshape(-1).contiguous()
    gd, gn = torch.sin(rd * 7), torch.cos(rn * 3)
    n = x.shape[0]
    perm = tns.trees[sid - 1].arrays()["perm"].clone()
    rnd = (torch.randperm(n, generator=torch.Generator().manual_seed(3)) + 1).to(torch.int32).cuda()
    out = []
    for order in (None, perm, rnd):
        st, g = _backward_raw(ob, tns, n, snd, rcv, rd, rn, gd, gn, r, dtype, order=order,
                              coords=None)
        assert st == 0
        out.append(g)
    xc = torch.from_numpy(x).cuda().contiguous()
    st, g_re = _backward_raw(ob, tns, n, snd, rcv, None, None, gd, gn, r, dtype, order=perm, coords=xc)
    assert st == 0
    for g in out[1:] + [g_re]:
        assert torch.equal(g, out[0])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_adjoint_of_ungrouped_coo(ob, oracle_mod, dtype):
    """Edges in any order (not grouped by receiver) go through the sorted
    path with a receiver sort and still match the reference rrule."""
    x = uniform(4000, 3, 8302, dtype=dtype)
    r = dtype(0.06)
    tns, sid, _ = setup(ob, x, r)
    e = ob.build_edges(tns, sid, sid)
    m = e.senders.numel()
    sh = torch.randperm(m, generator=torch.Generator().manual_seed(5)).cuda()
    snd, rcv = e.senders[sh].contiguous(), e.receivers[sh].contiguous()
    rd = e.rel_displacement.t()[sh].contiguous()
    rn = e.rel_dist_norm.reshape(-1)[sh].contiguous()
    gd, gn = 2 * rd, rn.clone()
    st, g = _backward_raw(ob, tns, x.shape[0], snd, rcv, rd, rn, gd, gn, r, dtype)
    assert st == 0
    go = oracle_mod.diff_backward(x.shape[0], snd.cpu().numpy(), rcv.cpu().numpy(), rd.cpu().numpy(),
                                  rn.cpu().numpy(), gd.cpu().numpy(), gn.cpu().numpy(), r)
    tol = 1e-12 if dtype == np.float64 else 2e-5
    assert np.abs(g.cpu().numpy() - go).max() <= tol * np.abs(go).max()
    # recomputing the features needs the grouped self-pair COO
    xc = torch.from_numpy(x).cuda().contiguous()
    st, _ = _backward_raw(ob, tns, x.shape[0], snd, rcv, None, None, gd, gn, r, dtype, coords=xc)
    assert st != 0


def test_adjoint_rejects_out_of_range_indices(ob):
    """A sender, receiver or order entry outside 1..n is an argument error
    (the kernels check every index before using it)."""
    x = uniform(2000, 3, 8303)
    r = np.float32(0.08)
    tns, sid, _ = setup(ob, x, r)
    e = ob.build_edges(tns, sid, sid)
    n = x.shape[0]
    rd = e.rel_displacement.t().contiguous()
    rn = e.rel_dist_norm.reshape(-1).contiguous()
    gd, gn = 2 * rd, rn.clone()
    for field, val in (("snd", n + 1), ("snd", 0), ("rcv", n + 5)):
        snd, rcv = e.senders.clone(), e.receivers.clone()
        (snd if field == "snd" else rcv)[len(snd) // 2] = val
        st, _ = _backward_raw(ob, tns, n, snd, rcv, rd, rn, gd, gn, r, np.float32)
        assert st != 0
        st, _ = _backward_raw(ob, tns, n, snd, rcv, rd, rn, gd, gn, r, np.float32,
                              order=torch.arange(1, n + 1, dtype=torch.int32, device="cuda"))
        assert st != 0
    bad_order = torch.arange(1, n + 1, dtype=torch.int32, device="cuda")
    bad_order[7] = n + 3
    st, _ = _backward_raw(ob, tns, n, e.senders, e.receivers, rd, rn, gd, gn, r, np.float32, order=bad_order)
    assert st != 0
    # the context stays usable after the errors
    st, g = _backward_raw(ob, tns, n, e.senders, e.receivers, rd, rn, gd, gn, r, np.float32)
    assert st == 0 and torch.isfinite(g).all()


def test_cross_pair_adjoint_ungrouped(ob):
    """Cross-pair adjoint of a shuffled COO equals that of the grouped one
    up to the order of the float64 sums."""
    import ctypes as C
    a = uniform(2500, 3, 8304)
    b = uniform(3000, 3, 8305)
    r = np.float32(0.09)
    tns = ob.TNS(torch.float32, ndims=3)
    ob.set_search_radius_(tns, r)
    ia = ob.add_point_set_(tns, torch.from_numpy(a).cuda().t())
    ib = ob.add_point_set_(tns, torch.from_numpy(b).cuda().t())
    ob.set_active_search_(tns, ia, ib)
    ob.run_(tns)
    e = ob.build_edges(tns, ia, ib)
    m = e.senders.numel()
    sh = torch.randperm(m, generator=torch.Generator().manual_seed(9)).cuda()
    rd = e.rel_displacement.t().contiguous()
    rn = e.rel_dist_norm.reshape(-1).contiguous()
    lc = tns._ctx
    lc.bind_stream()
    p = lambda t: C.c_void_p(t.data_ptr())
    res = []
    for idx in (torch.arange(m, device="cuda"), sh):
        snd, rcv = e.senders[idx].contiguous(), e.receivers[idx].contiguous()
        rdi, rni = rd[idx].contiguous(), rn[idx].contiguous()
        gq = torch.empty((len(a), 3), device="cuda")
        gt = torch.empty((len(b), 3), device="cuda")
        gd, gn = 2 * rdi, rni.clone()  # held for the call
        assert lc.lib.oct_edges_diff_backward_pair(lc.handle, 3, 0, len(a), len(b), m, p(snd), p(rcv), p(rdi),
                                                   p(rni), p(gd), p(gn), float(r), p(gq), p(gt)) == 0
        res.append((gq, gt))
    for u, v in zip(res[0], res[1]):
        assert torch.allclose(u, v, rtol=1e-5, atol=1e-6 * float(u.abs().max()))


def _fill_diff(ob, tns, sid):
    """oct_edges_count + oct_edges_fill_diff: the COO and each edge's mirror."""
    import ctypes as C
    ctx = tns._ctx
    ctx.bind_stream()
    h = tns.trees[sid - 1].handle
    ne = C.c_int64()
    ctx.check(ctx.lib.oct_edges_count(ctx.handle, h, h, 1, C.byref(ne)), "count")
    m = int(ne.value)
    T = tns.T
    snd = torch.empty(m, dtype=torch.int32, device="cuda")
    rcv = torch.empty(m, dtype=torch.int32, device="cuda")
    disp = torch.empty((m, tns.ndims), dtype=T, device="cuda")
    dist = torch.empty(m, dtype=T, device="cuda")
    mir = torch.full((m,), -5, dtype=torch.int32, device="cuda")
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    ctx.check(ctx.lib.oct_edges_fill_diff(ctx.handle, h, ptr(snd), ptr(rcv), ptr(disp), ptr(dist), ptr(mir), m),
              "fill_diff")
    torch.cuda.synchronize()
    return snd, rcv, disp, dist, mir


@pytest.mark.parametrize("d,dtype", [(3, np.float32), (2, np.float32), (3, np.float64)])
def test_mirror_indices_of_the_differentiable_fill(ob, d, dtype):
    """Every edge's mirror: senders[mirror[k]] = receivers[k] and back, the
    mirror of the mirror is the edge; the same COO as build_edges, also when
    the hit records overflow and the walking fill writes part of it."""
    x = uniform(30000, d, 8300 + d, dtype=dtype)
    r = dtype(0.05 if d == 3 else 0.01)
    tns, sid, c = setup(ob, x, r)
    snd, rcv, disp, dist, mir = _fill_diff(ob, tns, sid)
    e = ob.build_edges(tns, sid, sid)
    assert torch.equal(snd, e.senders) and torch.equal(rcv, e.receivers)
    assert torch.equal(disp, e.rel_displacement.t()) and torch.equal(dist, e.rel_dist_norm.reshape(-1))
    m = snd.numel()
    assert int(mir.min()) >= 0 and int(mir.max()) < m
    ml = mir.long()
    assert torch.equal(snd[ml], rcv) and torch.equal(rcv[ml], snd)
    assert torch.equal(ml[ml], torch.arange(m, device="cuda"))
    ctx = tns._ctx
    ctx.check(ctx.lib.oct_ctx_set_option(ctx.handle, ob._lib.OPT_RECORD_CAP, 1), "record cap")
    try:
        _, _, _, _, mir2 = _fill_diff(ob, tns, sid)
        import ctypes as C
        ov = C.c_int64()
        ctx.lib.oct_ctx_get_option(ctx.handle, ob._lib.STAT_RECORD_OVERFLOW, C.byref(ov))
        assert ov.value > 0
    finally:
        ctx.check(ctx.lib.oct_ctx_set_option(ctx.handle, ob._lib.OPT_RECORD_CAP, 0), "record cap")
    assert torch.equal(mir2, mir)


@pytest.mark.parametrize("recompute", [False, True])
def test_mirror_backward_equals_the_searching_backward(ob, recompute):
    """oct_edges_diff_backward_mirror gives the bits of
    oct_edges_diff_backward_ordered; corrupt mirror indices fall back to the
    checked path and still give them."""
    import ctypes as C
    x = uniform(50000, 3, 8401)
    r = np.float32(0.03)
    tns, sid, c = setup(ob, x, r)
    snd, rcv, disp, dist, mir = _fill_diff(ob, tns, sid)
    m, n = snd.numel(), len(x)
    gen = torch.Generator(device="cuda").manual_seed(5)
    dd = torch.randn((m, 3), generator=gen, device="cuda")
    dn = torch.randn(m, generator=gen, device="cuda")
    xc = torch.from_numpy(x).cuda()
    order = tns.trees[sid - 1].arrays()["perm"].clone()
    ctx = tns._ctx
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)  # noqa: E731
    fp = None if recompute else disp
    fd = None if recompute else dist
    xp = xc if recompute else None
    want = torch.empty((n, 3), device="cuda")
    ctx.check(ctx.lib.oct_edges_diff_backward_ordered(ctx.handle, 3, 0, n, m, ptr(snd), ptr(rcv), ptr(fp), ptr(fd),
                                                      ptr(xp), ptr(dd), ptr(dn), float(r), ptr(want), ptr(order)),
              "ordered")
    got = torch.empty((n, 3), device="cuda")
    ctx.check(ctx.lib.oct_edges_diff_backward_mirror(ctx.handle, 3, 0, n, m, ptr(snd), ptr(rcv), ptr(mir), ptr(fp),
                                                     ptr(fd), ptr(xp), ptr(dd), ptr(dn), float(r), ptr(got),
                                                     ptr(order)), "mirror")
    assert torch.equal(got, want)
    bad = mir.clone()
    bad[m // 2] = -1
    bad[m // 3] = m + 7
    got2 = torch.empty((n, 3), device="cuda")
    ctx.check(ctx.lib.oct_edges_diff_backward_mirror(ctx.handle, 3, 0, n, m, ptr(snd), ptr(rcv), ptr(bad), ptr(fp),
                                                     ptr(fd), ptr(xp), ptr(dd), ptr(dn), float(r), ptr(got2),
                                                     ptr(order)), "mirror fallback")
    assert torch.equal(got2, want)
