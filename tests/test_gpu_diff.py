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
