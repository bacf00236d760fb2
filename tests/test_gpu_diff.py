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
