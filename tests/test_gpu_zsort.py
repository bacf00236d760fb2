"""apply_zsort and its rrule on the GPU: out[:, i] = x[:, perm[i]] with the
tree's Morton permutation (src/cpu/zsort_cpu.jl:11-32, the CUDA gather of
ext/OctopusCUDAExt.jl:422-432), and the pullback's scatter grad[:, perm] = dy
(ext/OctopusChainRulesCoreExt.jl:65-94).  The permutation is pinned against
the oracle's."""
import numpy as np
import pytest
import torch

from conftest import uniform

pytestmark = pytest.mark.gpu


def built(ob, x, r=0.05, refit=False):
    T = torch.float32 if x.dtype == np.float32 else torch.float64
    tns = ob.TNS(T, ndims=x.shape[1])
    ob.set_search_radius_(tns, r)
    ob.set_refit_mode_(tns, refit)
    sid = ob.add_point_set_(tns, torch.from_numpy(x).cuda().t())
    ob.set_active_search_(tns, sid, sid)
    ob.run_(tns)
    return tns, sid


@pytest.mark.parametrize("shape,dtype", [((None,), torch.float32), ((5, None), torch.float32),
                                         ((3, None), torch.float64), ((4, None), torch.float32),
                                         ((None,), torch.int16), ((7, None), torch.uint8),
                                         ((2, None), torch.int64)])
def test_apply_zsort_matches_oracle_perm(ob, oracle_mod, shape, dtype):
    x = uniform(5000, 3, 901)
    tns, sid = built(ob, x)
    perm = oracle_mod.build_tree(x, np.float32(0.05)).perm.astype(np.int64) - 1
    assert np.array_equal(tns.trees[sid - 1].arrays()["perm"].cpu().numpy().astype(np.int64) - 1, perm)
    n = len(x)
    shp = tuple(n if s is None else s for s in shape)
    g = torch.Generator().manual_seed(7)
    a = (torch.rand(shp, generator=g) * 100).to(dtype).cuda()
    y = ob.apply_zsort(tns, sid, a)
    assert y.shape == a.shape and y.dtype == a.dtype
    want = a[..., torch.from_numpy(perm).cuda()]
    assert torch.equal(y, want)
    assert torch.equal(a, (torch.rand(shp, generator=torch.Generator().manual_seed(7)) * 100).to(dtype).cuda())


def test_apply_zsort_row_major_input(ob):
    """A (F, N) tensor laid out row-major is permuted by columns all the same."""
    x = uniform(3000, 2, 902)
    tns, sid = built(ob, x, 0.02)
    a = torch.randn(6, 3000, device="cuda")  # row-major (F, N)
    perm = tns.trees[sid - 1].arrays()["perm"].long() - 1
    assert torch.equal(ob.apply_zsort(tns, sid, a), a[:, perm])


def test_apply_zsort_gradient_is_the_scatter(ob):
    x = uniform(4000, 3, 903)
    tns, sid = built(ob, x)
    perm = tns.trees[sid - 1].arrays()["perm"].long() - 1
    a = torch.randn(3, 4000, device="cuda", dtype=torch.float32, requires_grad=True)
    w = torch.randn(3, 4000, device="cuda")
    (ob.apply_zsort(tns, sid, a) * w).sum().backward()
    want = torch.zeros_like(w)
    want[:, perm] = w
    assert torch.equal(a.grad, want)
    v = torch.randn(4000, device="cuda", requires_grad=True)
    (ob.apply_zsort(tns, sid, v) ** 2).sum().backward()
    assert torch.equal(v.grad, 2 * v.detach())


def test_apply_zsort_after_refit_steps(ob):
    """The permutation of every build path (full sort, changed keys merged,
    bounds only) is the one applied."""
    x = uniform(20000, 3, 904)
    tns, sid = built(ob, x, 0.03, refit=True)
    for y in [x, x + np.float32(1e-5), x]:
        ob.update_point_set_(tns, sid, torch.from_numpy(np.ascontiguousarray(y)).cuda().t())
        ob.run_(tns)
        perm = tns.trees[sid - 1].arrays()["perm"].long() - 1
        a = torch.arange(20000, device="cuda", dtype=torch.int32)
        assert torch.equal(ob.apply_zsort(tns, sid, a), perm.int())


def test_apply_zsort_errors(ob):
    x = uniform(100, 3, 905)
    tns, sid = built(ob, x)
    with pytest.raises(ob.ArgumentError):
        ob.apply_zsort(tns, sid, torch.zeros((2, 2, 100), device="cuda"))
    with pytest.raises(ob.DimensionMismatch):
        ob.apply_zsort(tns, sid, torch.zeros(99, device="cuda"))
    sid2 = ob.add_point_set_(tns, torch.from_numpy(uniform(50, 3, 906)).cuda().t())
    with pytest.raises(ob.OctopusError):  # added after the last run!
        ob.prepare_zsort(tns)
    ob.run_(tns)
    assert ob.apply_zsort(tns, sid2, torch.zeros(50, device="cuda")).shape == (50,)
    with pytest.deprecated_call():
        ob.apply_zsort_(tns, sid, torch.zeros(100, device="cuda"))
