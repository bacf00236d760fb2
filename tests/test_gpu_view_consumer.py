"""The reference-layout tree view serves user kernels.

A CUDA kernel written only against the public header's oct_tree_view
(tests/consumer/view_consumer.cu) walks the tree the way the reference's
inlined device traversal does (src/macros.jl:60-177: root pushed
unconditionally, first-slot-empty nodes scanned as leaves, children in slot
order, LIFO, no self filter).  Its neighbor lists must equal the oracle's per
query, in order -- the CPU iterator's order, which the COO also follows --
and the library's own for_each_neighbor.  Also: the zsort hook in the
reference's shape, oct_permute_rows(perm, ...)."""
import ctypes as C
import importlib.util
import os

import numpy as np
import pytest
import torch

from conftest import ROOT, clustered, lattice, uniform
from test_gpu_parity import gaussian_mixture_2d, gpu_run, torch_dtype

pytestmark = pytest.mark.gpu


def consumer_lib():
    spec = importlib.util.spec_from_file_location(
        "view_consumer_build", os.path.join(ROOT, "tests", "consumer", "build_consumer.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    lib = C.CDLL(mod.ensure_built())
    lib.view_consumer_neighbors.restype = C.c_int
    lib.view_consumer_neighbors.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                            C.c_void_p, C.c_int64, C.c_void_p]
    return lib


def consumer_lists(lib, view, xq_dev, xt_dev, nq, cap):
    counts = torch.zeros(nq, dtype=torch.int32, device="cuda")
    idx = torch.zeros(nq * cap, dtype=torch.int32, device="cuda")
    st = lib.view_consumer_neighbors(C.byref(view), C.c_void_p(xq_dev.data_ptr()), C.c_void_p(xt_dev.data_ptr()),
                                     nq, C.c_void_p(counts.data_ptr()), C.c_void_p(idx.data_ptr()), cap,
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    torch.cuda.synchronize()
    return counts.cpu().numpy(), idx.cpu().numpy().reshape(nq, cap)


CASES = {
    "u3d": (lambda: uniform(20000, 3, 301), 0.05),
    "lattice3d": (lambda: lattice(25, 3, 0.01, 0.001, 302), 0.02),
    "clustered3d": (lambda: clustered(8000, 3, 303), 0.03),
    "big_leaves": (lambda: np.repeat(uniform(60, 3, 304), 40, axis=0), 0.2),
    "mix2d": (lambda: gaussian_mixture_2d(30000, 12, 305), 0.004),
    "f64_3d": (lambda: uniform(5000, 3, 306, dtype=np.float64), 0.07),
    "f64_2d": (lambda: uniform(5000, 2, 307, dtype=np.float64), 0.03),
}


@pytest.mark.parametrize("name", list(CASES))
def test_user_kernel_on_the_tree_view_matches_the_oracle(ob, oracle_mod, name):
    gen, r = CASES[name]
    x = gen()
    r = x.dtype.type(r)
    tns, sid = gpu_run(ob, x, r)
    view = tns.trees[sid - 1].view()
    xd = torch.from_numpy(x).cuda()  # (n, D) row-major = (D, n) column-major
    oe = oracle_mod.build_edges(oracle_mod.build_tree(x, r), x, exclude_self=False)
    off = oe["offsets"]
    cap = int(np.diff(off).max()) + 1
    lib = consumer_lib()
    counts, idx = consumer_lists(lib, view, xd, xd, len(x), cap)
    assert np.array_equal(counts, np.diff(off))
    snd = oe["senders"]
    for i in range(len(x)):
        assert np.array_equal(idx[i, :counts[i]], snd[off[i]:off[i + 1]]), f"query {i + 1}"
    # the library's own host accessor (no self filter either) agrees on a sample
    for i in (0, len(x) // 2, len(x) - 1):
        got = []
        ob.for_each_neighbor(got.append, tns, sid, sid, i + 1)
        assert np.array_equal(np.array(got, np.int32), snd[off[i]:off[i + 1]])


def test_user_kernel_cross_pair(ob, oracle_mod):
    a = uniform(3000, 3, 311)
    b = uniform(7000, 3, 312)
    r = np.float32(0.06)
    tns = ob.TNS(torch.float32)
    ob.set_search_radius_(tns, r)
    ia = ob.add_point_set_(tns, torch.from_numpy(a).cuda().t())
    ib = ob.add_point_set_(tns, torch.from_numpy(b).cuda().t())
    ob.set_active_search_(tns, ia, ib)
    ob.run_(tns)
    view = tns.trees[ib - 1].view()
    oe = oracle_mod.build_edges(oracle_mod.build_tree(b, r), a, exclude_self=False)
    off = oe["offsets"]
    cap = int(np.diff(off).max()) + 1
    counts, idx = consumer_lists(consumer_lib(), view, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
                                 len(a), cap)
    assert np.array_equal(counts, np.diff(off))
    for i in range(len(a)):
        assert np.array_equal(idx[i, :counts[i]], oe["senders"][off[i]:off[i + 1]])


def _permute(ctx, perm_dev, rows, direction):
    """rows: an (n, F) row-major tensor, i.e. the memory of an (F, n)
    column-major matrix: n rows of F contiguous values."""
    out = torch.empty_like(rows)
    n = rows.shape[0]
    row_bytes = rows.element_size() * (rows.shape[1] if rows.dim() == 2 else 1)
    ctx.bind_stream()
    st = ctx.lib.oct_permute_rows(ctx.handle, C.c_void_p(perm_dev.data_ptr()), n, C.c_void_p(rows.data_ptr()),
                                  C.c_void_p(out.data_ptr()), row_bytes, direction)
    return st, out


@pytest.mark.parametrize("F,dtype", [(1, torch.float32), (3, torch.float32), (5, torch.float64), (16, torch.float16)])
def test_permute_rows_by_a_perm_vector(ob, oracle_mod, F, dtype):
    """_apply_zsort_cuda(perm, user_array) (ext/OctopusCUDAExt.jl:422-432):
    user_array[:, perm] for the tree's permutation, and the pullback's scatter."""
    x = uniform(4000, 3, 321)
    r = np.float32(0.05)
    tns, sid = gpu_run(ob, x, r)
    perm = oracle_mod.build_tree(x, r).perm
    perm_dev = torch.from_numpy(perm).cuda()
    ctx = tns._ctx
    n = len(x)
    rows = torch.arange(F * n, dtype=torch.float64).reshape(n, F).to(dtype).cuda()
    if F == 1:
        rows = rows.reshape(n)
    st, out = _permute(ctx, perm_dev, rows, 0)
    assert st == ob._lib.OK
    want = rows[torch.from_numpy(perm - 1).long().cuda()]
    assert torch.equal(out, want)
    st, back = _permute(ctx, perm_dev, out, 1)  # the pullback's scatter inverts the gather
    assert st == ob._lib.OK
    assert torch.equal(back, rows)
    # the tree-keyed entry point (apply_zsort on the (F, n) matrix) agrees
    z = ob.apply_zsort(tns, sid, rows if F == 1 else rows.t())
    assert torch.equal(z if F == 1 else z.t(), want)


def test_permute_rows_rejects_an_entry_out_of_range(ob):
    ctx = ob.api._Context.get(torch.cuda.current_device())
    n = 1000
    perm = torch.arange(1, n + 1, dtype=torch.int32, device="cuda").flip(0).contiguous()
    x = torch.rand(n, device="cuda")
    st, out = _permute(ctx, perm, x, 0)
    assert st == ob._lib.OK and torch.equal(out, x.flip(0))
    for bad in (0, n + 1, -5):
        p = perm.clone()
        p[17] = bad
        st, _ = _permute(ctx, p, x, 0)
        assert st == ob._lib.ERR_ARGUMENT
        assert b"outside" in ctx.lib.oct_ctx_last_error(ctx.handle)
    st, _ = _permute(ctx, perm, x, 2)
    assert st == ob._lib.ERR_ARGUMENT
