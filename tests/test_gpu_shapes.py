"""Every kernel shape the autotuner may choose gives the same tree and COO.

The tuned shapes (query points per traversal group, leaves merged into one
staged chunk, internal nodes expanded together, the fill's store path, the
group's sub-boxes, L1 prefetch in the traversal) change how the work is cut,
never a result.  Each shape is forced through the context options one value at
a time (the others left to the defaults), and once all together at their
non-default values; each run is compared with the oracle array for array."""
import numpy as np
import pytest
import torch

from conftest import clustered, lattice, uniform
from test_gpu_parity import assert_edges_equal, gpu_run, torch_dtype

pytestmark = pytest.mark.gpu

# option name (in the library's option table), forced values
SHAPES = [
    ("OPT_GROUP_CAP", (8, 16, 24, 32)),
    ("OPT_MAX_SEG", (1, 4, 8, 16)),
    ("OPT_MULTI_POP", (1, 2, 4)),
    ("OPT_FILL_CHUNK", (1, 32, 64, 128)),  # 1: direct stores; else bulk-copy chunks of that many edges
    ("OPT_SUB_BOXES", (1, 2, 4)),
    ("OPT_PREFETCH", (1, 2)),  # 1: off, 2: on
]
ALL_OTHER = {"OPT_GROUP_CAP": 16, "OPT_MAX_SEG": 8, "OPT_MULTI_POP": 2, "OPT_FILL_CHUNK": 64,
             "OPT_SUB_BOXES": 4, "OPT_PREFETCH": 2}


def _inputs():
    return {
        "uniform3d": (uniform(20_000, 3, 611), np.float32(0.05)),
        "lattice3d": (lattice(25, 3, 0.01, 0.001, 612), np.float32(0.02)),
        "clustered2d": (clustered(12_000, 2, 613), np.float32(0.02)),
        "uniform3d_f64": (uniform(8_000, 3, 614, dtype=np.float64), np.float64(0.07)),
    }


def _ctx(ob):
    return ob.api._Context.get(torch.cuda.current_device())


def _force(ob, ctx, opts):
    for name, v in opts.items():
        ctx.check(ctx.lib.oct_ctx_set_option(ctx.handle, getattr(ob._lib, name), int(v)), name)


@pytest.fixture
def shapes_reset(ob):
    ctx = _ctx(ob)
    yield ctx
    _force(ob, ctx, {name: 0 for name, _ in SHAPES})  # back to the table / defaults


def _self_pair(ob, x, r):
    tns, sid = gpu_run(ob, x, r)  # the build takes the forced group size
    return ob.build_edges(tns, sid, sid)


@pytest.mark.parametrize("case", list(_inputs()))
def test_each_shape_gives_the_oracle_coo(ob, oracle_mod, shapes_reset, case):
    x, r = _inputs()[case]
    want = oracle_mod.build_edges(oracle_mod.build_tree(x, r), x, exclude_self=True)
    ctx = shapes_reset
    for name, values in SHAPES:
        for v in values:
            _force(ob, ctx, {name: v})
            e = _self_pair(ob, x, r)
            assert_edges_equal(e, want)
        _force(ob, ctx, {name: 0})
    _force(ob, ctx, ALL_OTHER)
    assert_edges_equal(_self_pair(ob, x, r), want)


def test_shapes_on_a_cross_pair(ob, oracle_mod, shapes_reset):
    """Query set A against target set B (no self exclusion, no per-group start
    node): the fill store paths and the traversal shapes."""
    a = uniform(3000, 3, 621)
    b = uniform(5000, 3, 622)
    r = np.float32(0.1)
    want = oracle_mod.build_edges(oracle_mod.build_tree(b, r), a, exclude_self=False)
    ctx = shapes_reset
    for opts in ({"OPT_FILL_CHUNK": 1}, {"OPT_FILL_CHUNK": 32}, {"OPT_FILL_CHUNK": 128}, {"OPT_MAX_SEG": 1},
                 {"OPT_SUB_BOXES": 2}, {"OPT_GROUP_CAP": 8}, ALL_OTHER):
        _force(ob, ctx, {name: 0 for name, _ in SHAPES})
        _force(ob, ctx, opts)
        tns = ob.TNS(torch_dtype(a))
        ob.set_search_radius_(tns, r)
        ia = ob.add_point_set_(tns, torch.from_numpy(a).cuda().t())
        ib = ob.add_point_set_(tns, torch.from_numpy(b).cuda().t())
        ob.set_active_search_(tns, ia, ib)
        ob.run_(tns)
        assert_edges_equal(ob.build_edges(tns, ia, ib), want)
