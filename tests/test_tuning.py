"""Selection logic of the autotuner's table (oct_tuning_select: no device
needed).  The library picks, for a count or a build, the row of the same
ndims and dtype nearest to the point set's log2 size and log2(1 + neighbors
per point); the shapes change how work is cut, never a result."""
import os

import pytest

from conftest import ROOT

TABLE = """# ndims dtype nlog2 nbr_log2 max_seg multi_pop fill_chunk group_cap [sub_boxes [prefetch]]
3 0 16 4 8 2 32 24 2 1  # 100k points, ~25 neighbors
3 0 19 5 16 4 64 32   # 1M points, ~33 neighbors (sub_boxes absent: 1)
2 0 21 8 4 1 128 16 4 # 4M points 2D, ~390 neighbors
3 1 16 4 1 1 64 8 1   # Float64
"""


def select(ob, path, ndims, dtype, n, nbrs):
    import ctypes as C
    lib = ob._lib.load()
    shapes = (C.c_int32 * 6)()
    row = C.c_int32(-9)
    st = lib.oct_tuning_select(path.encode(), ndims, dtype, n, float(nbrs), shapes, C.byref(row))
    return st, list(shapes), row.value


def test_nearest_row_of_the_same_kind(ob, tmp_path):
    p = tmp_path / "t.tsv"
    p.write_text(TABLE)
    assert select(ob, str(p), 3, 0, 100_000, 25.6) == (0, [8, 2, 32, 24, 2, 1], 0)
    assert select(ob, str(p), 3, 0, 1_000_000, 28.3) == (0, [16, 4, 64, 32, 1, 0], 1)
    assert select(ob, str(p), 3, 0, 2_000_000, 14.3) == (0, [16, 4, 64, 32, 1, 0], 1)  # nearer in size than in neighbors
    assert select(ob, str(p), 2, 0, 4_000_000, 387.0) == (0, [4, 1, 128, 16, 4, 0], 2)
    assert select(ob, str(p), 3, 1, 5_000, 0.5) == (0, [1, 1, 64, 8, 1, 0], 3)
    # no row of that kind: the built-in defaults
    assert select(ob, str(p), 2, 1, 1000, 10) == (0, [16, 4, 0, 32, 1, 0], -1)
    # neighbors not known yet (before a first count): keyed as ~15 per point
    assert select(ob, str(p), 3, 0, 100_000, -1) == (0, [8, 2, 32, 24, 2, 1], 0)


def test_no_table_and_bad_tables(ob, tmp_path):
    assert select(ob, "", 3, 0, 100_000, 25) == (0, [16, 4, 0, 32, 1, 0], -1)
    for bad in ("3 0 16 4 8 2 32\n", "3 0 16 4 8 2 48 24\n", "3 0 16 4 8 9 32 24\n", "4 0 16 4 8 2 32 24\n",
                "3 0 16 4 8 2 32 24 3\n", "3 0 16 4 8 2 32 24 2 9\n",
                "3 0 16 4 8 2 32 24 2 0 5\n"):
        p = tmp_path / "bad.tsv"
        p.write_text(bad)
        st, _, _ = select(ob, str(p), 3, 0, 1000, 1)
        assert st == ob._lib.ERR_ARGUMENT, bad
    st, _, _ = select(ob, str(tmp_path / "missing.tsv"), 3, 0, 1000, 1)
    assert st == ob._lib.ERR_ARGUMENT


def test_packaged_table_parses_and_covers_the_benchmark_configurations(ob):
    path = os.path.join(ROOT, "octopus.jl_b200", "tuning.tsv")
    if not os.path.exists(path):
        pytest.skip("no tuning table packaged yet")
    for ndims, n, nbrs in ((3, 100_000, 25.6), (3, 1_000_000, 28.3), (2, 4_000_000, 387.0), (3, 2_000_000, 14.3)):
        st, shapes, row = select(ob, path, ndims, 0, n, nbrs)
        assert st == 0 and row >= 0, (ndims, n)
        assert shapes[2] in (0, 32, 64, 128) and 8 <= shapes[3] <= 32
