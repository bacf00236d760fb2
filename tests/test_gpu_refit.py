"""Refit mode across time steps: each step re-encodes the points in the
previous sorted order and merges the changed keys in (or, when no key
changed, recomputes the bounds only).  The reference rebuilds fully on every
run! (test/refit.jl:15-40, 63-86), so every step must equal the oracle's full
build of that step's coordinates bit for bit: tree, permutation, Morton codes
and COO."""
import numpy as np
import pytest
import torch

from conftest import lattice, uniform
from test_gpu_parity import assert_edges_equal, assert_tree_equal

pytestmark = pytest.mark.gpu


def morton_keys(oracle_mod, x, r):
    return oracle_mod.build_tree(x, r).morton


class Stepper:
    """One TNS in refit mode, stepped through update_point_set! + run!."""

    def __init__(self, ob, x0, r):
        self.ob = ob
        self.T = torch.float32 if x0.dtype == np.float32 else torch.float64
        self.tns = ob.TNS(self.T, ndims=x0.shape[1])
        ob.set_search_radius_(self.tns, r)
        ob.set_refit_mode_(self.tns, True)
        self.sid = ob.add_point_set_(self.tns, torch.from_numpy(x0).cuda().t())
        ob.set_active_search_(self.tns, self.sid, self.sid)
        self.r = r

    def step(self, x):
        ob = self.ob
        ob.update_point_set_(self.tns, self.sid, torch.from_numpy(x).cuda().t())
        ob.run_(self.tns)
        return self.tns.trees[self.sid - 1].last_build()

    def check(self, oracle_mod, x):
        ot = oracle_mod.build_tree(x, self.r)
        tree = self.tns.trees[self.sid - 1]
        assert_tree_equal(tree, ot)
        if self.tns.refit_mode:
            assert np.array_equal(tree.arrays()["morton"].cpu().numpy().view(np.uint64), ot.morton)
        e = self.ob.build_edges(self.tns, self.sid, self.sid)
        assert_edges_equal(e, oracle_mod.build_edges(ot, x, exclude_self=True), self.tns)


@pytest.mark.parametrize("ndims,dtype", [(3, np.float32), (2, np.float32), (3, np.float64)])
def test_time_steps_equal_full_rebuild(ob, oracle_mod, ndims, dtype):
    """A jittered lattice moved by small Gaussian steps (the SPH workload's
    shape at 24^3 / 150^2 points), with some larger steps mixed in."""
    per = 24 if ndims == 3 else 150
    x = lattice(per, ndims, 0.01, 0.001, 60 + ndims).astype(dtype)
    r = dtype(0.02)
    rng = np.random.default_rng(61)
    st = Stepper(ob, x, r)
    assert st.step(x) == (0, -1)  # first build: full sort
    st.check(oracle_mod, x)
    paths = []
    for k, sigma in enumerate([5e-5, 5e-5, 2e-4, 1e-3, 5e-5, 3e-3]):
        prev_keys = morton_keys(oracle_mod, x, r)
        x = (x + rng.normal(0.0, sigma, x.shape)).astype(dtype)
        path, moved = st.step(x)
        changed = int((morton_keys(oracle_mod, x, r) != prev_keys).sum())
        assert moved == changed, f"step {k}"
        paths.append(path)
        st.check(oracle_mod, x)
    assert 1 in paths


def test_unchanged_keys_refit_bounds_only(ob, oracle_mod):
    """Points that move inside their cells keep every key: the order and the
    topology are kept and only the bounds change."""
    x = lattice(20, 3, 0.01, 0.001, 70)
    r = np.float32(0.02)
    st = Stepper(ob, x, r)
    st.step(x)
    assert st.step(x) == (2, 0)  # the same coordinates again
    st.check(oracle_mod, x)
    # Shrink every point 1% toward its cell's centre: the cells stay put
    # only if the origin (min - 1e-6) does, so pin the minimum corner point.
    keys0 = morton_keys(oracle_mod, x, r)
    o = x.min(0) - np.float32(1e-6)
    cell = np.floor((x - o) / r)
    centre = o + (cell + 0.5) * r
    y = (x + np.float32(0.01) * (centre - x)).astype(np.float32)
    y[np.argmin(x[:, 0])] = x[np.argmin(x[:, 0])]
    y[np.argmin(x[:, 1])] = x[np.argmin(x[:, 1])]
    y[np.argmin(x[:, 2])] = x[np.argmin(x[:, 2])]
    expect = 2 if np.array_equal(morton_keys(oracle_mod, y, r), keys0) else 1
    assert st.step(y)[0] == expect
    st.check(oracle_mod, y)


def test_many_changed_keys_use_several_chunks(ob, oracle_mod):
    """About 6,000 relocated points: the changed keys span several sorted
    chunks that are ranked against each other before the merge."""
    x = uniform(100_000, 3, 71)
    r = np.float32(0.03)
    st = Stepper(ob, x, r)
    st.step(x)
    rng = np.random.default_rng(72)
    y = x.copy()
    pick = rng.choice(len(x), 6000, replace=False)
    y[pick] = rng.random((6000, 3)).astype(np.float32) * np.float32(0.999) + np.float32(0.0005)
    path, moved = st.step(y)
    assert path == 1 and 4096 < moved <= 6000
    st.check(oracle_mod, y)


def test_large_change_falls_back_to_full_sort(ob, oracle_mod):
    x = uniform(20_000, 3, 73)
    r = np.float32(0.05)
    st = Stepper(ob, x, r)
    st.step(x)
    y = uniform(20_000, 3, 74)  # every point somewhere else
    path, moved = st.step(y)
    assert path == 0 and moved > 2500
    st.check(oracle_mod, y)
    z = (y + np.float32(1e-4)).astype(np.float32)  # then small steps again
    assert st.step(z)[0] in (1, 2)
    st.check(oracle_mod, z)


def test_new_radius_or_size_rebuilds(ob, oracle_mod):
    x = uniform(5000, 3, 75)
    r = np.float32(0.05)
    st = Stepper(ob, x, r)
    st.step(x)
    ob.set_search_radius_(st.tns, np.float32(0.07))
    st.r = np.float32(0.07)
    assert st.step(x) == (0, -1)
    st.check(oracle_mod, x)
    y = uniform(6000, 3, 76)
    ob.resize_point_set_(st.tns, st.sid, torch.from_numpy(y).cuda().t())
    ob.run_(st.tns)
    assert st.tns.trees[st.sid - 1].last_build() == (0, -1)
    st.check(oracle_mod, y)


def test_refit_mode_off_always_sorts(ob, oracle_mod):
    x = uniform(3000, 3, 77)
    r = np.float32(0.05)
    st = Stepper(ob, x, r)
    ob.set_refit_mode_(st.tns, False)
    st.step(x)
    assert st.step(x) == (0, -1)
    st.check(oracle_mod, x)


def test_speculative_merge_fallbacks(ob, oracle_mod):
    """After a merging step the next build merges before it has read the
    bounds; when the merge does not apply (too many changed keys, a key past
    the key width, a non-finite coordinate) the build is redone on the usual
    path, with the same result as a full rebuild."""
    x = uniform(20_000, 3, 80)
    r = np.float32(0.05)
    rng = np.random.default_rng(81)
    st = Stepper(ob, x, r)
    st.step(x)

    def relocate(z, k):
        z = z.copy()
        pick = rng.choice(len(z), k, replace=False)
        z[pick] = rng.random((k, 3)).astype(np.float32) * np.float32(0.99) + np.float32(0.005)
        return z

    y = relocate(x, 40)
    assert st.step(y)[0] == 1  # merged
    st.check(oracle_mod, y)
    z = relocate(y, 8000)  # beyond the merge capacity (2,500 here)
    path, moved = st.step(z)
    assert path == 0 and moved > 2500
    st.check(oracle_mod, z)
    w = relocate(z, 40)
    assert st.step(w)[0] == 1
    v = w.copy()
    v[123] = np.float32(900.0)  # 18,000 cells per axis: the key no longer fits 32 bits
    path, _ = st.step(v)
    assert path == 0
    st.check(oracle_mod, v)
    u = relocate(v, 30)
    assert st.step(u)[0] == 1
    bad = u.copy()
    bad[7, 1] = np.float32(np.nan)
    with pytest.raises(ob.InexactError):
        st.step(bad)
    assert st.step(u)[0] == 0  # rebuilt in full after the error
    st.check(oracle_mod, u)
