"""The stable key sort of run!, through the tree's permutation, against the
oracle's stable sort (src/sort.jl:15-24: ties keep ascending original index).

Sizes sit at and around the sort's 2048-key tiles, and the points are drawn
from a handful of positions, so most keys tie: the ranks of equal keys across
tiles, and the prefixes each tile takes from the tiles before it, decide the
permutation.  One size runs the staged passes used from 6M keys on."""
import numpy as np
import pytest
import torch

from test_gpu_parity import assert_tree_equal, gpu_run

pytestmark = pytest.mark.gpu


def tied_points(n, n_sites, seed):
    rng = np.random.default_rng(seed)
    sites = rng.random((n_sites, 3)).astype(np.float32)
    return sites[rng.integers(0, n_sites, n)]


@pytest.mark.parametrize("n", [1, 2047, 2048, 2049, 6143, 6144, 6145, 100_003])
def test_sort_with_ties_matches_oracle(ob, oracle_mod, n):
    x = tied_points(n, 7, 900 + n % 97)
    r = np.float32(0.05)
    tns, sid = gpu_run(ob, x, r)
    ot = oracle_mod.build_tree(x, r)
    assert np.array_equal(tns.trees[sid - 1].arrays()["perm"].cpu().numpy(), ot.perm)


@pytest.mark.parametrize("n", [4099, 150_000])
def test_sort_uniform_matches_oracle(ob, oracle_mod, n):
    x = np.random.default_rng(n).random((n, 3)).astype(np.float32)
    r = np.float32(0.01)
    tns, sid = gpu_run(ob, x, r)
    assert_tree_equal(tns.trees[sid - 1], oracle_mod.build_tree(x, r))


def test_sort_of_6_5m_keys_with_ties(ob, oracle_mod):
    """6.5M keys (3,174 tiles of the point-carrying passes, 5,000 points per
    tied cell): the permutation is the oracle's."""
    n = 6_500_000
    x = tied_points(n, 5000, 77)
    r = np.float32(0.004)
    tns, sid = gpu_run(ob, x, r)
    ot = oracle_mod.build_tree(x, r, nthreads=0)
    assert np.array_equal(tns.trees[sid - 1].arrays()["perm"].cpu().numpy(), ot.perm)
