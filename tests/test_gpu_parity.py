"""GPU parity with the CPU oracle, through the C ABI (via the TNS mirror).

Bar: bit-exact.  Trees (BFS node numbering, ranges, children, bounds,
permutation) and the full COO -- senders, receivers, rel_displacement and
rel_dist_norm, in the reference's order -- must equal the oracle's arrays
exactly."""
import numpy as np
import pytest
import torch

from conftest import clustered, lattice, uniform

pytestmark = pytest.mark.gpu


def gaussian_mixture_2d(n, k, seed, dtype=np.float32):
    """Nonuniform 2D shape: k isotropic Gaussians (sigma in [0.005, 0.05],
    Dirichlet(1) weights) plus 10% uniform background, redrawn into [0,1)^2."""
    rng = np.random.default_rng(seed)
    centers = rng.random((k, 2))
    sig = rng.uniform(0.005, 0.05, k)
    w = rng.dirichlet(np.ones(k))
    nb = n // 10
    comp = rng.choice(k, size=n - nb, p=w)
    pts = centers[comp] + sig[comp, None] * rng.standard_normal((n - nb, 2))
    bad = ((pts < 0) | (pts >= 1)).any(1)
    while bad.any():
        pts[bad] = centers[comp[bad]] + sig[comp[bad], None] * rng.standard_normal((bad.sum(), 2))
        bad = ((pts < 0) | (pts >= 1)).any(1)
    return np.concatenate([pts, rng.random((nb, 2))]).astype(dtype)


CASES = {
    "u3d_2k": (lambda: uniform(2000, 3, 1), 0.08),
    "u3d_20k_dense": (lambda: uniform(20000, 3, 2), 0.04),
    "clustered3d": (lambda: clustered(5000, 3, 3), 0.03),
    "clustered3d_small_r": (lambda: (0.1 * np.random.default_rng(31).standard_normal((2000, 3))).astype(np.float32), 0.03),
    "lattice3d": (lambda: lattice(20, 3, 0.01, 0.001, 4), 0.02),
    "neg3d": (lambda: uniform(3000, 3, 5, -1.0, 1.0), 0.1),
    "u2d_20k": (lambda: uniform(20000, 2, 6), 0.01),
    "mix2d_50k": (lambda: gaussian_mixture_2d(50000, 16, 7), 0.002),
    "lattice2d": (lambda: lattice(120, 2, 0.01, 0.001, 8), 0.02),
    "f64_3d": (lambda: uniform(3000, 3, 9, dtype=np.float64), 0.07),
    "f64_2d": (lambda: uniform(3000, 2, 10, dtype=np.float64), 0.03),
    "big_leaves": (lambda: np.repeat(uniform(40, 3, 11), 50, axis=0), 0.2),
    "wide_extent": (lambda: uniform(5000, 3, 12, 0.0, 1000.0), 7.5),
    "tiny_r": (lambda: uniform(2000, 3, 13), 1e-8),
    "huge_r": (lambda: uniform(300, 3, 14), 100.0),
    "coincident": (lambda: np.zeros((100, 3), np.float32), 0.1),
    "u64_keys_3d": (lambda: uniform(5000, 3, 17, 0.0, 1000.0), 0.3),
    "u64_keys_2d": (lambda: uniform(5000, 2, 18, 0.0, 1e5), 1.0),
    "l_shape": (lambda: np.concatenate([uniform(1500, 3, 15) * [1, 0.2, 0.2], uniform(1500, 3, 16) * [0.2, 1, 0.2]]).astype(np.float32), 0.03),
}


def torch_dtype(x):
    return torch.float32 if x.dtype == np.float32 else torch.float64


def gpu_run(ob, x, r):
    d = x.shape[1]
    tns = ob.TNS(torch_dtype(x), ndims=d)
    ob.set_search_radius_(tns, r)
    sid = ob.add_point_set_(tns, torch.from_numpy(x).cuda().t())
    ob.set_active_search_(tns, sid, sid)
    ob.run_(tns)
    return tns, sid


def assert_tree_equal(tree, ot):
    a = tree.arrays()
    assert a["n_nodes"] == ot.n_nodes
    assert np.array_equal(a["node_first"].cpu().numpy(), ot.node_first)
    assert np.array_equal(a["node_last"].cpu().numpy(), ot.node_last)
    assert np.array_equal(a["node_children"].t().cpu().numpy(), ot.children)
    assert np.array_equal(a["node_bounds_min"].t().cpu().numpy(), ot.bmin)
    assert np.array_equal(a["node_bounds_max"].t().cpu().numpy(), ot.bmax)
    assert np.array_equal(a["perm"].cpu().numpy(), ot.perm)


def describe_mismatch(e, oe):
    """Where the GPU COO first departs from the oracle's, for the failure message."""
    gs, gr = e.senders.cpu().numpy(), e.receivers.cpu().numpy()
    os_, or_ = oe["senders"], oe["receivers"]
    msg = [f"n_edges gpu={len(gs)} oracle={len(os_)}"]
    m = min(len(gs), len(os_))
    bad = np.nonzero((gs[:m] != os_[:m]) | (gr[:m] != or_[:m]))[0]
    if len(bad):
        k = int(bad[0])
        i = int(or_[k])
        off = oe["offsets"]
        seg_o = os_[off[i - 1]:off[i]]
        seg_g = gs[gr == i]
        msg.append(f"first diff at edge {k}: receiver gpu={gr[k]} oracle={i}; diffs={len(bad)}")
        msg.append(f"receiver {i}: same set={sorted(seg_g.tolist()) == sorted(seg_o.tolist())} "
                   f"gpu={seg_g.tolist()[:40]} oracle={seg_o.tolist()[:40]}")
    return "; ".join(msg)


def assert_edges_equal(e, oe, tns=None):
    if tns is not None:
        import octopus_b200
        octopus_b200.synchronize(tns)
    assert np.array_equal(e.senders.cpu().numpy(), oe["senders"]), describe_mismatch(e, oe)
    assert np.array_equal(e.receivers.cpu().numpy(), oe["receivers"])
    assert np.array_equal(e.rel_displacement.t().cpu().numpy(), oe["rel_displacement"])
    assert np.array_equal(e.rel_dist_norm.reshape(-1).cpu().numpy(), oe["rel_dist_norm"])


@pytest.mark.parametrize("name", list(CASES))
def test_tree_and_edges_bit_exact(ob, oracle_mod, name):
    gen, r = CASES[name]
    x = gen()
    r = x.dtype.type(r)
    tns, sid = gpu_run(ob, x, r)
    ot = oracle_mod.build_tree(x, r)
    assert_tree_equal(tns.trees[sid - 1], ot)
    e = ob.build_edges(tns, sid, sid)
    oe = oracle_mod.build_edges(ot, x, exclude_self=True)
    assert_edges_equal(e, oe, tns)


def test_config1_full_size(ob, oracle_mod):
    """3D uniform N=100,000, r=0.04 -- the CPU-runnable configuration."""
    x = uniform(100_000, 3, 2024)
    r = np.float32(0.04)
    tns, sid = gpu_run(ob, x, r)
    e = ob.build_edges(tns, sid, sid)
    ot = oracle_mod.build_tree(x, r)
    assert_tree_equal(tns.trees[sid - 1], ot)
    oe = oracle_mod.build_edges(ot, x, exclude_self=True)
    assert_edges_equal(e, oe, tns)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_cross_pair(ob, oracle_mod, dtype):
    """test/edges_cpu.jl:99-124: query A -> target B, no self exclusion."""
    a = uniform(1500, 3, 41, dtype=dtype)
    b = uniform(2500, 3, 42, dtype=dtype)
    r = dtype(0.12)
    tns = ob.TNS(torch_dtype(a))
    ob.set_search_radius_(tns, r)
    ia = ob.add_point_set_(tns, torch.from_numpy(a).cuda().t())
    ib = ob.add_point_set_(tns, torch.from_numpy(b).cuda().t())
    ob.set_active_search_(tns, ia, ib)
    ob.run_(tns)
    e = ob.build_edges(tns, ia, ib)
    oe = oracle_mod.build_edges(oracle_mod.build_tree(b, r), a, exclude_self=False)
    assert_edges_equal(e, oe)


def test_edges_match_brute_force_set(ob, oracle_mod):
    x = gaussian_mixture_2d(30000, 8, 99)
    r = np.float32(0.003)
    tns, sid = gpu_run(ob, x, r)
    e = ob.build_edges(tns, sid, sid)
    bs, br = oracle_mod.brute_force(x, x, r, True)
    got = np.stack([e.receivers.cpu().numpy(), e.senders.cpu().numpy()], 1)
    got = got[np.lexsort((got[:, 1], got[:, 0]))]
    assert np.array_equal(got, np.stack([br, bs], 1))
