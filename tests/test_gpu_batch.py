"""Batched clouds: one forest, one sort, one set of launches; every cloud's
slice of the concatenated COO must be bit-identical to what the reference
CPU path (the oracle) produces for a TNS holding that cloud alone."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def make_clouds(n_clouds, ndims, seed, smin=50, smax=3000, dtype=np.float32, extras=True):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(smin), np.log(smax), n_clouds)).astype(np.int64)
    radii = rng.uniform(0.03, 0.08, n_clouds)
    clouds = [rng.random((int(s), ndims)).astype(dtype) for s in sizes]
    if extras:
        clouds[1] = np.zeros((0, ndims), dtype)                      # empty cloud
        clouds[2] = rng.random((1, ndims)).astype(dtype)             # single point
        clouds[3] = np.zeros((60, ndims), dtype) + dtype(0.5)        # coincident points
        clouds[4] = (rng.random((400, ndims)) * 10 - 5).astype(dtype)  # other box, offset origin
    sizes = np.array([len(c) for c in clouds], np.int64)
    radii = np.array([float(dtype(r)) for r in radii])
    return clouds, sizes, radii


def run_batch(ob, clouds, sizes, radii, dtype):
    T = torch.float32 if dtype == np.float32 else torch.float64
    ndims = clouds[0].shape[1]
    cat = np.concatenate(clouds) if len(clouds) else np.zeros((0, ndims), dtype)
    bs = ob.BatchedSearch(T, ndims)
    bs.run_(torch.from_numpy(np.ascontiguousarray(cat)).cuda().t(), sizes, radii)
    e = bs.build_edges()
    return e


def check_against_oracle(e, clouds, radii, oracle_mod):
    snd = e.senders.cpu().numpy()
    rcv = e.receivers.cpu().numpy()
    disp = e.rel_displacement.t().cpu().numpy()
    dist = e.rel_dist_norm.reshape(-1).cpu().numpy()
    eoff = e.edge_offsets
    assert eoff[-1] == len(snd)
    for c, x in enumerate(clouds):
        a, b = eoff[c], eoff[c + 1]
        r = x.dtype.type(radii[c])
        oe = oracle_mod.build_edges(oracle_mod.build_tree(x, r), x, exclude_self=True)
        assert b - a == len(oe["senders"]), f"cloud {c}"
        assert np.array_equal(snd[a:b], oe["senders"]), f"cloud {c}"
        assert np.array_equal(rcv[a:b], oe["receivers"]), f"cloud {c}"
        assert np.array_equal(disp[a:b], oe["rel_displacement"]), f"cloud {c}"
        assert np.array_equal(dist[a:b], oe["rel_dist_norm"]), f"cloud {c}"


@pytest.mark.parametrize("ndims,dtype", [(3, np.float32), (2, np.float32), (3, np.float64)])
def test_batch_matches_per_cloud_oracle(ob, oracle_mod, ndims, dtype):
    clouds, sizes, radii = make_clouds(40, ndims, 100 + ndims, dtype=dtype)
    if ndims == 2:
        radii = radii / 4
    e = run_batch(ob, clouds, sizes, radii, dtype)
    check_against_oracle(e, clouds, radii, oracle_mod)


def test_batch_repeated_runs_and_single_cloud(ob, oracle_mod):
    clouds, sizes, radii = make_clouds(12, 3, 7, extras=False)
    bs = ob.BatchedSearch(torch.float32, 3)
    for step in range(3):  # the same object re-run on moved clouds
        moved = [(c + np.float32(0.001 * step)).astype(np.float32) for c in clouds]
        cat = torch.from_numpy(np.concatenate(moved)).cuda().t()
        e = bs.run_(cat, sizes, radii).build_edges()
        check_against_oracle(e, moved, radii, oracle_mod)
    one = [clouds[0]]
    e = run_batch(ob, one, sizes[:1], radii[:1], np.float32)
    check_against_oracle(e, one, radii[:1], oracle_mod)


def test_batch_config4_shape(ob, oracle_mod):
    """512 clouds, sizes log-uniform in [500, 20000], radius U[0.03, 0.08] --
    the benchmarked batch: every cloud's slice of the concatenated COO -- all four arrays -- and the
    per-cloud edge offsets equal the oracle's per-cloud builds."""
    clouds, sizes, radii = make_clouds(512, 3, 4, smin=500, smax=20000, extras=False)
    e = run_batch(ob, clouds, sizes, radii, np.float32)
    assert e.edge_offsets[-1] == 26_680_134  # the benchmarked batch (same generator and seed)
    check_against_oracle(e, clouds, radii, oracle_mod)
