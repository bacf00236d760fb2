"""materialize_all_neighbors! on the GPU (CSR neighbor lists).  The reference
wires it for a CPU TNS only (src/api.jl:349-362, materialize_cpu! in
src/cpu/query_cpu.jl:149-192); its rows must equal the CPU path's: offsets
from 0, 1-based target indices in traversal order, the self pair excluded
for a self pair (qid == tid)."""
import numpy as np
import pytest
import torch

from conftest import uniform

pytestmark = pytest.mark.gpu


def tns_for(ob, sets, r, pairs):
    T = torch.float32 if sets[0].dtype == np.float32 else torch.float64
    tns = ob.TNS(T, ndims=sets[0].shape[1])
    ob.set_search_radius_(tns, r)
    ids = [ob.add_point_set_(tns, torch.from_numpy(x).cuda().t()) for x in sets]
    for q, t in pairs:
        ob.set_active_search_(tns, ids[q], ids[t])
    ob.run_(tns)
    return tns, ids


@pytest.mark.parametrize("d,dtype,r", [(3, np.float32, 0.07), (2, np.float32, 0.02), (3, np.float64, 0.06)])
def test_csr_equals_oracle(ob, oracle_mod, d, dtype, r):
    x = uniform(6000, d, 300 + d, dtype=dtype)
    r = dtype(r)
    tns, ids = tns_for(ob, [x], r, [(0, 0)])
    ob.materialize_all_neighbors_(tns)
    nb = tns.neighbor_buffers[0]
    assert nb.materialized
    oe = oracle_mod.build_edges(oracle_mod.build_tree(x, r), x, exclude_self=True)
    assert nb.offsets.dtype == torch.int32 and nb.offsets.numel() == len(x) + 1
    assert np.array_equal(nb.offsets.cpu().numpy().astype(np.int64), np.asarray(oe["offsets"], np.int64))
    assert np.array_equal(nb.flat.cpu().numpy(), oe["senders"])


def test_csr_cross_pair_keeps_self_index(ob, oracle_mod):
    """qid != tid: no self exclusion (src/cpu/query_cpu.jl:176)."""
    a = uniform(2500, 3, 311)
    b = uniform(3500, 3, 312)
    r = np.float32(0.09)
    tns, ids = tns_for(ob, [a, b], r, [(0, 1), (1, 0)])
    ob.materialize_all_neighbors_(tns)
    for pidx, (q, t) in enumerate([(a, b), (b, a)]):
        nb = tns.neighbor_buffers[pidx]
        oe = oracle_mod.build_edges(oracle_mod.build_tree(t, r), q, exclude_self=False)
        assert np.array_equal(nb.flat.cpu().numpy(), oe["senders"])
        assert np.array_equal(nb.offsets.cpu().numpy().astype(np.int64), np.asarray(oe["offsets"], np.int64))


def test_csr_agrees_with_build_edges(ob):
    """test/edges_cpu.jl:126-157, here row by row in order."""
    x = uniform(4000, 3, 51)
    r = np.float32(0.07)
    tns, ids = tns_for(ob, [x], r, [(0, 0)])
    ob.materialize_all_neighbors_(tns)
    e = ob.build_edges(tns, ids[0], ids[0])
    nb = tns.neighbor_buffers[0]
    assert torch.equal(nb.flat, e.senders)
    rows = torch.repeat_interleave(torch.arange(1, len(x) + 1, device="cuda", dtype=torch.int32),
                                   (nb.offsets[1:] - nb.offsets[:-1]).long())
    assert torch.equal(rows, e.receivers)


def test_run_invalidates_materialized(ob):
    """test/contracts.jl:252-271."""
    x = uniform(150, 3, 1012)
    tns, ids = tns_for(ob, [x], np.float32(0.1), [(0, 0)])
    ob.materialize_all_neighbors_(tns)
    ob.build_edges(tns, ids[0], ids[0])
    assert tns.neighbor_buffers[0].materialized and tns.edge_buffers[0].materialized
    ob.run_(tns)
    assert not tns.neighbor_buffers[0].materialized
    assert not tns.edge_buffers[0].materialized


def test_empty_point_set(ob):
    """test/edge_cases.jl:42-53."""
    tns = ob.TNS(torch.float32)
    ob.set_search_radius_(tns, 0.1)
    sid = ob.add_point_set_(tns, torch.empty((3, 0), device="cuda"))
    ob.set_active_search_(tns, sid, sid)
    ob.run_(tns)
    ob.materialize_all_neighbors_(tns)
    nb = tns.neighbor_buffers[0]
    assert nb.materialized and nb.flat.numel() == 0 and int(nb.offsets[0]) == 0


def test_float64_csr_agrees_with_get_neighborlist(ob):
    """test/float64.jl:93-110."""
    x = uniform(300, 3, 4004, dtype=np.float64)
    tns, ids = tns_for(ob, [x], 0.1, [(0, 0)])
    ob.materialize_all_neighbors_(tns)
    nb = tns.neighbor_buffers[0]
    off = nb.offsets.cpu().numpy()
    flat = nb.flat.cpu().numpy()
    for i in range(1, len(x) + 1, 7):
        got = np.sort(flat[off[i - 1]:off[i]])
        want = np.sort(np.asarray(ob.get_neighborlist(tns, ids[0], ids[0], i)))
        assert np.array_equal(got, want)
