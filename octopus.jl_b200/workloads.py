"""Seeded synthetic inputs with the shapes of the benchmark configurations,
and a small runner used for device profiling.

    python octopus.jl_b200/workloads.py <workload> [--steps S] [--scale F]

runs S time steps of run! + build_edges on cuda:0 (used as the target of
ncu captures; it prints the edge count per step; ``--stats`` adds the count
pass's traversal statistics).

Workloads (float32):
  uniform100k  3D, 100,000 points U[0,1)^3, r = 0.04
  sph          3D, 100^3 lattice, h = 0.01, jitter +-0.1h, r = 2h, Gaussian
               steps of sigma = 0.005h (``--scale`` shrinks the lattice side)
  mix2d        2D, 4,000,000 points: 64 Gaussians (sigma U[0.005, 0.05],
               Dirichlet(1) weights) + 10% uniform, in [0,1)^2, r = 0.002
  diff2m       3D, 2,000,000 points U[0,1)^3, r = 0.012
  batch512     3D, 512 clouds, sizes log-uniform in [500, 20000], each U[0,1)^3,
               radius U[0.03, 0.08] per cloud, one batched build + COO
  build16m     3D, 16,000,000 points U[0,1)^3, r = 0.006: run! alone (full sort path)
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

H = 0.01


def lattice(per: int, seed: int, h: float = H, jitter: float = 0.1 * H, ndims: int = 3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(*[np.arange(per)] * ndims, indexing="ij"), -1).reshape(-1, ndims).astype(np.float64)
    return (g * h + rng.uniform(-jitter, jitter, g.shape)).astype(np.float32)


def sph_snapshots(per: int, nsteps: int, seed: int, sigma: float = 0.005 * H) -> list[np.ndarray]:
    """Coordinates of time steps 0..nsteps-1: a jittered lattice moved by
    independent Gaussian displacements each step."""
    rng = np.random.default_rng(seed + 1)
    x = lattice(per, seed)
    out = [x]
    for _ in range(nsteps - 1):
        x = (x + rng.normal(0.0, sigma, x.shape)).astype(np.float32)
        out.append(x)
    return out


def uniform(n: int, ndims: int, seed: int, dtype=np.float32) -> np.ndarray:
    return np.random.default_rng(seed).random((n, ndims)).astype(dtype)


def gaussian_mixture_2d(n: int, k: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    centers = rng.random((k, 2))
    sig = rng.uniform(0.005, 0.05, k)
    w = rng.dirichlet(np.ones(k))
    nb = n // 10
    comp = rng.choice(k, size=n - nb, p=w)
    pts = centers[comp] + sig[comp, None] * rng.standard_normal((n - nb, 2))
    bad = ((pts < 0) | (pts >= 1)).any(1)
    while bad.any():
        pts[bad] = centers[comp[bad]] + sig[comp[bad], None] * rng.standard_normal((int(bad.sum()), 2))
        bad = ((pts < 0) | (pts >= 1)).any(1)
    return np.concatenate([pts, rng.random((nb, 2))]).astype(np.float32)


def traversal_stats(ob, tns, sid) -> dict:
    """The count pass's traversal statistics for the self pair of set `sid`
    (oct_edges_traversal_stats), with the derived ratios."""
    import ctypes as C
    names = ob._lib.TRAVERSAL_STATS
    buf = (C.c_uint64 * len(names))()
    ctx = tns._ctx
    ctx.bind_stream()
    h = tns.trees[sid - 1].handle
    ctx.check(ctx.lib.oct_edges_traversal_stats(ctx.handle, h, h, 1, buf, len(names)), "traversal stats")
    st = {k: int(v) for k, v in zip(names, buf)}
    hits = max(st["hits"], 1)
    st["pair_tests_per_hit"] = st["pair_tests"] / hits
    st["targets_per_chunk"] = st["targets_staged"] / max(st["leaf_chunks"], 1)
    st["steps_per_chunk"] = st["pair_steps"] / max(st["leaf_chunks"], 1)
    st["chunks_per_group"] = st["leaf_chunks"] / max(st["groups"], 1)
    st["expansions_per_group"] = st["expansions"] / max(st["groups"], 1)
    st["cycle_share_leaf"] = st["cycles_leaf"] / max(st["cycles_total"], 1)
    st["cycle_share_pairs"] = st["cycles_pairs"] / max(st["cycles_total"], 1)
    return st


def _run(name: str, steps: int, scale: float, stats: bool = False):
    import torch
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    import __graft_entry__
    ob = __graft_entry__.load_package()
    if name == "sph":
        per = max(4, int(round(100 * scale)))
        xs = sph_snapshots(per, steps, 12345)
        r = 2 * H
    elif name == "uniform100k":
        xs = [uniform(int(100_000 * scale), 3, 2024)] * steps
        r = 0.04
    elif name == "mix2d":
        xs = [gaussian_mixture_2d(int(4_000_000 * scale), 64, 2026)] * steps
        r = 0.002
    elif name == "diff2m":
        xs = [uniform(int(2_000_000 * scale), 3, 2025)] * steps
        r = 0.012 / scale ** (1 / 3)  # same neighbors per point at every scale
    elif name == "batch512":
        return _run_batch(ob, torch, steps)
    elif name == "build16m":
        return _run_build(ob, torch, uniform(int(16_000_000 * scale), 3, 2031), 0.006 / scale ** (1 / 3), steps)
    else:
        raise SystemExit(f"unknown workload {name}")
    if name == "diff2m":
        return _run_diff(ob, torch, xs, r)
    d = xs[0].shape[1]
    tns = ob.TNS(torch.float32, ndims=d)
    ob.set_search_radius_(tns, r)
    ob.set_refit_mode_(tns, True)
    dev = [torch.from_numpy(x).cuda().t() for x in xs]
    sid = ob.add_point_set_(tns, dev[0])
    ob.set_active_search_(tns, sid, sid)
    for x in dev:
        ob.update_point_set_(tns, sid, x)
        ob.run_(tns)
        e = ob.build_edges(tns, sid, sid)
        ob.synchronize(tns)
        print(f"{name}: n={x.shape[1]} edges={e.senders.numel()}")
    if stats:
        import json
        print(json.dumps(traversal_stats(ob, tns, sid)))


def _run_build(ob, torch, x, r, steps):
    """run! alone (full sort path every step: refit mode off)."""
    tns = ob.TNS(torch.float32, ndims=3)
    ob.set_search_radius_(tns, r)
    xd = torch.from_numpy(x).cuda().t()
    sid = ob.add_point_set_(tns, xd)
    ob.set_active_search_(tns, sid, sid)
    for _ in range(steps):
        ob.update_point_set_(tns, sid, xd)
        ob.run_(tns)
        ob.synchronize(tns)
        print(f"build16m: n={x.shape[0]} nodes={tns.trees[sid - 1].n_nodes}")


def batch_clouds(n_clouds: int = 512, seed: int = 4):
    """Sizes log-uniform in [500, 20000], points U[0,1)^3, radii U[0.03, 0.08]."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(500), np.log(20000), n_clouds)).astype(np.int64)
    radii = rng.uniform(0.03, 0.08, n_clouds)
    clouds = [rng.random((int(n), 3)).astype(np.float32) for n in sizes]
    return clouds, sizes, radii


def _run_batch(ob, torch, steps):
    clouds, sizes, radii = batch_clouds()
    cat = torch.from_numpy(np.concatenate(clouds)).cuda().t()
    bs = ob.BatchedSearch(torch.float32, 3)
    for _ in range(steps):
        e = bs.run_(cat, sizes, radii).build_edges()
        torch.cuda.synchronize()
        print(f"batch512: n={int(sizes.sum())} edges={e.senders.numel()}")


def _run_diff(ob, torch, xs, r):
    """build_edges_diff forward + adjoint, with the library's phase times."""
    import ctypes as C
    tns = ob.TNS(torch.float32, ndims=3)
    ob.set_search_radius_(tns, r)
    c0 = torch.from_numpy(xs[0]).cuda().t()
    sid = ob.add_point_set_(tns, c0)
    ob.set_active_search_(tns, sid, sid)
    lib, ctx = tns._ctx.lib, tns._ctx
    nph = len(ob._lib.PHASES)
    ms = (C.c_double * nph)()
    cnt = (C.c_int64 * nph)()
    for step, x in enumerate(xs):
        c = torch.from_numpy(x).cuda().t().requires_grad_(True)
        lib.oct_profile_enable(ctx.handle, 1)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record()
        ob.update_point_set_(tns, sid, c.detach())
        ob.run_(tns)
        ev[1].record()
        e = ob.build_edges_diff(c, tns, sid, r)
        loss = (e.rel_displacement ** 2).sum() + 0.5 * (e.rel_dist_norm ** 2).sum()
        ev[2].record()
        loss.backward()
        ev[3].record()
        torch.cuda.synchronize()
        lib.oct_profile_read(ctx.handle, ms, cnt, nph)
        lib.oct_profile_enable(ctx.handle, 0)
        ph = {ob._lib.PHASES[i]: round(ms[i], 4) for i in range(nph) if cnt[i]}
        print(f"diff2m step {step}: edges={e.senders.numel()} build={ev[0].elapsed_time(ev[1]):.3f} ms "
              f"forward={ev[1].elapsed_time(ev[2]):.3f} ms backward={ev[2].elapsed_time(ev[3]):.3f} ms phases={ph}")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("workload")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--stats", action="store_true", help="print the count pass's traversal statistics")
    a = ap.parse_args()
    _run(a.workload, a.steps, a.scale, a.stats)
