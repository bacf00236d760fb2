#!/usr/bin/env python
"""Benchmark: edges/s of run! + build_edges on the SPH time-stepping workload.

Workload (one GPU): 1,000,000 Float32 points on a 100^3 cubic lattice,
spacing h = 0.01, uniform jitter +-0.1h, radius 2h; every step adds a
Gaussian displacement sigma = 0.005h, then update_point_set! -> run! (refit
mode) -> build_edges (count, allocate, fill).  A step is one such time step;
`value` is total edges / device time of K steps with the coordinates already
resident in HBM; `e2e` is the same through host buffers (H2D of the step's
coordinates from pinned memory, D2H of the full COO).

Under torchrun (N>1) every rank runs an independent replica of the workload
(the path has no cross-GPU exchange); the time is the max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

H = 0.01
PER = 100
RADIUS = 2 * H
JITTER = 0.1 * H
SIGMA = 0.005 * H
METRIC = "edges/s build+query+COO @1M pts; batched & fwd+bwd vs plain, exact edges"
WORKLOAD = "sph_lattice_timestep_1M"
# DRAM bytes per edge of the fill launch (k_expand_direct), from an ncu capture of
# the same kernel on the 70^3-point lattice (same density, radius and leaf
# structure): dram__bytes_read.sum + dram__bytes_write.sum = 57.2 + 178.5 MB
# for 9,623,512 edges.  The traffic is per edge, so it scales to the
# 1M-point launch by edge count.
FILL_DRAM_BYTES_PER_EDGE = 24.5


def phase_bytes(n, e, n_nodes, path, passes=3):
    """Algorithmic HBM bytes per step of the HBM-bound build phases and of
    the edge write, for float32 3D and the kernels that run in `path`
    (0 full sort: the key sort that carries the points, with the encode fused
    in; 1 refit-mode merge: k_resort_mark + k_resort_merge, which also gathers)."""
    b = {"bounds": 12 * n}                          # coordinates read once
    if path == 1:
        b["encode"] = (4 + 12 + 4 + 1) * n            # perm, gathered coords, old key in; changed flag out
        b["sort"] = (4 + 4 + 1 + 12 + 4 + 4 + 16 + 4) * n  # key, perm, flag, coords in; key, perm, point, inverse out
    else:
        # digit counts read the coordinates (12); the first pass reads them
        # again and writes key + point (12 + 20); a middle pass moves key +
        # point (20 + 20); the last also writes the permutation (20 + 20 + 4)
        # (its inverse is scattered later, on first use by the fill)
        if passes <= 1:
            b["sort"] = (12 + 12 + 20 + 4) * n
        else:
            b["sort"] = (12 + 32 + 40 * (passes - 2) + 44) * n
    b["refit"] = 16 * n + 2 * 32 * n_nodes          # sorted points in; node records read and written
    if e:
        b["fill"] = (12 + 4 * 3) * e + 8 * n        # (12 + 4D) E + 8N
    return b


def _peak_gbs():
    """Measured HBM copy bandwidth (GB/s) of MEASURED_PEAKS.json, else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


def config_dict(extra=None):
    c = {
        "workload": WORKLOAD,
        "n_points": PER ** 3,
        "ndims": 3,
        "lattice": f"{PER}^3, h={H}, jitter=+-0.1h",
        "radius": RADIUS,
        "displacement_sigma": SIGMA,
        "refit_mode": True,
        "l2": "inputs+outputs per step exceed L2: ~680 MB of COO written per step (126 MB L2)",
        "seed": 12345,
    }
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------- inputs -----
def _workloads():
    import importlib.util
    spec = importlib.util.spec_from_file_location("octopus_b200_workloads",
                                                  os.path.join(ROOT, "octopus.jl_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def snapshots_np(per, nsteps, seed):
    """Coordinates of steps 0..nsteps-1 (float32, (N,3)) on the host."""
    return _workloads().sph_snapshots(per, nsteps, seed, sigma=SIGMA)


# ------------------------------------------------------------- clocks -----
class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in out.strip().splitlines():
            p = [v.strip() for v in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                smax.append(float(p[1]))
            except ValueError:
                continue
            for nm, v in zip(names, p[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- ranks ------
def dist_setup(gpus):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(value: float, world: int, device=None) -> float:
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, world: int, device=None) -> float:
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def replica_totals(ms: float, edges: float, world: int, device=None):
    """Whole-job figures of N independent replicas: the slowest rank's time,
    the edges of all ranks, and their throughput (edges/s) over that time."""
    ms_max = max_over_ranks(ms, world, device)
    tot = sum_over_ranks(float(edges), world, device)
    return ms_max, tot, tot / (ms_max / 1e3)


def tuning_used(ob, lib, ctx, ndims, n, nbrs):
    """The tuning-table row the last count used and the shapes it gives."""
    row = C.c_int64(-1)
    lib.oct_ctx_get_option(ctx.handle, ob._lib.STAT_TUNING_ROW, C.byref(row))
    table = os.environ.get("OCTOPUS_B200_TUNING", ob.api.TUNING_TABLE)
    shapes = (C.c_int32 * 6)()
    r2 = C.c_int32(-1)
    st = lib.oct_tuning_select((table if table and os.path.exists(table) else "").encode(), ndims, 0, int(n),
                               float(nbrs), shapes, C.byref(r2))
    names = ("max_seg", "multi_pop", "fill_chunk", "group_cap", "sub_boxes", "prefetch")
    return {"table": os.path.relpath(table, ROOT) if table and os.path.exists(table) else None,
            "row": int(row.value), "shapes": dict(zip(names, list(shapes))) if st == 0 else None}


# ------------------------------------------------------------ our arm -----
def run_ours(args, rank, world, local):
    import torch
    import __graft_entry__
    ob = __graft_entry__.load_package()
    lib = ob._lib.load()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    W, K = args.warmup, args.steps
    # W warm-up steps, K timed steps, then K more steps of the same trajectory
    # with the library's phase timers on (the timed steps run without them).
    host = snapshots_np(PER, W + 2 * K, 12345 + rank)
    snaps = [torch.from_numpy(x).to(dev).t() for x in host]  # (3, N) column-major views
    N = host[0].shape[0]

    tns = ob.TNS(torch.float32, ndims=3)
    ob.set_search_radius_(tns, RADIUS)
    ob.set_refit_mode_(tns, True)
    sid = ob.add_point_set_(tns, snaps[0])
    ob.set_active_search_(tns, sid, sid)
    ctx = tns._ctx

    def step(x):
        ob.update_point_set_(tns, sid, x)
        ob.run_(tns)
        e = ob.build_edges(tns, sid, sid)
        return e.senders.numel()

    for w in range(W):
        step(snaps[w])
    torch.cuda.synchronize()
    barrier(world)

    nph = len(ob._lib.PHASES)
    ms_buf = (C.c_double * nph)()
    cnt_buf = (C.c_int64 * nph)()
    launches0 = lib.oct_profile_kernel_launches(ctx.handle)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.5)  # let the sampler start before the timed region
    stream = torch.cuda.current_stream(dev)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    edges = 0
    for k in range(K):
        edges += step(snaps[W + k])
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = t0.elapsed_time(t1)
    launches = lib.oct_profile_kernel_launches(ctx.handle) - launches0
    tuning = tuning_used(ob, lib, ctx, 3, N, edges / K / N)
    # phase breakdown: the next K steps with the per-phase event timers on
    lib.oct_profile_read(ctx.handle, ms_buf, cnt_buf, nph)  # clear
    lib.oct_profile_enable(ctx.handle, 1)
    for k in range(K):
        step(snaps[W + K + k])
    torch.cuda.synchronize()
    lib.oct_profile_read(ctx.handle, ms_buf, cnt_buf, nph)
    lib.oct_profile_enable(ctx.handle, 0)
    phases = {ob._lib.PHASES[i]: round(ms_buf[i] / K, 5) for i in range(nph) if cnt_buf[i]}
    phase_calls = {ob._lib.PHASES[i]: int(cnt_buf[i]) for i in range(nph) if cnt_buf[i]}

    # --- end to end through host buffers (pinned), same steps.  A user's
    # pipelined time loop: build_edges returns the pair's buffer, which the
    # next call overwrites (the reference's aliasing), so each step's COO is
    # first snapshotted on the device (two staging sets, in turn) and then
    # copied to the host on a copy stream while the next step computes.
    hpin = [torch.from_numpy(x).pin_memory() for x in host[:W + K]]
    dcoords = torch.empty((N, 3), dtype=torch.float32, device=dev)
    e_last = edges // K
    cap = int(e_last * 1.2) + 1024

    def coo_set(make):
        return (make((cap,), torch.int32), make((cap,), torch.int32), make((cap, 3), torch.float32),
                make((cap,), torch.float32))

    hbufs = [coo_set(lambda shape, dt: torch.empty(shape, dtype=dt).pin_memory()) for _ in range(2)]
    stage = [coo_set(lambda shape, dt: torch.empty(shape, dtype=dt, device=dev)) for _ in range(2)]
    copy_stream = torch.cuda.Stream(device=dev)
    copied = [None, None]  # per staging set: its last host copy
    last = {}

    def e2e_step(k):
        dcoords.copy_(hpin[k], non_blocking=True)
        ob.update_point_set_(tns, sid, dcoords.t())
        ob.run_(tns)
        e = ob.build_edges(tns, sid, sid)
        m = e.senders.numel()
        if m > cap:
            raise RuntimeError("e2e host buffer too small")
        j = k % 2
        if copied[j] is not None:
            stream.wait_event(copied[j])  # the set's previous host copy has read it
        srcs = (e.senders, e.receivers, e.rel_displacement.t(), e.rel_dist_norm.reshape(-1))
        for st, d in zip(stage[j], srcs):
            st[:m].copy_(d, non_blocking=True)
        done = torch.cuda.Event()
        done.record(stream)
        copy_stream.wait_event(done)
        with torch.cuda.stream(copy_stream):
            for h, st in zip(hbufs[j], stage[j]):
                h[:m].copy_(st[:m], non_blocking=True)
        copied[j] = torch.cuda.Event()
        copied[j].record(copy_stream)
        last.update(k=k, m=m, e=e)
        return m

    for w in range(W):
        e2e_step(w)
    stream.wait_stream(copy_stream)
    torch.cuda.synchronize()
    barrier(world)
    t0.record(stream)
    e2e_edges = 0
    for k in range(K):
        e2e_edges += e2e_step(W + k)
    stream.wait_stream(copy_stream)  # the last step's copies are inside the timed region
    t1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = t0.elapsed_time(t1)
    # the host holds the last step's COO exactly
    jl, ml, el = last["k"] % 2, last["m"], last["e"]
    if not (torch.equal(hbufs[jl][0][:ml], el.senders.cpu()) and torch.equal(hbufs[jl][1][:ml], el.receivers.cpu())
            and torch.equal(hbufs[jl][2][:ml], el.rel_displacement.t().cpu())
            and torch.equal(hbufs[jl][3][:ml], el.rel_dist_norm.reshape(-1).cpu())):
        raise RuntimeError("e2e: the host copy of the last step's COO differs from the device's")
    del stage, last

    ms_max, tot_edges, value = replica_totals(ms, edges, world, dev)
    e2e_ms_max, tot_e2e, _ = replica_totals(e2e_ms, e2e_edges, world, dev)

    # --- roofline of the dominant HBM kernel (edge write = fill), live timing
    from_peaks = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            from_peaks = json.load(f)
    except Exception:
        pass
    peak = float(from_peaks["hbm_gbs"]) if from_peaks else 6650.0
    peak_src = "measured" if from_peaks else "fallback"
    e_per_step = edges / K
    fill_ms = phases.get("fill", float("nan"))
    fill_bytes = (12 + 4 * 3) * e_per_step + 8 * N  # (12 + 4D) E + 8N
    achieved = fill_bytes / (fill_ms / 1e3) / 1e9
    dominant = max(phases, key=phases.get) if phases else None
    path, _ = tns.trees[sid - 1].last_build()
    pb = phase_bytes(N, e_per_step, tns.trees[sid - 1].n_nodes, path)
    phase_hbm = {k: {"bytes": v, "gbs": v / (phases[k] / 1e3) / 1e9, "frac": v / (phases[k] / 1e3) / 1e9 / peak}
                 for k, v in pb.items() if phases.get(k)}

    result = None
    if rank == 0:
        sec = secondary_configs(ob, torch, dev)
        cpu = cpu_baseline(args)
        result = {
            "metric": METRIC,
            "value": value,
            "unit": "edges/s",
            "n_gpus": world,
            "steps": K,
            "warmup": W,
            "ms_per_step": ms_max / K,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded jittered lattice + Gaussian steps)",
            "config": config_dict({"edges_per_step": e_per_step, "parallelism": f"replicas x{world}"}),
            "e2e": {"value": tot_e2e / (e2e_ms_max / 1e3), "unit": "edges/s",
                    "h2d_bytes_per_step": N * 12, "d2h_bytes_per_step": int(24 * e2e_edges / K),
                    "ms_per_step": e2e_ms_max / K},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_src, "kernel": "fill (k_expand_direct)",
                         "traffic": (args.fill_traffic if args.fill_traffic is not None
                                     else FILL_DRAM_BYTES_PER_EDGE * e_per_step),
                         "traffic_source": "ncu dram bytes/edge of the fill kernel on the 343k-point "
                                           "lattice, scaled by edges per launch",
                         "algorithmic_bytes_per_launch": fill_bytes},
            "phases_ms_per_step": phases,
            "phase_hbm": phase_hbm,
            "build_path": {0: "full sort", 1: "changed keys merged", 2: "bounds only"}[path],
            "phase_records": phase_calls,
            "dominant_phase": dominant,
            "gpu_launches": int(launches),
            "tuning": tuning,
            "clocks": clk,
            "cpu_baseline": cpu,
            "other_configs": sec,
        }
    return result


# ------------------------------------------------- other configurations -----
def _timed(torch, stream, fn, reps):
    """Device time (ms) of `reps` calls of fn, CUDA events on the stream."""
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    acc = 0
    for _ in range(reps):
        acc += fn()
    t1.record(stream)
    torch.cuda.synchronize()
    return t0.elapsed_time(t1), acc


def secondary_configs(ob, torch, dev):
    """The other configurations of the path, each at its full size:
    uniform 100k (r = 0.04), nonuniform 2D 4M (r = 0.002), 512 batched clouds
    against a per-cloud loop of the same kernels, and the differentiable 2M
    configuration with its FP64 central-difference gradient check."""
    wl = _workloads()
    stream = torch.cuda.current_stream(dev)
    out = {}

    def plain(name, x, r, reps):
        tns = ob.TNS(torch.float32, ndims=x.shape[1])
        ob.set_search_radius_(tns, r)
        xd = torch.from_numpy(x).to(dev).t()
        sid = ob.add_point_set_(tns, xd)
        ob.set_active_search_(tns, sid, sid)

        def step():
            ob.update_point_set_(tns, sid, xd)
            ob.run_(tns)
            return ob.build_edges(tns, sid, sid).senders.numel()

        step()
        step()  # the second build sizes the library's scratch (hit records) for this workload
        ms, edges = _timed(torch, stream, step, reps)
        out[name] = {"n_points": int(x.shape[0]), "radius": r, "edges_per_step": edges // reps,
                     "ms_per_step": ms / reps, "edges_per_s": edges / (ms / 1e3)}
        del tns, xd
        torch.cuda.empty_cache()

    plain("uniform_100k_r0.04", wl.uniform(100_000, 3, 2024), 0.04, 10)
    plain("nonuniform2d_4M_r0.002_seed2026", wl.gaussian_mixture_2d(4_000_000, 64, 2026), 0.002, 2)

    # --- the build alone (run!) at 16M uniform points, where its kernels move
    # enough bytes to be bandwidth-bound rather than launch-bound
    def build_only(name, x, r, reps):
        lib = ob._lib.load()
        tns = ob.TNS(torch.float32, ndims=3)
        ob.set_search_radius_(tns, r)
        xd = torch.from_numpy(x).to(dev).t()
        sid = ob.add_point_set_(tns, xd)
        ob.set_active_search_(tns, sid, sid)

        def step():
            ob.update_point_set_(tns, sid, xd)
            ob.run_(tns)
            return 0

        step()
        step()
        ms, _ = _timed(torch, stream, step, reps)
        nph = len(ob._lib.PHASES)
        ms_buf = (C.c_double * nph)()
        cnt_buf = (C.c_int64 * nph)()
        ctx = tns._ctx
        lib.oct_profile_read(ctx.handle, ms_buf, cnt_buf, nph)
        lib.oct_profile_enable(ctx.handle, 1)
        for _ in range(reps):
            step()
        torch.cuda.synchronize()
        lib.oct_profile_read(ctx.handle, ms_buf, cnt_buf, nph)
        lib.oct_profile_enable(ctx.handle, 0)
        phases = {ob._lib.PHASES[i]: ms_buf[i] / reps for i in range(nph) if cnt_buf[i]}
        n = x.shape[0]
        # 8-bit radix passes over keys of 3 x (bits of the largest cell index), cell size r
        passes = (3 * int(math.floor(1.0 / r)).bit_length() + 7) // 8
        peak = _peak_gbs()
        hbm = {k: {"bytes": v, "gbs": v / (phases[k] / 1e3) / 1e9, "frac": v / (phases[k] / 1e3) / 1e9 / peak}
               for k, v in phase_bytes(n, 0, tns.trees[sid - 1].n_nodes, 0, passes).items() if phases.get(k)}
        out[name] = {"n_points": n, "radius": r, "ms_per_build": ms / reps, "radix_passes": passes,
                     "phases_ms": {k: round(v, 5) for k, v in phases.items()}, "phase_hbm": hbm}
        del tns, xd
        torch.cuda.empty_cache()

    build_only("build_only_uniform_16M_r0.006", wl.uniform(16_000_000, 3, 2031), 0.006, 5)

    # --- batched: 512 clouds, sizes log-uniform [500, 20000], r ~ U[0.03, 0.08]
    rng = np.random.default_rng(4)
    sizes = np.exp(rng.uniform(np.log(500), np.log(20000), 512)).astype(np.int64)
    radii = rng.uniform(0.03, 0.08, 512)
    clouds = [rng.random((int(n), 3)).astype(np.float32) for n in sizes]
    cat = torch.from_numpy(np.concatenate(clouds)).to(dev).t()
    bs = ob.BatchedSearch(torch.float32, 3)

    def batched():
        bs.run_(cat, sizes, radii)
        return bs.build_edges().senders.numel()

    batched()
    ms_b, e_b = _timed(torch, stream, batched, 5)
    tnss = []
    for x, r in zip(clouds, radii):
        t = ob.TNS(torch.float32)
        ob.set_search_radius_(t, float(r))
        xd = torch.from_numpy(x).to(dev).t()
        i = ob.add_point_set_(t, xd)
        ob.set_active_search_(t, i, i)
        tnss.append((t, i, xd))

    def loop():
        m = 0
        for t, i, xd in tnss:
            ob.update_point_set_(t, i, xd)
            ob.run_(t)
            m += ob.build_edges(t, i, i).senders.numel()
        return m

    loop()
    ms_l, e_l = _timed(torch, stream, loop, 1)
    out["batched_512_clouds"] = {
        "n_points": int(sizes.sum()), "edges": e_b // 5, "ms_batched": ms_b / 5, "ms_per_cloud_loop": ms_l,
        "edges_per_s_batched": e_b / (ms_b / 1e3), "edges_per_s_loop": e_l / (ms_l / 1e3),
        "speedup_vs_loop": (ms_l) / (ms_b / 5), "same_edge_count": e_l == e_b // 5}
    del tnss, bs, cat
    torch.cuda.empty_cache()

    # --- differentiable: 2M uniform, r = 0.012, fwd + adjoint, FP64 FD check
    x = wl.uniform(2_000_000, 3, 2025)
    r = 0.012
    tns = ob.TNS(torch.float32)
    ob.set_search_radius_(tns, r)
    xd = torch.from_numpy(x).to(dev).t()
    sid = ob.add_point_set_(tns, xd)
    ob.set_active_search_(tns, sid, sid)
    state = {}

    def fwd_bwd():
        state.clear()  # the previous step's COO and gradient go back to the allocator first
        c = xd.detach().clone().requires_grad_(True)
        ob.update_point_set_(tns, sid, c.detach())
        ob.run_(tns)
        e = ob.build_edges_diff(c, tns, sid, r)
        loss = (e.rel_displacement ** 2).sum() + 0.5 * (e.rel_dist_norm ** 2).sum()
        loss.backward()
        state["grad"], state["e"] = c.grad, e
        return e.senders.numel()

    fwd_bwd()
    fwd_bwd()
    ms_d, e_d = _timed(torch, stream, fwd_bwd, 3)
    g = state["grad"].t().cpu().numpy().astype(np.float64)
    e = state["e"]
    rcv = e.receivers.cpu().numpy()
    snd = e.senders.cpu().numpy()
    rf = float(np.float32(r))
    x64 = x.astype(np.float64)
    pick = np.random.default_rng(0).choice(x.size, 1000, replace=False)
    lo = np.searchsorted(rcv, np.arange(1, x.shape[0] + 1), "left")
    hi = np.searchsorted(rcv, np.arange(1, x.shape[0] + 1), "right")
    errs, fds = [], []
    h = 1e-4
    for k in pick:
        p, d = divmod(int(k), 3)
        nb = snd[lo[p]:hi[p]] - 1  # frozen neighbor set; each pair is two directed edges

        def f(delta):
            xp = x64[p].copy()
            xp[d] += delta
            dd = (xp[None, :] - x64[nb]) / rf
            return 2 * 1.5 * (dd * dd).sum()

        fd = (-f(2 * h) + 8 * f(h) - 8 * f(-h) + f(-2 * h)) / (12 * h)
        errs.append(abs(g[p, d] - fd))
        fds.append(abs(fd))
    errs, fds = np.array(errs), np.array(fds)
    out["diff_2M_r0.012"] = {
        "n_points": int(x.shape[0]), "edges": e_d // 3, "ms_fwd_bwd": ms_d / 3,
        "edges_per_s_fwd_bwd": e_d / (ms_d / 1e3),
        "grad_max_abs_err_over_max_abs_fd": float(errs.max() / fds.max()),
        "grad_median_rel_err": float(np.median(errs / np.maximum(fds, 1e-30))),
        "fd": "4-point central differences in FP64, h = 1e-4, frozen edge set, 1000 random coordinates"}
    del tns, xd, state
    torch.cuda.empty_cache()
    return out


def cpu_baseline(args, budget_s=None):
    """The oracle (C++ restatement of the reference CPU path) on the host's
    cores, on full-size time steps, stopping after ~10 s of work."""
    import oracle
    budget_s = budget_s if budget_s is not None else args.cpu_budget
    nthreads = oracle.max_threads()
    snaps = snapshots_np(PER, 40, 999)  # more steps than the budget takes
    edges, secs, steps = 0, 0.0, 0
    for x in snaps[1:]:
        t0 = time.perf_counter()
        t = oracle.build_tree(x, np.float32(RADIUS), nthreads=nthreads)
        e = oracle.build_edges(t, x, exclude_self=True, nthreads=nthreads)
        secs += time.perf_counter() - t0
        edges += len(e["senders"])
        steps += 1
        if secs >= budget_s:
            break
    out = {"value": edges / secs, "unit": "edges/s", "cores": nthreads, "kind": "port",
           "sample": f"{steps} full 1M-point time steps (build + count + scan + fill), "
                     f"{secs:.1f} s of CPU work"}
    out["other_configs"] = cpu_other_configs(oracle, nthreads)
    return out


def cpu_other_configs(oracle, nthreads):
    """The CPU port on the other configurations, one full run each (the
    nonuniform 2D case is left out: its 1.5 G-edge COO needs ~37 GB of host
    memory)."""
    wl = _workloads()
    res = {}

    def timed(fn):
        t0 = time.perf_counter()
        e = fn()
        return e, time.perf_counter() - t0

    x = wl.uniform(100_000, 3, 2024)
    e, t = timed(lambda: len(oracle.build_edges(oracle.build_tree(x, np.float32(0.04), nthreads=nthreads), x,
                                                exclude_self=True, nthreads=nthreads)["senders"]))
    res["uniform_100k_r0.04"] = {"edges": e, "s": t, "edges_per_s": e / t}
    rng = np.random.default_rng(4)
    sizes = np.exp(rng.uniform(np.log(500), np.log(20000), 512)).astype(np.int64)
    radii = rng.uniform(0.03, 0.08, 512)
    clouds = [rng.random((int(n), 3)).astype(np.float32) for n in sizes]

    def per_cloud():
        m = 0
        for c, r in zip(clouds, radii):
            rr = np.float32(r)
            m += len(oracle.build_edges(oracle.build_tree(c, rr, nthreads=nthreads), c, exclude_self=True,
                                        nthreads=nthreads)["senders"])
        return m

    e, t = timed(per_cloud)
    res["batched_512_clouds_per_cloud_loop"] = {"edges": e, "s": t, "edges_per_s": e / t}
    x = wl.uniform(2_000_000, 3, 2025)

    def diff():
        tr = oracle.build_tree(x, np.float32(0.012), nthreads=nthreads)
        oe = oracle.build_edges(tr, x, exclude_self=True, nthreads=nthreads)
        rd, rn = oe["rel_displacement"], oe["rel_dist_norm"]
        oracle.diff_backward(len(x), oe["senders"], oe["receivers"], rd, rn, 2 * rd, rn, np.float32(0.012))
        return len(oe["senders"])

    e, t = timed(diff)
    res["diff_2M_r0.012_fwd_bwd"] = {"edges": e, "s": t, "edges_per_s": e / t}
    return res


# ------------------------------------------------------ reference arm -----
def run_reference(args, rank, world):
    """The reference's CPU path (the oracle port: the Julia original cannot
    run here) on all host threads, on the same workload as our arm: the same
    1,000,000-point lattice trajectory (same seed), W warm-up steps and K
    timed steps, each step a full build + count + scan + fill."""
    if rank != 0:
        return None
    import oracle
    nthreads = oracle.max_threads()
    snaps = snapshots_np(PER, args.warmup + args.steps, 12345)
    r = np.float32(RADIUS)
    for x in snaps[:args.warmup]:
        oracle.build_edges(oracle.build_tree(x, r, nthreads=nthreads), x, exclude_self=True, nthreads=nthreads)
    edges, secs = 0, 0.0
    for x in snaps[args.warmup:]:
        t0 = time.perf_counter()
        t = oracle.build_tree(x, r, nthreads=nthreads)
        e = oracle.build_edges(t, x, exclude_self=True, nthreads=nthreads)
        secs += time.perf_counter() - t0
        edges += len(e["senders"])
    v = edges / secs
    sample = (f"{args.steps} time steps of the {PER}^3-point lattice trajectory (the timed steps of our arm, "
              f"same seed), each a full build + count + scan + fill")
    return {
        "impl": "reference",
        "metric": METRIC, "value": v, "unit": "edges/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded jittered lattice + Gaussian steps)",
        "config": config_dict({"edges_per_step": edges / args.steps, "parallelism": "host threads",
                               "reference_sample": sample}),
        "cpu_baseline": {"value": v, "unit": "edges/s", "cores": nthreads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--fill-traffic", type=float, default=None,
                    help="dram bytes per fill launch from an ncu capture (reported as roofline.traffic)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res))
        return
    rank, world, local = dist_setup(args.gpus)
    try:
        res = run_ours(args, rank, world, local)
        if res is not None:
            print(json.dumps(res))
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
