"""Autotuner of the kernel shapes (leaf chunks per traversal step, internal
nodes expanded together, fill staging depth, query points per traversal
group, sub-boxes of a group for the target test, L1 prefetch in the
traversal).

    python octopus.jl_b200/tune.py [--out PATH] [--steps K] [--rounds R]

For each benchmark configuration it measures the time of a whole step
(run! + build_edges, CUDA events on the stream) for each value of one shape
while the others are held, keeps the fastest (coordinate descent, R rounds),
and writes one row per configuration to the table (default
``octopus.jl_b200/tuning.tsv``):

    ndims dtype nlog2 nbr_log2 max_seg multi_pop fill_chunk group_cap sub_boxes prefetch

keyed by the configuration's point count (log2) and neighbors per point
(log2 of 1 + the average), the key the library uses to pick a row
(oct_ctx_load_tuning).  No shape changes any result, only the time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import math
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(HERE, "tuning.tsv")

# option id and candidate values of each shape, in the order they are tuned
SHAPES = [
    ("group_cap", 9, (16, 24, 32)),
    ("max_seg", 6, (1, 4, 8, 16)),
    ("multi_pop", 7, (1, 2, 4)),
    ("fill_chunk", 8, (0, 32, 64, 128)),
    ("sub_boxes", 10, (1, 2, 4)),
    ("prefetch", 11, (0, 1)),
]
DEFAULTS = {"group_cap": 32, "max_seg": 16, "multi_pop": 4, "fill_chunk": 0, "sub_boxes": 1, "prefetch": 0}


def _package():
    sys.path.insert(0, os.path.dirname(HERE))
    import __graft_entry__
    return __graft_entry__.load_package()


def _workloads():
    import importlib.util
    spec = importlib.util.spec_from_file_location("octopus_b200_workloads", os.path.join(HERE, "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def configurations(wl):
    """(name, snapshots (N, D) float32, radius, refit mode) of the benchmark
    configurations (the batched clouds are tuned through their own forest)."""
    return [
        ("uniform_100k_r0.04", [wl.uniform(100_000, 3, 2024)], 0.04, False),
        ("sph_lattice_1M_r0.02", wl.sph_snapshots(100, 4, 12345), 0.02, True),
        ("nonuniform2d_4M_r0.002", [wl.gaussian_mixture_2d(4_000_000, 64, 2026)], 0.002, False),
        ("uniform_2M_r0.012", [wl.uniform(2_000_000, 3, 2025)], 0.012, False),
    ]


def key_of(ndims, n, edges):
    nlog2 = int(math.floor(math.log2(max(n, 1))))
    nbr_log2 = int(math.floor(math.log2(edges / max(n, 1) + 1.0)))
    return ndims, 0, nlog2, nbr_log2


class Runner:
    """One configuration on one TNS; time_step() is the device time of one
    run! + build_edges with the given shapes forced."""

    def __init__(self, ob, torch, xs, r, refit):
        self.ob, self.torch = ob, torch
        self.xs = [torch.from_numpy(x).cuda().t() for x in xs]
        self.tns = ob.TNS(torch.float32, ndims=xs[0].shape[1])
        ob.set_search_radius_(self.tns, r)
        ob.set_refit_mode_(self.tns, refit)
        self.sid = ob.add_point_set_(self.tns, self.xs[0])
        ob.set_active_search_(self.tns, self.sid, self.sid)
        self.ctx = self.tns._ctx
        self.k = 0

    def force(self, shapes):
        for name, opt, _ in SHAPES:
            v = shapes.get(name)
            # 0 hands a shape back to the table; prefetch is forced as 1 (off) /
            # 2 (on), direct fill stores (fill_chunk 0) as 1
            if v is None:
                v = 0
            elif name == "prefetch":
                v = v + 1
            elif name == "fill_chunk" and v == 0:
                v = 1
            self.ctx.check(self.ctx.lib.oct_ctx_set_option(self.ctx.handle, opt, int(v)), name)

    def step(self):
        x = self.xs[self.k % len(self.xs)]
        self.k += 1
        self.ob.update_point_set_(self.tns, self.sid, x)
        self.ob.run_(self.tns)
        return self.ob.build_edges(self.tns, self.sid, self.sid).senders.numel()

    def time_step(self, shapes, steps):
        torch = self.torch
        self.force(shapes)
        for _ in range(2):  # the first applies a new group size to the tree, the second warms up
            self.step()
        s = torch.cuda.current_stream()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0.record(s)
        for _ in range(steps):
            edges = self.step()
        t1.record(s)
        torch.cuda.synchronize()
        return t0.elapsed_time(t1) / steps, edges


def tune(steps=10, rounds=2, out=DEFAULT_TABLE, names=None, log=print):
    import torch
    ob = _package()
    wl = _workloads()
    rows = []
    for name, xs, r, refit in configurations(wl):
        if names and name not in names:
            continue
        run = Runner(ob, torch, xs, r, refit)
        best = dict(DEFAULTS)
        best_ms, edges = run.time_step(best, steps)
        base_ms = best_ms
        for _ in range(rounds):
            for sname, _, values in SHAPES:
                for v in values:
                    if v == best[sname]:
                        continue
                    trial = dict(best, **{sname: v})
                    ms, _ = run.time_step(trial, steps)
                    log(f"{name}: {trial} {ms:.4f} ms")
                    if ms < best_ms * 0.995:  # a change must beat the noise
                        best, best_ms = trial, ms
        run.force({})
        key = key_of(xs[0].shape[1], xs[0].shape[0], edges)
        rows.append((key, best, name, base_ms, best_ms))
        log(f"{name}: key {key} best {best} {best_ms:.4f} ms (defaults {base_ms:.4f} ms)")
        del run
        torch.cuda.empty_cache()
    write_table(out, rows, torch.cuda.get_device_name())
    return rows


def write_table(path, rows, device):
    with open(path, "w") as f:
        f.write("# Kernel shapes per workload, measured by octopus.jl_b200/tune.py on " + device + " "
                + time.strftime("%Y-%m-%d") + "\n")
        f.write("# ndims dtype nlog2 nbr_log2 max_seg multi_pop fill_chunk group_cap sub_boxes prefetch"
                "   # configuration: step ms with these shapes / with the defaults\n")
        for (ndims, dtype, nlog2, nbr), s, name, base_ms, ms in rows:
            f.write(f"{ndims} {dtype} {nlog2} {nbr} {s['max_seg']} {s['multi_pop']} {s['fill_chunk']} "
                    f"{s['group_cap']} {s['sub_boxes']} {s['prefetch']}   # {name}: {ms:.4f} / {base_ms:.4f} ms\n")


def select(path, ndims, dtype, n, nbrs_per_point):
    """The shapes and row the library would pick from the table at `path`."""
    ob = _package()
    lib = ob._lib.load()
    shapes = (C.c_int32 * 6)()
    row = C.c_int32(-2)
    st = lib.oct_tuning_select((path or "").encode(), ndims, dtype, n, float(nbrs_per_point), shapes, C.byref(row))
    if st != 0:
        raise ValueError(f"tuning table {path} could not be read")
    return dict(zip(("max_seg", "multi_pop", "fill_chunk", "group_cap", "sub_boxes", "prefetch"), list(shapes))), int(row.value)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--rounds", type=int, default=2)
    ap.add_argument("--only", nargs="*", default=None, help="configuration names to tune")
    a = ap.parse_args()
    tune(a.steps, a.rounds, a.out, a.only)
