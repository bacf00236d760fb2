"""Host-side mirror of Octopus.jl's public API (src/api.jl, src/types.jl).

Names follow the reference with Julia's ``!`` spelled as a trailing ``_``
(``run!`` -> ``run_``).  Arrays keep the reference's memory layout: a
``(NDIMS, N)`` coordinate matrix is a torch tensor of that shape whose memory
is column-major (``x.stride() == (1, NDIMS)``, i.e. ``xyz xyz ...``), and all
indices are 1-based ``int32``.  Every computation runs in
``liboctopus_b200.so`` on the GPU; there is no CPU fallback.

Exceptions mirror the reference's: :class:`ArgumentError`,
:class:`DimensionMismatch`, :class:`InexactError`, :class:`OctopusError`
(Julia's ``ErrorException``), ``AssertionError`` and ``TypeError``
(Julia's ``MethodError``).
"""
from __future__ import annotations

import ctypes as C
import os
from collections import namedtuple
from typing import Callable

import numpy as np
import torch

from . import _lib


TUNING_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.tsv")


# ----------------------------------------------------------------- errors --
class ArgumentError(ValueError):
    """Julia ``ArgumentError``."""


class DimensionMismatch(ValueError):
    """Julia ``DimensionMismatch``."""


class InexactError(OverflowError):
    """Julia ``InexactError`` (``floor(Int32, x)`` out of range or NaN)."""


class OctopusError(RuntimeError):
    """Julia ``ErrorException`` raised by the reference (``error(...)``)."""


_STATUS_EXC = {
    _lib.ERR_ARGUMENT: ArgumentError,
    _lib.ERR_DIMENSION: DimensionMismatch,
    _lib.ERR_INEXACT: InexactError,
    _lib.ERR_STATE: OctopusError,
}


class _Context:
    """One ``oct_ctx`` per CUDA device, shared by every TNS on that device."""

    _by_device: dict = {}

    def __init__(self, device: int):
        self.lib = _lib.load()
        h = C.c_void_p()
        st = self.lib.oct_ctx_create(device, C.byref(h))
        if st != _lib.OK:
            raise RuntimeError(f"oct_ctx_create({device}) failed: status {st}")
        self.handle = h
        self.device = device
        # Kernel shapes measured by tune.py: the packaged table unless
        # OCTOPUS_B200_TUNING names another (or is empty: built-in defaults).
        table = os.environ.get("OCTOPUS_B200_TUNING", TUNING_TABLE)
        if table and os.path.exists(table):
            self.check(self.lib.oct_ctx_load_tuning(self.handle, table.encode()), "oct_ctx_load_tuning")

    @classmethod
    def get(cls, device: int) -> "_Context":
        ctx = cls._by_device.get(device)
        if ctx is None:
            ctx = cls(device)
            cls._by_device[device] = ctx
        return ctx

    def bind_stream(self):
        s = torch.cuda.current_stream(self.device).cuda_stream
        self.lib.oct_ctx_set_stream(self.handle, C.c_void_p(s))

    def check(self, st: int, what: str):
        if st == _lib.OK:
            return
        msg = self.lib.oct_ctx_last_error(self.handle).decode(errors="replace")
        exc = _STATUS_EXC.get(st, RuntimeError)
        raise exc(f"{what}: {msg or self.lib.oct_status_string(st).decode()}")


# ---------------------------------------------------------------- helpers --
def _dtype_code(T) -> int:
    if T == torch.float32:
        return 0
    if T == torch.float64:
        return 1
    raise TypeError(f"TNS element type must be torch.float32 or torch.float64, got {T}")


def colmajor(x: torch.Tensor) -> torch.Tensor:
    """Return ``x`` (shape ``(NDIMS, N)``) with column-major memory, the
    layout of a Julia matrix; no copy when it already has it."""
    if x.dim() != 2:
        raise DimensionMismatch("coords must be a 2-D (NDIMS, N) tensor")
    d, n = x.shape
    if n <= 1 or (x.stride(0) == 1 and x.stride(1) == d):
        return x
    return x.t().contiguous().t()


def _ptr(x: torch.Tensor | None):
    return C.c_void_p(x.data_ptr()) if x is not None and x.numel() > 0 else C.c_void_p(0)


class _DevArray:
    """Zero-copy wrapper exposing library-owned device memory to torch."""

    def __init__(self, ptr: int, shape, typestr: str, owner):
        self.__cuda_array_interface__ = {
            "shape": tuple(int(s) for s in shape), "typestr": typestr,
            "data": (int(ptr or 0), False), "version": 3, "strides": None,
        }
        self._owner = owner


def _wrap(ptr, shape, dtype: torch.dtype, device: int, owner) -> torch.Tensor:
    if int(np.prod(shape)) == 0 or not ptr:
        return torch.empty(shape, dtype=dtype, device=f"cuda:{device}")
    typestr = {torch.int32: "<i4", torch.float32: "<f4", torch.float64: "<f8", torch.int64: "<i8"}[dtype]
    return torch.as_tensor(_DevArray(ptr, shape, typestr, owner), device=f"cuda:{device}")


# ----------------------------------------------------------------- types ---
class PointSet:
    """src/types.jl:12-20: coordinates held by reference, ``n`` points."""

    def __init__(self, coords: torch.Tensor):
        self.coords = coords
        self.n = int(coords.shape[1])


class Octree:
    """A library-owned tree (src/types.jl:23-42).  Its arrays are exposed by
    :func:`device_view` and :meth:`arrays`."""

    def __init__(self, ctx: _Context, ndims: int, dtype_code: int):
        self._ctx = ctx
        h = C.c_void_p()
        ctx.check(ctx.lib.oct_tree_create(ctx.handle, ndims, dtype_code, C.byref(h)), "oct_tree_create")
        self.handle = h
        self.ndims = ndims
        self.dtype_code = dtype_code
        self.built = False
        self.n_nodes = 0

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._ctx.lib.oct_tree_destroy(h)
            except Exception:
                pass
            self.handle = None

    def last_build(self) -> tuple[int, int]:
        """How the last run! ordered the points: (path, n_changed) with path
        0 = full sort, 1 = changed keys merged into the previous order,
        2 = no key changed (bounds only); n_changed = -1 when the previous
        order was not reusable (refit mode off, first build, new size or
        radius)."""
        path, moved = C.c_int(), C.c_int64()
        self._ctx.check(self._ctx.lib.oct_tree_last_build(self.handle, C.byref(path), C.byref(moved)),
                        "last_build")
        return int(path.value), int(moved.value)

    def view(self) -> _lib.TreeView:
        v = _lib.TreeView()
        self._ctx.bind_stream()
        self._ctx.check(self._ctx.lib.oct_tree_view_get(self._ctx.handle, self.handle, C.byref(v)),
                        "device_view")
        return v

    def arrays(self) -> dict:
        """The tree in the reference's layout, as torch tensors aliasing the
        library's memory (valid until the next build of this tree)."""
        v = self.view()
        dev = self._ctx.device
        nch = 1 << self.ndims
        T = torch.float32 if self.dtype_code == 0 else torch.float64
        nn, n = int(v.n_nodes), int(v.n_points)
        out = {
            "n_nodes": nn,
            "node_first": _wrap(v.node_first, (nn,), torch.int32, dev, self),
            "node_last": _wrap(v.node_last, (nn,), torch.int32, dev, self),
            # (NCH, n_nodes) column-major == (n_nodes, NCH) row-major, transposed view
            "node_children": _wrap(v.node_children, (nn, nch), torch.int32, dev, self).t(),
            "node_bounds_min": _wrap(v.bounds_min, (nn, self.ndims), T, dev, self).t(),
            "node_bounds_max": _wrap(v.bounds_max, (nn, self.ndims), T, dev, self).t(),
            "perm": _wrap(v.perm, (n,), torch.int32, dev, self),
        }
        if v.morton:
            out["morton"] = _wrap(v.morton, (n,), torch.int64, dev, self)
        return out


class EdgeBuffer:
    """src/types.jl:84-100: flat COO of one active pair."""

    def __init__(self, T: torch.dtype, ndims: int, device: int):
        dev = f"cuda:{device}"
        self.senders = torch.empty(0, dtype=torch.int32, device=dev)
        self.receivers = torch.empty(0, dtype=torch.int32, device=dev)
        self.rel_displacement = torch.empty((0, ndims), dtype=T, device=dev).t()
        self.rel_dist_norm = torch.empty((0, 1), dtype=T, device=dev).t()
        self.n_edges = 0
        self.materialized = False


class NeighborBuffer:
    """src/types.jl:44-54: CSR neighbor lists of one active pair: ``flat``
    (1-based target indices) and ``offsets`` (n_query + 1 Int32, starting at
    0); row i of query point i+1 is ``flat[offsets[i]:offsets[i+1]]``."""

    def __init__(self, device: int):
        dev = f"cuda:{device}"
        self.flat = torch.empty(0, dtype=torch.int32, device=dev)
        self.offsets = torch.zeros(1, dtype=torch.int32, device=dev)
        self.materialized = False


EdgesTuple = namedtuple("EdgesTuple", ["senders", "receivers", "rel_displacement", "rel_dist_norm"])
DeviceView = namedtuple("DeviceView", ["coords_q", "coords_t", "bounds_min", "bounds_max", "node_first",
                                       "node_last", "node_children", "perm", "n_nodes", "radius",
                                       "radius_sq"])


class TNS:
    """src/types.jl:132-183.  ``TNS(T=torch.float32, ndims=3)``."""

    def __init__(self, T: torch.dtype = torch.float32, ndims: int = 3):
        if ndims not in (2, 3):
            raise ArgumentError("ndims must be 2 or 3")
        _dtype_code(T)
        self.T = T
        self.ndims = ndims
        self.dev = "uninitialized"
        self.device = None
        self.radius = 0.0
        self.target_leaf_size = 32
        self.refit_mode = False
        self.point_sets: list[PointSet] = []
        self.active_pairs: list[tuple[int, int]] = []
        self.trees: list[Octree] = []
        self.edge_buffers: list[EdgeBuffer] = []
        self.neighbor_buffers: list[NeighborBuffer] = []
        self.dirty: list[bool] = []
        self._ctx: _Context | None = None

    # convenience accessors mirroring tns.permutation / tns.morton_codes
    @property
    def permutation(self):
        return [t.arrays()["perm"] if t.built else torch.empty(0, dtype=torch.int32) for t in self.trees]

    @property
    def morton_codes(self):
        out = []
        for t in self.trees:
            a = t.arrays() if t.built else {}
            out.append(a.get("morton", torch.empty(0, dtype=torch.int64)))
        return out


def _mark_all_dirty(tns: TNS):
    for i in range(len(tns.dirty)):
        tns.dirty[i] = True


def set_search_radius_(tns: TNS, r) -> TNS:
    """src/api.jl:24-29."""
    if not (r > 0):
        raise ArgumentError("search radius must be positive")
    tns.radius = float(torch.tensor(float(r), dtype=tns.T).item())
    _mark_all_dirty(tns)
    return tns


def set_refit_mode_(tns: TNS, on: bool) -> TNS:
    """src/api.jl:43-47."""
    tns.refit_mode = bool(on)
    _mark_all_dirty(tns)
    return tns


def _check_coords(tns: TNS, coords: torch.Tensor) -> torch.Tensor:
    if not isinstance(coords, torch.Tensor) or coords.dim() != 2 or coords.shape[0] != tns.ndims:
        raise DimensionMismatch(f"coords must be ({tns.ndims}, N)")
    if coords.dtype != tns.T:
        raise TypeError(f"coords element type {coords.dtype} does not match TNS element type {tns.T}")
    return coords


def _infer_dev(tns: TNS, coords: torch.Tensor):
    """src/api.jl:58-72.  Only CUDA tensors are accepted: this package is the
    GPU backend and has no CPU path."""
    new_dev = "cuda" if coords.is_cuda else "cpu"
    if new_dev != "cuda":
        raise ArgumentError("coords must be a CUDA tensor: this backend runs on the GPU only")
    if tns.dev == "uninitialized":
        tns.dev = new_dev
        tns.device = coords.device.index if coords.device.index is not None else torch.cuda.current_device()
        tns._ctx = _Context.get(tns.device)
    elif tns.dev != new_dev or coords.device.index not in (None, tns.device):
        raise ArgumentError(f"TNS was initialized on :{tns.dev} (device {tns.device}) but got coords on "
                            f"{coords.device}; all point sets must share a backend")


def add_point_set_(tns: TNS, coords: torch.Tensor) -> int:
    """src/api.jl:96-106.  Returns the 1-based set id."""
    coords = _check_coords(tns, coords)
    _infer_dev(tns, coords)
    tns.point_sets.append(PointSet(colmajor(coords)))
    tns.trees.append(Octree(tns._ctx, tns.ndims, _dtype_code(tns.T)))
    tns.dirty.append(True)
    return len(tns.point_sets)


def resize_point_set_(tns: TNS, set_id: int, coords: torch.Tensor) -> TNS:
    """src/api.jl:119-124."""
    coords = _check_coords(tns, coords)
    _infer_dev(tns, coords)
    tns.point_sets[set_id - 1] = PointSet(colmajor(coords))
    tns.dirty[set_id - 1] = True
    return tns


def update_point_set_(tns: TNS, set_id: int, coords: torch.Tensor) -> TNS:
    """src/api.jl:134-142."""
    coords = _check_coords(tns, coords)
    ps = tns.point_sets[set_id - 1]
    if coords.shape[1] != ps.n:
        raise DimensionMismatch("update_point_set! expects same size; use resize_point_set! otherwise")
    _infer_dev(tns, coords)
    tns.point_sets[set_id - 1] = PointSet(colmajor(coords))
    tns.dirty[set_id - 1] = True
    return tns


def set_active_search_(tns: TNS, q: int, t: int) -> TNS:
    """src/api.jl:156-165 (idempotent)."""
    pair = (int(q), int(t))
    if pair in tns.active_pairs:
        return tns
    tns.active_pairs.append(pair)
    dev = tns.device if tns.device is not None else 0
    tns.edge_buffers.append(EdgeBuffer(tns.T, tns.ndims, dev))
    tns.neighbor_buffers.append(NeighborBuffer(dev))
    return tns


def _build_set(tns: TNS, sid: int):
    ps = tns.point_sets[sid]
    tree = tns.trees[sid]
    ctx = tns._ctx
    ctx.bind_stream()
    st = ctx.lib.oct_tree_build(ctx.handle, tree.handle, _ptr(ps.coords), ps.n, tns.radius,
                                1 if tns.refit_mode else 0)
    ctx.check(st, "run!")
    nn = C.c_int64()
    ctx.lib.oct_tree_n_nodes(ctx.handle, tree.handle, C.byref(nn))
    tree.n_nodes = int(nn.value)
    tree.built = True
    tree.coords_ref = ps.coords


def run_(tns: TNS) -> TNS:
    """src/api.jl:183-250: build every dirty point set."""
    if not (tns.radius > 0):
        raise ArgumentError("set_search_radius! before run!")
    if tns.dev == "uninitialized":
        raise ArgumentError("add at least one point set before run!")
    for sid in range(len(tns.point_sets)):
        if not tns.dirty[sid]:
            continue
        _build_set(tns, sid)
        tns.dirty[sid] = False
    for buf in tns.edge_buffers:
        buf.materialized = False
    for buf in tns.neighbor_buffers:
        buf.materialized = False
    return tns


def _pair_index(tns: TNS, q: int, t: int) -> int:
    try:
        return tns.active_pairs.index((int(q), int(t)))
    except ValueError:
        raise OctopusError(f"build_edges!: pair ({q}, {t}) not registered; call set_active_search! first") from None


def _reserve_buffer(buf: EdgeBuffer, T, ndims, n_edges, device):
    """Grow-only backing storage of the buffer's arrays (1.25x slack), so a
    time-stepping loop whose edge count fluctuates does not reallocate every
    step."""
    cap = getattr(buf, "_capacity", -1)
    if n_edges > cap:
        dev = f"cuda:{device}"
        cap = n_edges + n_edges // 4
        buf._capacity = cap
        buf._snd = torch.empty(cap, dtype=torch.int32, device=dev)
        buf._rcv = torch.empty(cap, dtype=torch.int32, device=dev)
        buf._disp = torch.empty((cap, ndims), dtype=T, device=dev)
        buf._dist = torch.empty((cap, 1), dtype=T, device=dev)


def _resize_buffer(buf: EdgeBuffer, T, ndims, n_edges, device):
    """Size the buffer's arrays to n_edges: views of the grow-only backing
    storage; like the reference, the arrays are replaced whenever the edge
    count changes."""
    _reserve_buffer(buf, T, ndims, n_edges, device)
    if buf.senders.numel() != n_edges or buf.senders.data_ptr() != buf._snd.data_ptr():
        buf.senders = buf._snd[:n_edges]
        buf.receivers = buf._rcv[:n_edges]
        buf.rel_displacement = buf._disp[:n_edges].t()
        buf.rel_dist_norm = buf._dist[:n_edges].t()
    buf.n_edges = n_edges


def _count_pair(tns: TNS, qid: int, tid: int, what: str):
    """Pass A for the pair (qid, tid): returns (ctx, qtree, ttree, exclude_self,
    n_edges), or None when the pair has no edges by construction (an empty
    query set, or a target never built: ext/OctopusCUDAExt.jl:353-367,
    test/backend_errors_cpu.jl:40-57)."""
    if tns.dev != "cuda":
        raise OctopusError(f"{what}: TNS not initialized; add a point set first")
    qs = tns.point_sets[qid - 1]
    qtree, ttree = tns.trees[qid - 1], tns.trees[tid - 1]
    if qs.n == 0 or not ttree.built or ttree.n_nodes == 0:
        return None
    if not qtree.built:
        # The query set was added after the last run!; its Morton order is
        # needed to group the queries, so build it now.
        _build_set(tns, qid - 1)
    ctx = tns._ctx
    ctx.bind_stream()
    excl = 1 if qid == tid else 0
    ne = C.c_int64()
    ctx.check(ctx.lib.oct_edges_count(ctx.handle, qtree.handle, ttree.handle, excl, C.byref(ne)), what)
    return ctx, qtree, ttree, excl, int(ne.value)


def build_edges_(tns: TNS, qid: int, tid: int) -> EdgeBuffer:
    """src/api.jl:304-320 with the CUDA path of ext/OctopusCUDAExt.jl:345-415."""
    pidx = _pair_index(tns, qid, tid)
    buf = tns.edge_buffers[pidx]
    got = _count_pair(tns, qid, tid, "build_edges!")
    if got is None:
        _resize_buffer(buf, tns.T, tns.ndims, 0, tns.device)
        buf.materialized = True
        return buf
    ctx, qtree, ttree, excl, n_edges = got
    if n_edges > 2**31 - 1:
        raise OctopusError(f"build_edges!: {n_edges} edges exceed the Int32 edge count of EdgeBuffer")
    # The fill goes into the backing storage first (its arrays start there, and
    # _disp is (capacity, D) row-major = the (D, E) column-major matrix), so the
    # device is busy while the host makes the sized views.
    _reserve_buffer(buf, tns.T, tns.ndims, n_edges, tns.device)
    if n_edges > 0:
        ctx.check(ctx.lib.oct_edges_fill(ctx.handle, qtree.handle, ttree.handle, excl, _ptr(buf._snd),
                                         _ptr(buf._rcv), _ptr(buf._disp), _ptr(buf._dist), n_edges),
                  "build_edges!")
    _resize_buffer(buf, tns.T, tns.ndims, n_edges, tns.device)
    buf.materialized = True
    return buf


def synchronize(tns: TNS) -> None:
    """Wait for the TNS's device work; raises if a kernel's bounds guard fired."""
    if tns._ctx is not None:
        tns._ctx.check(tns._ctx.lib.oct_synchronize(tns._ctx.handle), "synchronize")


def build_edges(tns: TNS, qid: int, tid: int) -> EdgesTuple:
    """src/api.jl:329-337: the buffer's arrays as a named tuple (aliased)."""
    buf = build_edges_(tns, qid, tid)
    return EdgesTuple(buf.senders, buf.receivers, buf.rel_displacement, buf.rel_dist_norm)


def _neighbors(tns: TNS, qid: int, tid: int, idx: list[int]) -> list[np.ndarray]:
    ttree = tns.trees[tid - 1]
    qs = tns.point_sets[qid - 1]
    if not ttree.built or ttree.n_nodes == 0:
        return [np.zeros(0, np.int32) for _ in idx]
    sel = torch.as_tensor([i - 1 for i in idx], dtype=torch.int64, device=qs.coords.device)
    qc = qs.coords[:, sel].t().contiguous()  # (nsel, D) == (D, nsel) column-major
    ctx = tns._ctx
    ctx.bind_stream()
    nsel = len(idx)
    counts = torch.zeros(nsel, dtype=torch.int32, device=qc.device)
    cap = 64
    while True:
        out = torch.zeros((nsel, cap), dtype=torch.int32, device=qc.device)
        ctx.check(ctx.lib.oct_neighbors(ctx.handle, ttree.handle, _ptr(qc), nsel, _ptr(counts), _ptr(out), cap),
                  "for_each_neighbor")
        cmax = int(counts.max().item()) if nsel else 0
        if cmax <= cap:
            break
        cap = cmax
    c = counts.cpu().numpy()
    o = out.cpu().numpy()
    return [o[s, :c[s]].copy() for s in range(nsel)]


def for_each_neighbor(f: Callable[[int], None], tns: TNS, qid: int, tid: int, i: int) -> None:
    """src/cpu/iterator_cpu.jl:245-263: call ``f(j)`` for every target point
    within the radius of query point ``i``, in the reference's traversal
    order, without the self filter.  (The reference raises for a CUDA TNS;
    here the query runs on the GPU and ``f`` runs on the host.)"""
    for j in _neighbors(tns, qid, tid, [i])[0]:
        f(int(j))


def get_neighborlist(tns: TNS, qid: int, tid: int, i: int) -> np.ndarray:
    """src/api.jl:282-292: neighbor indices of point ``i``; self filtered
    when ``qid == tid``."""
    js = _neighbors(tns, qid, tid, [i])[0]
    if qid == tid:
        js = js[js != i]
    return js.astype(np.int32)


def materialize_all_neighbors_(tns: TNS) -> TNS:
    """src/api.jl:349-362 / materialize_cpu! (src/cpu/query_cpu.jl:149-192):
    CSR neighbor lists for every active pair, in each pair's NeighborBuffer.
    The reference wires this for a CPU TNS only; here it runs on the GPU:
    the same count pass as build_edges, then the senders column alone."""
    if tns.dev != "cuda":
        raise OctopusError("materialize_all_neighbors!: TNS not initialized; add a point set first")
    for pidx, (qid, tid) in enumerate(tns.active_pairs):
        buf = tns.neighbor_buffers[pidx]
        dev = f"cuda:{tns.device}"
        nq = tns.point_sets[qid - 1].n
        got = _count_pair(tns, qid, tid, "materialize_all_neighbors!")
        if got is None:
            buf.flat = torch.empty(0, dtype=torch.int32, device=dev)
            buf.offsets = torch.zeros(nq + 1, dtype=torch.int32, device=dev)
            buf.materialized = True
            continue
        ctx, qtree, ttree, excl, n = got
        if n > 2**31 - 1:
            raise OctopusError(f"materialize_all_neighbors!: {n} neighbors exceed the Int32 offsets")
        buf.flat = torch.empty(n, dtype=torch.int32, device=dev)
        buf.offsets = torch.empty(nq + 1, dtype=torch.int32, device=dev)
        ctx.check(ctx.lib.oct_csr_fill(ctx.handle, qtree.handle, ttree.handle, excl, _ptr(buf.offsets),
                                       _ptr(buf.flat), n), "materialize_all_neighbors!")
        buf.materialized = True
    return tns


def device_view(tns: TNS, qid: int, tid: int) -> DeviceView:
    """src/api.jl:451-454 / ext/OctopusCUDAExt.jl:37-56."""
    if tns.dev != "cuda":
        raise OctopusError("device_view requires a CUDA TNS")
    tree = tns.trees[tid - 1]
    if not tree.built:
        raise OctopusError("device_view: call run! first")
    a = tree.arrays()
    r = tns.radius
    r_t = torch.tensor(r, dtype=tns.T)
    return DeviceView(tns.point_sets[qid - 1].coords, tns.point_sets[tid - 1].coords, a["node_bounds_min"],
                      a["node_bounds_max"], a["node_first"], a["node_last"], a["node_children"], a["perm"],
                      a["n_nodes"], r, float((r_t * r_t).item()))


# --------------------------------------------------------- build_edges_diff --
class _EdgesDiff(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, tns, set_id, radius, recompute):
        # The primal writes fresh arrays (the reference copies build_edges'
        # buffer, ext/OctopusCUDAChainRulesCoreExt.jl:21-32).  The backward
        # pass finds each edge's mirror itself: searching the sender's
        # segment there costs less than writing mirror indices here.
        n_edges = 0
        _pair_index(tns, set_id, set_id)  # the pair must be registered, as for build_edges
        got = _count_pair(tns, set_id, set_id, "build_edges_diff")
        if got is not None:
            lc, qtree, ttree, excl, n_edges = got
            if n_edges > 2**31 - 1:
                raise OctopusError(f"build_edges_diff: {n_edges} edges exceed the Int32 edge count")
        dev = f"cuda:{tns.device}"
        snd = torch.empty(n_edges, dtype=torch.int32, device=dev)
        rcv = torch.empty(n_edges, dtype=torch.int32, device=dev)
        disp_rows = torch.empty((n_edges, tns.ndims), dtype=tns.T, device=dev)
        dist = torch.empty((1, n_edges), dtype=tns.T, device=dev)
        if n_edges > 0:
            lc.check(lc.lib.oct_edges_fill(lc.handle, qtree.handle, ttree.handle, excl, _ptr(snd), _ptr(rcv),
                                           _ptr(disp_rows), _ptr(dist), n_edges), "build_edges_diff")
        disp = disp_rows.t()  # (D, E) column-major
        ctx.tns = tns
        ctx.radius = float(radius)
        ctx.coords_shape = coords.shape
        ctx.recompute = bool(recompute)
        # The tree's Morton permutation (1-based, gathered from 1..n by the
        # tree's order): the backward pass visits the points in this order,
        # which keeps the mirror edges it reads in L2.
        n_pts = coords.shape[1]
        order = torch.arange(1, n_pts + 1, dtype=torch.int32, device=snd.device)
        if n_pts > 0:
            lc = tns._ctx
            lc.bind_stream()
            tree = tns.trees[set_id - 1]
            order_in, order = order, torch.empty_like(order)
            lc.check(lc.lib.oct_zsort_apply(lc.handle, tree.handle, _ptr(order_in), _ptr(order), n_pts, 4, 0),
                     "build_edges_diff order")
        if ctx.recompute:
            # Keep only the indices and the coordinates: the backward pass
            # recomputes the features (memory-lean mode).
            ctx.save_for_backward(snd, rcv, colmajor(coords.detach()), order)
        else:
            ctx.save_for_backward(snd, rcv, disp, dist, order)
        ctx.mark_non_differentiable(snd, rcv)
        return snd, rcv, disp, dist

    @staticmethod
    def backward(ctx, g_snd, g_rcv, g_disp, g_dist):
        tns = ctx.tns
        d, n = ctx.coords_shape
        T = tns.T
        dev = f"cuda:{tns.device}"
        grad = torch.empty((n, d), dtype=T, device=dev)
        dd = None if g_disp is None else g_disp.t().contiguous()
        dn = None if g_dist is None else g_dist.reshape(-1).contiguous()
        lc = tns._ctx
        lc.bind_stream()
        if ctx.recompute:
            snd, rcv, xc, order = ctx.saved_tensors
            disp_p, dist_p, xc_p = None, None, _ptr(xc)
        else:
            snd, rcv, disp, dist, order = ctx.saved_tensors
            disp_p, dist_p, xc_p = _ptr(disp.t()), _ptr(dist), None
        lc.check(lc.lib.oct_edges_diff_backward_ordered(
            lc.handle, d, _dtype_code(T), n, snd.numel(), _ptr(snd), _ptr(rcv), disp_p, dist_p, xc_p, _ptr(dd),
            _ptr(dn), ctx.radius, _ptr(grad), _ptr(order) if order.numel() == n else None),
            "build_edges_diff pullback")
        return grad.t(), None, None, None, None


def build_edges_diff(coords: torch.Tensor, tns: TNS, set_id: int, radius, recompute: bool = False) -> EdgesTuple:
    """ext/OctopusChainRulesCoreExt.jl:103-192: differentiable build_edges for
    a self pair; gradients flow to ``coords`` through a deterministic
    adjoint kernel.  ``recompute=True`` keeps no feature arrays for the
    backward pass and recomputes them from ``coords`` (identical values)."""
    return EdgesTuple(*_EdgesDiff.apply(coords, tns, set_id, radius, recompute))


class _EdgesDiffPair(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords_q, coords_t, tns, qid, tid, radius):
        e = build_edges(tns, qid, tid)
        snd, rcv = e.senders.clone(), e.receivers.clone()
        disp = e.rel_displacement.t().contiguous().t()
        dist = e.rel_dist_norm.t().contiguous().t()
        ctx.tns = tns
        ctx.radius = float(radius)
        ctx.shapes = (coords_q.shape, coords_t.shape)
        ctx.save_for_backward(snd, rcv, disp, dist)
        ctx.mark_non_differentiable(snd, rcv)
        return snd, rcv, disp, dist

    @staticmethod
    def backward(ctx, g_snd, g_rcv, g_disp, g_dist):
        tns = ctx.tns
        (d, nq), (_, nt) = ctx.shapes
        T = tns.T
        dev = f"cuda:{tns.device}"
        gq = torch.empty((nq, d), dtype=T, device=dev)
        gt = torch.empty((nt, d), dtype=T, device=dev)
        dd = None if g_disp is None else g_disp.t().contiguous()
        dn = None if g_dist is None else g_dist.reshape(-1).contiguous()
        snd, rcv, disp, dist = ctx.saved_tensors
        lc = tns._ctx
        lc.bind_stream()
        lc.check(lc.lib.oct_edges_diff_backward_pair(
            lc.handle, d, _dtype_code(T), nq, nt, snd.numel(), _ptr(snd), _ptr(rcv), _ptr(disp.t()), _ptr(dist),
            _ptr(dd), _ptr(dn), ctx.radius, _ptr(gq), _ptr(gt)), "build_edges_diff pullback")
        return gq.t(), gt.t(), None, None, None, None


def build_edges_diff_pair(coords_q: torch.Tensor, coords_t: torch.Tensor, tns: TNS, qid: int, tid: int,
                          radius) -> EdgesTuple:
    """Differentiable build_edges for a cross pair (qid != tid): gradients
    flow to both ``coords_q`` (receivers) and ``coords_t`` (senders).  The
    reference's rrule is self-pair only and names this extension
    (ext/OctopusChainRulesCoreExt.jl:134-135); the per-edge term is its
    rrule's (ext/OctopusChainRulesCoreExt.jl:150-189)."""
    if int(qid) == int(tid):
        raise ArgumentError("build_edges_diff_pair is for qid != tid; use build_edges_diff for a self pair")
    return EdgesTuple(*_EdgesDiffPair.apply(coords_q, coords_t, tns, int(qid), int(tid), radius))


# ----------------------------------------------------------- batched clouds --
BatchedEdges = namedtuple("BatchedEdges", ["senders", "receivers", "rel_displacement", "rel_dist_norm",
                                           "edge_offsets"])


def prepare_zsort(tns: TNS) -> TNS:
    """src/api.jl:380-386: checks that every point set's permutation is
    available (run! since its last change); mutates nothing."""
    for sid, ps in enumerate(tns.point_sets):
        tree = tns.trees[sid]
        if tns.dirty[sid] or not tree.built:
            raise OctopusError(f"prepare_zsort: call run! first so the permutation for set {sid + 1} is available")
    return tns


def _zsort_rows(tns: TNS, set_id: int, x: torch.Tensor, direction: int) -> torch.Tensor:
    """One oct_zsort_apply call on a 1-D (N,) or 2-D (F, N) tensor, returning
    a new tensor of the same shape (2-D results are column-major, like the
    coordinate matrices of this API)."""
    if x.dim() > 2:
        raise ArgumentError(f"apply_zsort supports 1-D or 2-D arrays only; got {x.dim()}-D")
    if not x.is_cuda:
        raise ArgumentError("apply_zsort: the array must be a CUDA tensor: this backend runs on the GPU only")
    n = tns.point_sets[set_id - 1].n
    if x.shape[-1] != n:
        raise DimensionMismatch(f"perm length {n} does not match last axis {x.shape[-1]}")
    if x.dim() == 1:
        xin = x.contiguous()
        out = torch.empty_like(xin)
        row = xin.element_size()
    else:
        xin = x.t().contiguous()  # (N, F): each point's F values contiguous
        out = torch.empty((x.shape[1], x.shape[0]), dtype=x.dtype, device=x.device).t()
        row = x.shape[0] * xin.element_size()
    if n == 0 or row == 0:
        return out
    ctx = tns._ctx
    ctx.bind_stream()
    ctx.check(ctx.lib.oct_zsort_apply(ctx.handle, tns.trees[set_id - 1].handle, _ptr(xin), _ptr(out), n, row,
                                      direction), "apply_zsort")
    return out


class _ZSort(torch.autograd.Function):
    """apply_zsort with the reference's rrule (ext/OctopusChainRulesCoreExt.jl:65-94):
    the pullback scatters the cotangent back, grad[:, perm] = dy."""

    @staticmethod
    def forward(ctx, x, tns, set_id):
        ctx.tns, ctx.set_id = tns, set_id
        ctx.shape = x.shape
        return _zsort_rows(tns, set_id, x, 0)

    @staticmethod
    def backward(ctx, dy):
        if dy is None:
            return None, None, None
        g = _zsort_rows(ctx.tns, ctx.set_id, dy, 1)
        return g, None, None


def apply_zsort(tns: TNS, set_id: int, user_array: torch.Tensor) -> torch.Tensor:
    """src/api.jl:388-409: a new array whose entries (1-D) or columns (2-D,
    (F, N)) follow point set ``set_id``'s z-order: out[:, i] =
    user_array[:, perm[i]].  ``user_array`` is read, never written.
    Differentiable (the rrule's scatter is the backward)."""
    if tns.dev != "cuda":
        raise OctopusError("apply_zsort: TNS not initialized; add a point set first")
    prepare_zsort(tns)
    return _ZSort.apply(user_array, tns, int(set_id))


def prepare_zsort_(tns: TNS) -> TNS:
    """Deprecated v0.1 spelling of :func:`prepare_zsort` (src/api.jl:411-412)."""
    import warnings
    warnings.warn("prepare_zsort! is deprecated, use prepare_zsort", DeprecationWarning, stacklevel=2)
    return prepare_zsort(tns)


def apply_zsort_(tns: TNS, set_id: int, user_array: torch.Tensor) -> torch.Tensor:
    """Deprecated v0.1 spelling of :func:`apply_zsort` (src/api.jl:411-412)."""
    import warnings
    warnings.warn("apply_zsort! is deprecated, use apply_zsort", DeprecationWarning, stacklevel=2)
    return apply_zsort(tns, set_id, user_array)


class BatchedSearch:
    """Many independent point clouds searched in one pass (no counterpart in
    the reference, which needs one TNS per radius, src/api.jl:24-29).

    ``run_(coords, sizes, radii)`` builds every cloud -- cloud ``c`` is the
    next ``sizes[c]`` columns of the ``(NDIMS, N)`` tensor ``coords`` with
    search radius ``radii[c]`` -- and ``build_edges()`` returns one
    concatenated COO (cloud by cloud, each exactly what ``build_edges`` of a
    TNS holding that cloud alone returns, with 1-based cloud-local indices)
    plus ``edge_offsets`` (numpy int64, ``n_clouds + 1``)."""

    def __init__(self, T: torch.dtype = torch.float32, ndims: int = 3, device: int | None = None):
        if ndims not in (2, 3):
            raise ArgumentError("ndims must be 2 or 3")
        self.T, self.ndims = T, ndims
        self.device = torch.cuda.current_device() if device is None else device
        self._ctx = _Context.get(self.device)
        self.tree = Octree(self._ctx, ndims, _dtype_code(T))
        self.n_clouds = 0
        self._buf = EdgeBuffer(T, ndims, self.device)

    def run_(self, coords: torch.Tensor, sizes, radii) -> "BatchedSearch":
        if coords.dim() != 2 or coords.shape[0] != self.ndims:
            raise DimensionMismatch(f"coords must be ({self.ndims}, N)")
        if coords.dtype != self.T:
            raise TypeError(f"coords element type {coords.dtype} does not match {self.T}")
        if not coords.is_cuda:
            raise ArgumentError("coords must be a CUDA tensor: this backend runs on the GPU only")
        sizes = np.asarray(sizes, dtype=np.int64)
        radii = np.ascontiguousarray(np.asarray(radii, dtype=np.float64))
        if len(sizes) != len(radii) or len(sizes) == 0:
            raise DimensionMismatch("sizes and radii need one entry per cloud")
        # radii in the element type, like set_search_radius! (src/api.jl:26)
        radii = np.asarray([float(torch.tensor(float(r), dtype=self.T).item()) for r in radii], np.float64)
        coff = np.zeros(len(sizes) + 1, np.int64)
        coff[1:] = np.cumsum(sizes)
        self.coords = colmajor(coords)
        self.n_clouds = len(sizes)
        self.coff = coff
        ctx = self._ctx
        ctx.bind_stream()
        ctx.check(ctx.lib.oct_tree_build_batch(ctx.handle, self.tree.handle, _ptr(self.coords),
                                               int(self.coords.shape[1]), coff.ctypes.data_as(C.c_void_p),
                                               radii.ctypes.data_as(C.c_void_p), self.n_clouds), "batched run!")
        self.tree.built = True
        return self

    def build_edges(self) -> BatchedEdges:
        ctx = self._ctx
        ctx.bind_stream()
        buf = self._buf
        ne = C.c_int64()
        ctx.check(ctx.lib.oct_edges_count(ctx.handle, self.tree.handle, self.tree.handle, 1, C.byref(ne)),
                  "batched build_edges")
        n_edges = int(ne.value)
        _resize_buffer(buf, self.T, self.ndims, n_edges, self.device)
        eoff = np.zeros(self.n_clouds + 1, np.int64)
        ctx.check(ctx.lib.oct_batch_edge_offsets(ctx.handle, self.tree.handle, eoff.ctypes.data_as(C.c_void_p)),
                  "batched build_edges")
        if n_edges > 0:
            ctx.check(ctx.lib.oct_edges_fill(ctx.handle, self.tree.handle, self.tree.handle, 1, _ptr(buf.senders),
                                             _ptr(buf.receivers), _ptr(buf.rel_displacement.t()),
                                             _ptr(buf.rel_dist_norm), n_edges), "batched build_edges")
        return BatchedEdges(buf.senders, buf.receivers, buf.rel_displacement, buf.rel_dist_norm, eoff)
