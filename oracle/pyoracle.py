"""ctypes bindings of the CPU oracle (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_LOCK = threading.Lock()


def lib_path() -> str:
    return os.path.join(_HERE, "lib", "liboctopus_oracle.so")


def ensure_built() -> str:
    """Compile the oracle with its Makefile when the shared object is missing
    or older than its source."""
    so = lib_path()
    src = os.path.join(_HERE, "octopus_oracle.cpp")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return so


def load():
    global _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        lib = C.CDLL(ensure_built())
        P = C.c_void_p
        i64, i32 = C.c_int64, C.c_int32
        lib.oracle_morton_encode3.restype = C.c_uint64
        lib.oracle_morton_encode3.argtypes = [C.c_uint32] * 3
        lib.oracle_morton_encode2.restype = C.c_uint64
        lib.oracle_morton_encode2.argtypes = [C.c_uint32] * 2
        lib.oracle_morton_decode3.argtypes = [C.c_uint64, P]
        lib.oracle_morton_decode2.argtypes = [C.c_uint64, P]
        lib.oracle_bin_point_f32.restype = C.c_int
        lib.oracle_bin_point_f32.argtypes = [C.c_int, P, P, C.c_float, P]
        lib.oracle_tree_build.restype = P
        lib.oracle_tree_build.argtypes = [P, i64, C.c_int, C.c_int, C.c_double, i32, C.c_int,
                                          C.POINTER(C.c_int)]
        lib.oracle_tree_n_nodes.restype = i64
        lib.oracle_tree_n_nodes.argtypes = [P]
        lib.oracle_tree_copy.argtypes = [P] * 9
        lib.oracle_tree_free.argtypes = [P]
        lib.oracle_edges_build.restype = P
        lib.oracle_edges_build.argtypes = [P, P, i64, P, C.c_double, C.c_int, C.c_int]
        lib.oracle_edges_build_range.restype = P
        lib.oracle_edges_build_range.argtypes = [P, P, i64, P, C.c_double, C.c_int, C.c_int, i64, i64]
        lib.oracle_edges_n.restype = i64
        lib.oracle_edges_n.argtypes = [P]
        lib.oracle_edges_copy.argtypes = [P, C.c_int, C.c_int, P, P, P, P, P, i64]
        lib.oracle_edges_free.argtypes = [P]
        lib.oracle_brute_force.restype = i64
        lib.oracle_brute_force.argtypes = [P, i64, P, i64, C.c_int, C.c_int, C.c_double, C.c_int,
                                           P, P, i64]
        lib.oracle_diff_backward.argtypes = [C.c_int, C.c_int, i64, i64, P, P, P, P, P, P,
                                             C.c_double, P]
        lib.oracle_max_threads.restype = C.c_int
        _LIB = lib
        return lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _dtype_code(a: np.ndarray) -> int:
    if a.dtype == np.float32:
        return 0
    if a.dtype == np.float64:
        return 1
    raise TypeError(f"oracle supports float32/float64 coordinates, got {a.dtype}")


def max_threads() -> int:
    return int(load().oracle_max_threads())


def morton_encode3(x: int, y: int, z: int) -> int:
    return int(load().oracle_morton_encode3(x, y, z))


def morton_encode2(x: int, y: int) -> int:
    return int(load().oracle_morton_encode2(x, y))


def morton_decode3(c: int):
    out = np.zeros(3, np.uint32)
    load().oracle_morton_decode3(c, _ptr(out))
    return tuple(int(v) for v in out)


def morton_decode2(c: int):
    out = np.zeros(2, np.uint32)
    load().oracle_morton_decode2(c, _ptr(out))
    return tuple(int(v) for v in out)


def bin_point_f32(p, o, inv_cs):
    """bin_point (src/morton.jl:83-95) in Float32.  Returns the cell tuple or
    raises OverflowError where Julia raises InexactError."""
    p = np.ascontiguousarray(p, np.float32)
    o = np.ascontiguousarray(o, np.float32)
    out = np.zeros(len(p), np.int32)
    st = load().oracle_bin_point_f32(len(p), _ptr(p), _ptr(o), C.c_float(np.float32(inv_cs)), _ptr(out))
    if st:
        raise OverflowError("InexactError: floor(Int32, x) out of range")
    return tuple(int(v) for v in out)


class OracleTree:
    """One point set's tree, as ``_run_cpu!`` (src/api.jl:194-250) builds it."""

    def __init__(self, coords: np.ndarray, radius: float, leaf_size: int = 32, nthreads: int = 0):
        coords = np.ascontiguousarray(coords)
        if coords.ndim != 2 or coords.shape[1] not in (2, 3):
            raise ValueError("coords must have shape (N, NDIMS) with NDIMS in (2, 3)")
        self.coords = coords
        self.n, self.ndims = coords.shape
        self.dtype = coords.dtype
        self.radius = float(radius)
        lib = load()
        st = C.c_int(0)
        nthreads = nthreads or max_threads()
        self._h = lib.oracle_tree_build(_ptr(coords), self.n, self.ndims, _dtype_code(coords),
                                        self.radius, leaf_size, nthreads, C.byref(st))
        self.status = int(st.value)
        nn = int(lib.oracle_tree_n_nodes(self._h))
        nch = 1 << self.ndims
        self.n_nodes = nn
        self.node_first = np.zeros(nn, np.int32)
        self.node_last = np.zeros(nn, np.int32)
        self.children = np.zeros((nn, nch), np.int32)
        self.bmin = np.zeros((nn, self.ndims), coords.dtype)
        self.bmax = np.zeros((nn, self.ndims), coords.dtype)
        self.perm = np.zeros(self.n if self.status == 0 else 0, np.int32)
        self.morton = np.zeros(self.n if self.n else 0, np.uint64)
        self.origin = np.zeros(3, np.float64)
        lib.oracle_tree_copy(self._h, _ptr(self.node_first), _ptr(self.node_last),
                             _ptr(self.children), _ptr(self.bmin), _ptr(self.bmax),
                             _ptr(self.perm) if self.perm.size else None,
                             _ptr(self.morton) if self.morton.size else None, _ptr(self.origin))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _LIB is not None:
            _LIB.oracle_tree_free(h)
            self._h = None


def build_tree(coords, radius, leaf_size=32, nthreads=0) -> OracleTree:
    return OracleTree(coords, radius, leaf_size, nthreads)


def build_edges(tree: OracleTree, coords_q: np.ndarray, radius=None, exclude_self=None,
                nthreads: int = 0, query_range=None):
    """build_edges_cpu! (src/cpu/edges_cpu.jl:172-247) for query coords against
    ``tree``.  Returns a dict of numpy arrays in the reference's COO order.

    ``query_range = (lo, hi)`` (0-based, half-open) returns only the edges of
    queries lo..hi-1: the slice of the full COO that those queries own, with
    ``offsets`` (hi - lo + 1 entries) counted from the slice's first edge."""
    lib = load()
    coords_q = np.ascontiguousarray(coords_q, tree.dtype)
    radius = tree.radius if radius is None else float(radius)
    if exclude_self is None:
        exclude_self = coords_q is tree.coords
    nthreads = nthreads or max_threads()
    nq = coords_q.shape[0]
    lo, hi = (0, nq) if query_range is None else (int(query_range[0]), int(query_range[1]))
    if not 0 <= lo <= hi <= nq:
        raise ValueError("query_range out of bounds")
    h = lib.oracle_edges_build_range(tree._h, _ptr(coords_q), nq, _ptr(tree.coords), radius,
                                     int(bool(exclude_self)), nthreads, lo + 1, hi)
    try:
        m = int(lib.oracle_edges_n(h))
        d = tree.ndims
        out = {
            "senders": np.zeros(m, np.int32),
            "receivers": np.zeros(m, np.int32),
            "rel_displacement": np.zeros((m, d), tree.dtype),
            "rel_dist_norm": np.zeros(m, tree.dtype),
            "offsets": np.zeros(hi - lo + 1, np.int64),
        }
        lib.oracle_edges_copy(h, d, _dtype_code(coords_q), _ptr(out["senders"]),
                              _ptr(out["receivers"]), _ptr(out["rel_displacement"]),
                              _ptr(out["rel_dist_norm"]), _ptr(out["offsets"]), hi - lo)
    finally:
        lib.oracle_edges_free(h)
    return out


def brute_force(coords_q, coords_t, radius, exclude_self):
    """All (receiver, sender) pairs within radius under the reference's
    formula, ordered by (receiver, sender)."""
    lib = load()
    cq = np.ascontiguousarray(coords_q)
    ct = np.ascontiguousarray(coords_t, cq.dtype)
    m = lib.oracle_brute_force(_ptr(cq), cq.shape[0], _ptr(ct), ct.shape[0], cq.shape[1],
                               _dtype_code(cq), float(radius), int(bool(exclude_self)), None, None, 0)
    snd = np.zeros(m, np.int32)
    rcv = np.zeros(m, np.int32)
    lib.oracle_brute_force(_ptr(cq), cq.shape[0], _ptr(ct), ct.shape[0], cq.shape[1],
                           _dtype_code(cq), float(radius), int(bool(exclude_self)),
                           _ptr(snd), _ptr(rcv), m)
    return snd, rcv


def diff_backward(n_points, senders, receivers, rel_disp, rel_dist, d_disp, d_dist, radius):
    """Serial pullback of build_edges_diff (ext/OctopusChainRulesCoreExt.jl:150-189)."""
    lib = load()
    rel_disp = np.ascontiguousarray(rel_disp)
    ndims = rel_disp.shape[1]
    dt = rel_disp.dtype
    grad = np.zeros((n_points, ndims), dt)
    lib.oracle_diff_backward(ndims, _dtype_code(rel_disp), n_points, len(senders),
                             _ptr(np.ascontiguousarray(senders, np.int32)),
                             _ptr(np.ascontiguousarray(receivers, np.int32)), _ptr(rel_disp),
                             _ptr(np.ascontiguousarray(rel_dist, dt)),
                             None if d_disp is None else _ptr(np.ascontiguousarray(d_disp, dt)),
                             None if d_dist is None else _ptr(np.ascontiguousarray(d_dist, dt)),
                             float(radius), _ptr(grad))
    return grad
