"""ctypes binding of ``liboctopus_b200.so`` (declared in include/octopus_b200.h).

Loading fails loudly when the shared object is missing: there is no CPU
fallback behind this package.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "liboctopus_b200.so")

OK = 0
ERR_ARGUMENT = 1
ERR_DIMENSION = 2
ERR_INEXACT = 3
ERR_CUDA = 4
ERR_OVERFLOW = 5
ERR_CAPACITY = 6
ERR_TIMEOUT = 7
ERR_STATE = 8

# Context options (oct_ctx_set_option / oct_ctx_get_option).
OPT_WAIT_LIMIT = 1
OPT_NODE_CAPACITY = 2
OPT_RECORD_CAP = 3
OPT_GUARD_CHECK = 4
OPT_WITHHOLD_TILE = 5
OPT_MAX_SEG = 6
OPT_MULTI_POP = 7
OPT_FILL_CHUNK = 8
OPT_GROUP_CAP = 9
OPT_SUB_BOXES = 10
OPT_PREFETCH = 11
STAT_TUNING_ROW = 99
STAT_BUILD_ATTEMPTS = 100
STAT_RECORD_OVERFLOW = 101
STAT_RECORD_CAP = 102


class TreeView(C.Structure):
    """oct_tree_view."""
    _fields_ = [
        ("n_points", C.c_int64),
        ("n_nodes", C.c_int64),
        ("ndims", C.c_int32),
        ("dtype", C.c_int32),
        ("radius", C.c_double),
        ("node_first", C.c_void_p),
        ("node_last", C.c_void_p),
        ("node_children", C.c_void_p),
        ("bounds_min", C.c_void_p),
        ("bounds_max", C.c_void_p),
        ("perm", C.c_void_p),
        ("morton", C.c_void_p),
    ]


# (name, restype, argtypes) for every entry point of include/octopus_b200.h.
P, I, I64, D = C.c_void_p, C.c_int, C.c_int64, C.c_double
SIGNATURES = [
    ("oct_version", I, []),
    ("oct_status_string", C.c_char_p, [I]),
    ("oct_ctx_create", I, [I, C.POINTER(P)]),
    ("oct_ctx_destroy", I, [P]),
    ("oct_ctx_set_stream", I, [P, P]),
    ("oct_ctx_last_error", C.c_char_p, [P]),
    ("oct_synchronize", I, [P]),
    ("oct_tree_create", I, [P, I, I, C.POINTER(P)]),
    ("oct_tree_destroy", I, [P]),
    ("oct_tree_build", I, [P, P, P, I64, D, I]),
    ("oct_tree_build_batch", I, [P, P, P, I64, P, P, C.c_int32]),
    ("oct_batch_edge_offsets", I, [P, P, P]),
    ("oct_tree_last_build", I, [P, C.POINTER(I), C.POINTER(I64)]),
    ("oct_tree_n_nodes", I, [P, P, C.POINTER(I64)]),
    ("oct_tree_view_get", I, [P, P, C.POINTER(TreeView)]),
    ("oct_edges_count", I, [P, P, P, I, C.POINTER(I64)]),
    ("oct_edges_traversal_stats", I, [P, P, P, I, P, I]),
    ("oct_edges_fill", I, [P, P, P, I, P, P, P, P, I64]),
    ("oct_edges_fill_diff", I, [P, P, P, P, P, P, P, I64]),
    ("oct_csr_fill", I, [P, P, P, I, P, P, I64]),
    ("oct_zsort_apply", I, [P, P, P, P, I64, I64, I]),
    ("oct_permute_rows", I, [P, P, I64, P, P, I64, I]),
    ("oct_neighbors", I, [P, P, P, I64, P, P, I64]),
    ("oct_edges_diff_backward", I, [P, I, I, I64, I64, P, P, P, P, P, P, D, P]),
    ("oct_edges_diff_backward_pair", I, [P, I, I, I64, I64, I64, P, P, P, P, P, P, D, P, P]),
    ("oct_edges_diff_backward_recompute", I, [P, I, I, I64, I64, P, P, P, P, P, D, P]),
    ("oct_edges_diff_backward_ordered", I, [P, I, I, I64, I64, P, P, P, P, P, P, P, D, P, P]),
    ("oct_edges_diff_backward_mirror", I, [P, I, I, I64, I64, P, P, P, P, P, P, P, P, D, P, P]),
    ("oct_edges_count_noalloc", I, [P, P, P, I, P, P, C.POINTER(I64)]),
    ("oct_ctx_set_option", I, [P, I, I64]),
    ("oct_ctx_get_option", I, [P, I, C.POINTER(I64)]),
    ("oct_ctx_load_tuning", I, [P, C.c_char_p]),
    ("oct_tuning_select", I, [C.c_char_p, I, I, I64, D, P, P]),
    ("oct_profile_enable", I, [P, I]),
    ("oct_profile_phase_name", C.c_char_p, [I]),
    ("oct_profile_read", I, [P, P, P, I]),
    ("oct_profile_kernel_launches", I64, [P]),
]

TRAVERSAL_STATS = ["groups", "queries", "expansions", "children_tested", "leaf_chunks", "targets_staged",
                   "pair_steps", "pair_tests", "hits", "cycles_total", "cycles_leaf", "cycles_pairs"]

PHASES = ["bounds", "encode", "sort", "gather", "topology", "refit", "count", "scan", "fill", "adjoint", "groups"]

_LIB = None
_LOCK = threading.Lock()


def load(path: str | None = None):
    """Load (once) and type the shared library.  Raises if it is absent."""
    global _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        path = path or LIB_PATH
        if not os.path.exists(path):
            raise ImportError(
                f"liboctopus_b200.so not found at {path}; build it with "
                "`python octopus.jl_b200/build.py` (nvcc, sm_100a)")
        lib = C.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
        return lib


def declared_symbols():
    return [name for name, _, _ in SIGNATURES]
