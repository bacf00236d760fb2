"""B200-native fixed-radius octree neighbor search behind Octopus.jl's TNS API.

The compute lives in ``lib/liboctopus_b200.so`` (CUDA, sm_100a, C ABI in
``include/octopus_b200.h``); this package is the host-side mirror of the
reference's public functions (src/Octopus.jl:31-44) over that library.
"""
from .api import (  # noqa: F401
    ArgumentError, DimensionMismatch, InexactError, OctopusError,
    TNS, PointSet, Octree, EdgeBuffer, NeighborBuffer, EdgesTuple, DeviceView,
    set_search_radius_, set_refit_mode_, add_point_set_, resize_point_set_,
    update_point_set_, set_active_search_, run_, build_edges_, build_edges,
    for_each_neighbor, get_neighborlist, materialize_all_neighbors_,
    device_view, build_edges_diff, colmajor, synchronize, BatchedSearch, BatchedEdges,
    prepare_zsort, apply_zsort, prepare_zsort_, apply_zsort_, build_edges_diff_pair,
)
from . import _lib  # noqa: F401

__all__ = [
    "TNS", "set_search_radius_", "set_refit_mode_", "add_point_set_", "resize_point_set_",
    "update_point_set_", "set_active_search_", "run_", "for_each_neighbor", "get_neighborlist",
    "materialize_all_neighbors_", "NeighborBuffer", "build_edges", "build_edges_", "EdgeBuffer", "build_edges_diff", "build_edges_diff_pair",
    "device_view", "prepare_zsort", "apply_zsort", "ArgumentError", "DimensionMismatch", "InexactError", "OctopusError",
]
