"""CPU oracle for the Octopus.jl neighbor-search path -- TEST INFRASTRUCTURE.

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  It wraps ``octopus_oracle.cpp`` (a
C++ restatement of the reference's ``src/cpu`` path) through ctypes.

Arrays follow the reference's memory layout: a Julia ``(NDIMS, N)``
column-major matrix is a C-contiguous numpy array of shape ``(N, NDIMS)``.
Indices are 1-based Int32, as in the reference.
"""
from .pyoracle import (  # noqa: F401
    lib_path, load, ensure_built, morton_encode3, morton_encode2, morton_decode3,
    morton_decode2, bin_point_f32, build_tree, build_edges, brute_force,
    diff_backward, max_threads,
)
