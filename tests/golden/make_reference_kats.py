"""Writes reference_kats.json: the known-answer cases of Octopus.jl's own test
suite for the neighbor-search path, transcribed from the literal values in
its test files (cited per case), plus Morton codes computed by an
independent bit-by-bit interleave.

Run: python tests/golden/make_reference_kats.py
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def interleave3(x, y, z):
    """Bit-by-bit Morton interleave, bit i of x -> bit 3i (z<<2 | y<<1 | x)."""
    c = 0
    for i in range(21):
        c |= ((x >> i) & 1) << (3 * i)
        c |= ((y >> i) & 1) << (3 * i + 1)
        c |= ((z >> i) & 1) << (3 * i + 2)
    return c


def interleave2(x, y):
    c = 0
    for i in range(31):
        c |= ((x >> i) & 1) << (2 * i)
        c |= ((y >> i) & 1) << (2 * i + 1)
    return c


def main():
    m3 = [(0, 0, 0), (1, 2, 3), (7, 11, 19), (0x1FFFFF, 0x1FFFFF, 0x1FFFFF), (1_000_000, 500_000, 750_000)]
    m2 = [(0, 0), (1, 2), (7, 11), (0x7FFFFFFF, 0x7FFFFFFF), (1_000_000, 500_000), (123_456_789, 987_654_321)]
    kats = {
        "morton3_roundtrip": {
            "source": "test/morton.jl:10-19",
            "cases": [{"xyz": list(t), "code": interleave3(*t)} for t in m3],
        },
        "morton3_monotone_x": {"source": "test/morton.jl:21-29", "y": 42, "z": 7, "x_max": 64},
        "bin_point3": {
            "source": "test/morton.jl:31-38",
            "cases": [
                {"p": [0.5, 1.5, 2.9], "o": [0.0, 0.0, 0.0], "inv_cs": "1f0", "cell": [0, 1, 2]},
                {"p": [3.2, 3.2, 3.2], "o": [3.0, 3.0, 3.0], "inv_cs": "1f0/0.1f0", "cell": [2, 2, 2]},
            ],
        },
        "morton2_roundtrip": {
            "source": "test/morton.jl:42-50",
            "cases": [{"xy": list(t), "code": interleave2(*t)} for t in m2],
        },
        "morton2_top_bits_zero": {
            "source": "test/morton.jl:52-58",
            "cases": [[0x7FFFFFFF, 0x7FFFFFFF], [1_000_000, 999_999], [0, 0x7FFFFFFF]],
        },
        "morton2_monotone_x": {"source": "test/morton.jl:60-68", "y": 42, "x_max": 64},
        "bin_point2": {
            "source": "test/morton.jl:70-75",
            "cases": [
                {"p": [0.5, 1.5], "o": [0.0, 0.0], "inv_cs": "1f0", "cell": [0, 1]},
                {"p": [3.2, 3.2], "o": [3.0, 3.0], "inv_cs": "1f0/0.1f0", "cell": [2, 2]},
            ],
        },
        "exact_radius_included_3d": {
            "source": "test/edge_cases.jl:68-78",
            "coords": [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]], "r": 1.0,
            "neighbors": {"1": [2], "2": [1]},
        },
        "just_past_radius_excluded_3d": {
            "source": "test/edge_cases.jl:80-89",
            "coords": [[0.0, 0.0, 0.0], ["1.001f0*1f0", 0.0, 0.0]], "r": 1.0,
            "neighbors": {"1": [], "2": []},
        },
        "exact_radius_included_2d": {
            "source": "test/edge_cases.jl:91-99",
            "coords": [[0.0, 0.0], [1.0, 0.0]], "r": 1.0,
            "neighbors": {"1": [2]},
        },
        "coincident_3d": {"source": "test/edge_cases.jl:103-116", "n": 100, "ndims": 3, "r": 0.1},
        "coincident_2d": {"source": "test/edge_cases.jl:118-128", "n": 50, "ndims": 2, "r": 0.1},
        "coincident_perm_3d": {"source": "test/edge_cases.jl:182-193", "n": 64, "ndims": 3, "r": 0.1},
        "docstring_example": {
            "source": "src/api.jl:263-280",
            "coords": [[0.0, 0.0, 0.0], [0.0, 0.0, 0.0], [1.0, 0.0, 0.0]], "r": 0.5,
            "neighbors": {"1": [2]},
        },
        "single_point": {
            "source": "test/build.jl:108-117",
            "coords": [[0.0, 0.0, 0.0]], "r": 1.0, "n_nodes": 1, "neighbors": {"1": []},
        },
        "empty_set": {
            "source": "test/edge_cases.jl:16-64",
            "ndims": [3, 2], "r": 0.1, "n_nodes": 0, "n_edges": 0,
        },
        "tiny_radius": {"source": "test/edge_cases.jl:157-167", "n": 200, "ndims": 3, "r": 1e-8},
        "huge_radius": {"source": "test/edge_cases.jl:169-180", "n": 100, "ndims": 3, "r": 100.0},
    }
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump(kats, f, indent=1)


if __name__ == "__main__":
    main()
