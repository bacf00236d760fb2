"""Helpers that turn tests/golden/reference_kats.json into concrete inputs."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_kats():
    with open(os.path.join(HERE, "golden", "reference_kats.json")) as f:
        return json.load(f)


def f32(v):
    """Evaluate a Float32 literal expression the way Julia does."""
    if isinstance(v, str):
        if v == "1f0":
            return np.float32(1.0)
        if v == "1f0/0.1f0":
            return np.float32(1.0) / np.float32(0.1)
        if v == "1.001f0*1f0":
            return np.float32(1.001) * np.float32(1.0)
        raise ValueError(v)
    return np.float32(v)


def coords_of(case):
    return np.array([[f32(c) for c in row] for row in case["coords"]], dtype=np.float32)
