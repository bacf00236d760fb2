import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ob():
    """The octopus.jl_b200 package (imported as octopus_b200)."""
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.ensure_built()
    return oracle


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


# ---- seeded synthetic inputs with the shapes of the reference's test cases --
def uniform(n, d, seed, lo=0.0, hi=1.0, dtype=np.float32):
    rng = np.random.default_rng(seed)
    return (lo + (hi - lo) * rng.random((n, d))).astype(dtype)


def clustered(n, d, seed, dtype=np.float32):
    """Two Gaussian blobs (test/build.jl:94-106 shape)."""
    rng = np.random.default_rng(seed)
    a = 0.1 * rng.standard_normal((n // 2, d)) + 0.25
    b = 0.1 * rng.standard_normal((n - n // 2, d)) - 0.25
    return np.concatenate([a, b]).astype(dtype)


def lattice(per, d, h, jitter, seed, dtype=np.float32):
    """Jittered cubic lattice (the SPH configuration's shape)."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(*[np.arange(per)] * d, indexing="ij"), -1).reshape(-1, d).astype(np.float64)
    x = g * h + rng.uniform(-jitter, jitter, g.shape)
    return x.astype(dtype)
