"""Shared test set-up.

Markers: `gpu` tests need a CUDA device (they run on a B200); everything else
runs on CPU.  The library and the oracle are built on first use if missing.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def built():
    """Builds libbbrt_cuda.so and the oracle port when they are missing."""
    from billardballraytracing3d_b200 import _capi
    import oracle
    if not os.path.exists(_capi.LIB_PATH):
        from billardballraytracing3d_b200 import build as B
        B.build(verbose=False)
    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build()
    return True


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


@pytest.fixture(scope="session")
def workloads():
    """Seeded workloads at test sizes: name -> (patches, origins, dirs, max_bounces, coarse_n, tol)."""
    from billardballraytracing3d_b200 import scenes
    cache = {}

    def get(name, n=None):
        key = (name, n)
        if key not in cache:
            cache[key] = scenes.workload(name, n)
        return cache[key]
    return get
