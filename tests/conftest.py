"""Shared test setup.

Markers: `gpu` tests need a CUDA sm_100 device and call the engine through
its C ABI (librq.so); everything else runs on the CPU (oracle, host logic,
ABI exports).  The oracle (oracle/) is imported here only as the checker.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "rdna2-accel-raster_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) and runs the CUDA kernels")


@pytest.fixture(scope="session")
def ctx():
    import torch
    import rq
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    c = rq.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def have_ref():
    import pyoracle
    return pyoracle.have_ref()


def soup(n, seed, scale=1.0):
    """Random triangle soup: non-indexed float32 [3n, 3] vertices."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-scale, scale, size=(n, 1, 3)).astype(np.float32)
    e = rng.uniform(-0.05 * scale, 0.05 * scale, size=(n, 3, 3)).astype(np.float32)
    return (c + e).reshape(-1, 3).astype(np.float32)
