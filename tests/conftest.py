import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls through libbzgrav.so")


@pytest.fixture(scope="session")
def gpu():
    """The built engine library on a visible GPU; GPU tests fail loudly without them."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected without a visible CUDA device")
    from blitzar_b200 import _lib

    return _lib.load()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.lib()
    return O


def plummer(n, seed=1, a=1.0):
    """Small seeded Plummer sphere (positions only) for parity tests."""
    rng = np.random.default_rng(seed)
    u = rng.random(n) * 0.999
    r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return (r[:, None] * v).astype(np.float32)
