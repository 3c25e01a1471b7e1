import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def random_points(dtype, n, d, seed):
    rng = np.random.default_rng(seed)
    if dtype == np.float32:
        return rng.standard_normal((n, d)).astype(np.float32)
    if dtype == np.uint8:
        return rng.integers(0, 256, (n, d)).astype(np.uint8)
    return rng.integers(-128, 128, (n, d)).astype(np.int8)


@pytest.fixture(scope="session")
def lib_built():
    from parlayann_b200 import build_ext

    build_ext.build()
    from oracle import oracle

    oracle.build()
    return True
