import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libhp2d.so")
    config.addinivalue_line("markers", "slow: long-running")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def hp2d_lib():
    from hydropol2d_b200 import build
    build.build()
    from hydropol2d_b200 import _abi
    return _abi.lib()


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    """Bit-level equality that treats NaN == NaN and +0 == -0 as equal."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    return bool(np.array_equal(a, b, equal_nan=True))


def first_mismatch(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    idx = np.argwhere(bad)
    if idx.size == 0:
        return None
    i = tuple(idx[0])
    return i, a[i], b[i], int(bad.sum())
