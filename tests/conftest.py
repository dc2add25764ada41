"""Shared fixtures.  Tests marked `gpu` need a CUDA device and call the CUDA
library through its C ABI; everything else runs on CPU."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device; calls libmarfa_gpu.so")


@pytest.fixture(scope="session")
def tips():
    from marfa_b200 import data_path
    from marfa_b200.io import read_tips
    return read_tips(data_path("TIPS_subset.dat"))


@pytest.fixture(scope="session")
def gpu():
    """Fails (does not skip) when the CUDA library or device is missing."""
    import torch
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    from marfa_b200 import build
    build.build()
    from marfa_b200 import _lib
    return _lib.load()


def rel_err(a, b, floor_frac=1e-6):
    """Max relative error of a vs reference b over points with
    b > floor_frac * max(b)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    m = b > floor_frac * b.max()
    return float(np.max(np.abs(a[m] - b[m]) / b[m])), int(m.sum())
