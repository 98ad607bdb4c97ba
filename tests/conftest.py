"""Shared test configuration.

Tests marked ``gpu`` need a CUDA device and libblond_b200.so; everything
else runs on the CPU (oracle, golden fixtures, host logic, C ABI exports).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def normwise(a, b):
    """max|a-b| / max|b| -- the parity measure for coordinates and voltages."""
    a, b = np.asarray(a), np.asarray(b)
    # complex arrays (spectra, impedances) are compared as complex numbers
    t = np.complex128 if (np.iscomplexobj(a) or np.iscomplexobj(b)) else np.float64
    a, b = a.astype(t), b.astype(t)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    from blond_b200 import _lib
    _lib.load()
    torch.cuda.set_device(0)
    return torch.device("cuda", 0)
