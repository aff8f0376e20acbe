"""Shared test set-up.

``-m gpu`` tests need a CUDA device and the built libugks_b200.so; the others
run on the CPU.  The oracle (``oracle/``) is imported here as the checker.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libugks_b200.so")


def rel_err(a, b):
    """max |a - b| / max |b| (0 when both are zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b))
    num = np.max(np.abs(a - b))
    return float(num / den) if den > 0 else float(num)


def fields_err(fa, fb):
    """Worst rel_err over blocks and over rho, U, V, T, qx, qy."""
    worst = 0.0
    for x, y in zip(fa, fb):
        for k in ("rho", "U", "V", "T", "qx", "qy"):
            worst = max(worst, rel_err(x[k], y[k]))
    return worst


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyugks_b200 import build
    build.build()
    return torch.device("cuda:0")
