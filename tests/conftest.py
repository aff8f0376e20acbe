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


def vec_err(ax, ay, bx, by):
    """Error of a 2-vector field relative to its largest magnitude."""
    den = max(float(np.max(np.abs(bx))), float(np.max(np.abs(by))))
    num = max(float(np.max(np.abs(np.asarray(ax) - bx))), float(np.max(np.abs(np.asarray(ay) - by))))
    return num / den if den > 0 else num


def field_errors(x, y):
    """Per-field errors: rho and T relative to their maxima, velocity (U, V)
    and heat flux (qx, qy) relative to the largest vector magnitude."""
    return {"rho": rel_err(x["rho"], y["rho"]), "T": rel_err(x["T"], y["T"]),
            "UV": vec_err(x["U"], x["V"], y["U"], y["V"]),
            "q": vec_err(x["qx"], x["qy"], y["qx"], y["qy"])}


def fields_err(fa, fb):
    """Worst field error over blocks."""
    worst = 0.0
    for x, y in zip(fa, fb):
        worst = max(worst, max(field_errors(x, y).values()))
    return worst


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyugks_b200 import build
    build.build()
    return torch.device("cuda:0")
