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


# ---------------------------------------------------------------------------
# block connections: two equal square blocks and ghost-exchange arguments for
# every pairing the reference's edgeExchange accepts (clGhostRoutines.c:407-538)
# ---------------------------------------------------------------------------
FACES = (0, 1, 2, 3)   # NORTH, EAST, SOUTH, WEST
FLIPS = (0, 1, 2, 3)   # NO_FLIP, FLIP_NS, FLIP_D, FLIP_EW


def square_pair_case(flux_method="vanLeer", n=5, m=4, links=None):
    """Two n x n unit-square blocks (block 1 shifted by 2 along x, so that no
    face corners coincide).  links: {(block, face): (other block, other face,
    orientation, flip)}; unlinked faces are diffuse walls."""
    from pyugks_b200 import configs
    from pyugks_b200 import defs as D
    case = configs.base_case(flux_method, 0.05, m, 4.0, 0.3)
    for b in range(2):
        x, y = configs.uniform_grid(n, n, 2.0 * b, 2.0 * b + 1.0)
        bc = [configs.diffuse(1.0) for _ in range(4)]
        for f in range(4):
            if links and (b, f) in links:
                ob, of, ori, flip = links[(b, f)]
                bc[f] = dict(configs.adjacent(ob, of, orientation=ori, flip=flip), transform=D.NO_TRANSFORM)
        case["blocks"].append(dict(ni=n, nj=n, x=x, y=y, bc=bc,
                                   fill=dict(D=1.0, U=0.0, V=0.0, T=1.0, qx=0.0, qy=0.0)))
    return case


def ghosted_xy(case, k, G):
    """Block k's vertex array with ghost layers (NaN there), the layout the
    kernels read (Ni+1, Nj+1, 2)."""
    b = case["blocks"][k]
    xy = np.full((b["ni"] + 2 * G + 1, b["nj"] + 2 * G + 1, 2), np.nan)
    xy[G:G + b["ni"] + 1, G:G + b["nj"] + 1, 0] = b["x"]
    xy[G:G + b["ni"] + 1, G:G + b["nj"] + 1, 1] = b["y"]
    return xy


def face_corner_ids(face, NI, NJ, G):
    """The two corner vertices of a face (edgeExchange's A1/A2, B1/B2)."""
    return {0: ((G, NJ - G), (NI - G, NJ - G)), 1: ((NI - G, G), (NI - G, NJ - G)),
            2: ((G, G), (NI - G, G)), 3: ((G, G), (G, NJ - G))}[face]


def exchange_args(case, G, this_face, that_face, aligned):
    """xyA, xyB for one pairing: with aligned, block 1's corners of
    that_face are set to block 0's corners of this_face, so edgeExchange
    sees the faces aligned; otherwise all four corners differ."""
    xyA, xyB = ghosted_xy(case, 0, G), ghosted_xy(case, 1, G)
    if aligned:
        NI, NJ = xyA.shape[0] - 1, xyA.shape[1] - 1
        a = face_corner_ids(this_face, NI, NJ, G)
        b = face_corner_ids(that_face, NI, NJ, G)
        for (ai, aj), (bi, bj) in zip(a, b):
            xyB[bi, bj] = xyA[ai, aj]
    return np.ascontiguousarray(xyA), np.ascontiguousarray(xyB)


def pairings():
    """Every (this face, that face, orientation, flip, aligned) combination."""
    return [(t, o, ori, fl, al) for t in FACES for o in FACES for ori in (0, 1) for fl in FLIPS
            for al in (False, True)]
