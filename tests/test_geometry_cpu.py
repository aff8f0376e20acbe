"""Geometry set-up (UGKSBlock.updateGeom, ugks_block.py:667-760) on a
curvilinear multi-block grid: the oracle's restatement of xyExchange,
xyExtrapolate and cellGeom against the reference's own kernels compiled for
the CPU, run block by block and face by face in the reference's order (one
thread: the reference's extrapolation work items overlap)."""
import numpy as np
import pytest

import host  # noqa: F401  (puts oracle/ on the path)
import programs
import ugks_setup as us
from pyugks_b200 import configs
from pyugks_b200.problem import geometry

CASES = {
    "warped_1x1": lambda: configs.warped_cavity(nb=1, n=8, m=8),
    "warped_2x2_weno": lambda: configs.warped_cavity(nb=2, n=8, m=8, flux_method="WENO5", vlim=5.0),
}


def reference_geometry(case):
    c = us.Constants(case)
    G = c.ghost
    blocks = case["blocks"]
    progs, xys = [], []
    for k, b in enumerate(blocks):
        if not programs.reference_available(c, b, k):
            pytest.skip("compiled reference not available")
        progs.append(programs.RefProgram(c, b, k, threads=1))
        xy = np.full((b["ni"] + 2 * G + 1, b["nj"] + 2 * G + 1, 2), np.nan)
        xy[G:G + b["ni"] + 1, G:G + b["nj"] + 1, 0] = b["x"]
        xy[G:G + b["ni"] + 1, G:G + b["nj"] + 1, 1] = b["y"]
        xys.append(xy)
    out = []
    for k, b in enumerate(blocks):
        ni, nj = b["ni"], b["nj"]
        for face, bc in enumerate(b["bc"]):
            ns = face in (us.NORTH, us.SOUTH)
            if bc["type"] == us.ADJACENT:
                o = bc["other_block"]
                g = (ni, G - 1) if ns else (G - 1, nj)
                progs[k].xyExchange(g, xys[k], face, xys[o], blocks[o]["ni"] + 2 * G, blocks[o]["nj"] + 2 * G,
                                    bc["other_face"], bc.get("orientation", 1), bc.get("transform", us.TRANSFORM),
                                    bc.get("flip_normal", 0), k, o)
            else:
                g = (ni, G) if ns else (G, nj)
                progs[k].xyExtrapolate(g, xys[k], face)
        Ni, Nj = ni + 2 * G, nj + 2 * G
        area, centre = np.zeros((Ni, Nj)), np.zeros((Ni, Nj, 2))
        mid, normal, length = np.zeros((Ni, Nj, 2, 2)), np.zeros((Ni, Nj, 2, 2)), np.zeros((Ni, Nj, 2))
        progs[k].cellGeom((Ni, Nj), xys[k], area, centre, mid, normal, length)
        out.append(dict(xy=xys[k], area=area, centre=centre, mid_side=mid, normal=normal, side_length=length))
    return out


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(np.nan_to_num(a), np.nan_to_num(b))


@pytest.mark.parametrize("name", sorted(CASES))
def test_geometry_restatements_match_the_reference_kernels(name):
    case = CASES[name]()
    ref = reference_geometry(case)
    G = us.Constants(case).ghost
    ora = us.block_geometry(case, G)
    prod = geometry(case, G)
    for r, o, p in zip(ref, ora, prod):
        for key in ("xy", "area", "centre", "mid_side", "normal", "side_length"):
            assert same(o[key], r[key]), (name, key, "oracle")
            assert same(p[key], r[key]), (name, key, "product host set-up")
    # the grid really is curvilinear: interior face normals are not axis-aligned
    n = ora[0]["normal"][G:-G, G:-G]
    assert np.max(np.abs(n[..., 0, 0])) > 1e-3
