"""Block geometry set-up on the device, as UGKSim.initGeom /
UGKSBlock.updateGeom run it (ugks_sim.py:256-262, ugks_block.py:667-760):
per block, face by face (N, E, S, W), ghost vertices from the neighbouring
block (xyExchange) or by extrapolation (xyExtrapolate), then the cell metrics
of every cell (cellGeom), through the drop-in kernels.  The result is the
per-block dict problem.geometry builds on the host: xy, area, centre,
mid_side, normal, side_length.
"""
from __future__ import annotations

import numpy as np

from . import defs as D
from .desc import VelocityTables, block_desc
from .kernel_program import KernelProgram
from .problem import Constants


def device_geometry(case: dict, device="cuda", queue=None, host=True):
    """Geometry of every block of `case` computed on the device; numpy
    arrays when host is True, else the device tensors."""
    import torch
    const = Constants(case)
    G = const.ghost
    tabs = VelocityTables(const, device)
    blocks = case["blocks"]
    progs, xys = [], []
    for b in blocks:
        progs.append(KernelProgram(block_desc(const, b, tabs)))
        xy = np.full((b["ni"] + 2 * G + 1, b["nj"] + 2 * G + 1, 2), np.nan)
        xy[G:G + b["ni"] + 1, G:G + b["nj"] + 1, 0] = b["x"]
        xy[G:G + b["ni"] + 1, G:G + b["nj"] + 1, 1] = b["y"]
        xys.append(torch.from_numpy(xy).to(device))
    out = []
    for k, b in enumerate(blocks):
        ni, nj = b["ni"], b["nj"]
        Ni, Nj = ni + 2 * G, nj + 2 * G
        for face, bc in enumerate(b["bc"]):
            ns = face in (D.NORTH, D.SOUTH)
            if bc["type"] == D.ADJACENT:
                o = bc["other_block"]
                g = (ni, G - 1, 1) if ns else (G - 1, nj, 1)
                progs[k].xyExchange(queue, g, None, xys[k], face, xys[o], blocks[o]["ni"] + 2 * G,
                                    blocks[o]["nj"] + 2 * G, bc["other_face"], bc.get("orientation", 1),
                                    bc.get("transform", D.TRANSFORM), bc.get("flip_normal", 0), k, o)
            else:
                g = (ni, G, 1) if ns else (G, nj, 1)
                progs[k].xyExtrapolate(queue, g, None, xys[k], face)
        z = lambda *s: torch.zeros(s, dtype=torch.float64, device=device)
        geo = dict(xy=xys[k], area=z(Ni, Nj), centre=z(Ni, Nj, 2), mid_side=z(Ni, Nj, 2, 2),
                   normal=z(Ni, Nj, 2, 2), side_length=z(Ni, Nj, 2))
        progs[k].cellGeom(queue, (Ni, Nj, 1), None, geo["xy"], geo["area"], geo["centre"], geo["mid_side"],
                          geo["normal"], geo["side_length"])
        out.append({key: v.cpu().numpy() for key, v in geo.items()} if host else geo)
    return out
