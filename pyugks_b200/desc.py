"""Per-block kernel descriptors and device velocity tables.

``ugks_block_desc`` carries what the reference compiled into each block's
OpenCL header (``ugks_CL.py:58-395``): sizes, physics constants, the velocity
tables (as device pointers) and the wall / adsorption values per face.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from . import defs as D
from .problem import Constants, isotherm_tables, wall_values


class VelocityTables:
    """Device copies of quad, weight and the mirror permutations."""

    def __init__(self, const: Constants, device):
        self.keep = []  # device tables referenced by block descriptors (isotherms)
        import torch
        vg = const.vgrid
        self.quad = torch.from_numpy(np.ascontiguousarray(vg.quad)).to(device)
        self.weight = torch.from_numpy(np.ascontiguousarray(vg.weight)).to(device)
        self.mirror_NS = torch.from_numpy(np.ascontiguousarray(vg.mirror_NS, dtype=np.int32)).to(device)
        self.mirror_EW = torch.from_numpy(np.ascontiguousarray(vg.mirror_EW, dtype=np.int32)).to(device)
        self.mirror_D = torch.from_numpy(np.ascontiguousarray(vg.mirror_D, dtype=np.int32)).to(device)


def block_desc(const: Constants, block: dict, tabs: VelocityTables) -> "_lib.BlockDesc":
    d = _lib.BlockDesc()
    G = const.ghost
    d.ni, d.nj = block["ni"], block["nj"]
    d.Ni, d.Nj = block["ni"] + 2 * G, block["nj"] + 2 * G
    d.ghost, d.Nv = G, const.Nv
    d.flux_method, d.relax_type = const.flux_code, const.relax_type
    d.u_num, d.v_num = const.vgrid.u_num, const.vgrid.v_num
    d.PI, d.Pr, d.umax, d.vmax = const.PI, const.Pr, const.umax, const.vmax
    d.Kn_eff, d.gam, d.K, d.omega = const.Kn_eff, const.gam, const.K, const.omega
    d.B = const.B
    d.quad, d.weight = tabs.quad.data_ptr(), tabs.weight.data_ptr()
    d.mirror_NS, d.mirror_EW, d.mirror_D = (tabs.mirror_NS.data_ptr(), tabs.mirror_EW.data_ptr(),
                                            tabs.mirror_D.data_ptr())
    fill_walls(d, block, tabs.keep, tabs.quad.device)
    return d


REFLECT_CODES = {"S": 0, "D": 1, "CL": 2}


def fill_walls(d, block: dict, keep: list, device):
    """Wall values and the adsorbing-wall tables of ugks_block_desc, printed
    as the reference's generated header prints them (ugks_CL.py:102-185);
    the device copies of tabulated isotherms are appended to ``keep``."""
    import torch
    for f, bc in enumerate(block["bc"]):
        d.wall_D[f], d.wall_U[f], d.wall_V[f], d.wall_T[f], d.wall_P[f] = wall_values(bc)
        if bc["type"] == D.ADSORBING:
            d.beta_n[f] = float("%0.15e" % bc.get("beta_n", 0.0))
            d.beta_t[f] = float("%0.15e" % bc.get("beta_t", 0.0))
            d.gamma_f[f] = float("%0.15e" % bc["gamma_f"])
            d.alpha_p[f] = float("%0.15e" % bc["alpha_p"])
            d.alpha_n[f] = float("%0.15e" % bc.get("alpha_n", 1.0))
            d.alpha_t[f] = float("%0.15e" % bc.get("alpha_t", 1.0))
            d.dynamic[f] = int(bc.get("dynamic", 1))
            scalar = np.ndim(bc["adsorb"]) == 0
            d.constant_adsorb[f] = 1 if scalar else 0
            d.adsorb[f] = float("%g" % bc["adsorb"]) if scalar else 0.0
            if not scalar:
                pts, tri, nbr = isotherm_tables(bc["adsorb"])
                tabs = [torch.from_numpy(x).to(device) for x in (pts, tri, nbr)]
                keep.extend(tabs)
                d.iso[f], d.tri[f], d.nbr[f] = (t.data_ptr() for t in tabs)
                d.n_tri[f] = tri.shape[0]
            d.k_des[f] = float(bc.get("k_des", 0.0))
            rt = bc.get("reflect_type", "S")
            d.reflect[f] = REFLECT_CODES.get(rt, 0)
        else:
            d.beta_n[f] = d.beta_t[f] = d.gamma_f[f] = d.alpha_p[f] = -1.0
            d.alpha_n[f] = d.alpha_t[f] = -1.0
            d.dynamic[f] = -1
            d.reflect[f] = -1
