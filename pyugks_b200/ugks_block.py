"""UGKSBlock: one block's device state and its kernel sequence.

Python-3 restatement of pyUGKS's ``UGKSBlock`` (``ugks_block.py:46-1623``) for
the time-step path, over torch CUDA tensors and the ``KernelProgram`` drop-in
(``prg.<kernel>(queue, global_size, local_size, *args)``).  Method names and
launch order follow the reference so that the per-kernel path can be checked
against it kernel by kernel:

* ``initFunctions``  ugks_block.py:258-432 (fresh start: f := fEQ(fill, Q),
  macro and Q re-taken from f, wall values)
* ``updateBC``       ugks_block.py:621-665 (ghost cells of the four faces)
* ``wall_flux``      ugks_block.py:930-983
* ``UGKS_flux``      ugks_block.py:1049-1260
* ``UGKS_update``    ugks_block.py:1262-1329 (incl. the residual)
* ``getDT``          ugks_block.py:1415-1433
* ``get_flag``       ugks_block.py:840-876 (status word read back)

Arrays use the reference layouts: f-like (Ni, Nj, Nv, 2), macro (ni, nj, 4) as
(rho, U, V, 1/T), per-face geometry (Ni, Nj, 2, ...).
"""
from __future__ import annotations

import sys

import numpy as np

from . import defs as D
from .desc import block_desc
from .kernel_program import KernelProgram
from .problem import fill_arrays


def _m_tuple(x, y):
    """ugks_block.py:28-32"""
    return tuple(a * b for a, b in zip(x, y)), y


class UGKSBlock:
    def __init__(self, sim, block_id: int, spec: dict, geom: dict, tabs, device, queue=None):
        import torch
        self.sim = sim
        self.id = block_id
        self.queue = queue
        const = sim.const
        self.ghost = G = const.ghost
        self.ni, self.nj = spec["ni"], spec["nj"]
        self.Ni, self.Nj = self.ni + 2 * G, self.nj + 2 * G
        if self.ni < G or self.nj < G:
            raise ValueError("a block needs at least %d cells per direction" % G)
        self.Nv = const.Nv
        self.bc_list = spec["bc"]
        self.desc = block_desc(const, spec, tabs)
        self.prg = KernelProgram(self.desc)
        dev = device
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        z = lambda *s: torch.zeros(s, dtype=torch.float64, device=dev)
        self.xy_D = t(geom["xy"])
        self.area_D = t(np.nan_to_num(geom["area"]))
        self.centre_D = t(np.nan_to_num(geom["centre"]))
        self.side_D = t(np.nan_to_num(geom["mid_side"]))
        self.normal_D = t(np.nan_to_num(geom["normal"]))
        self.length_D = t(np.nan_to_num(geom["side_length"]))
        self.area_H = geom["area"]
        Ni, Nj, Nv = self.Ni, self.Nj, self.Nv
        self.f_D = z(Ni, Nj, Nv, 2)
        self.flux_f_S_D, self.flux_f_W_D, self.sigma_D = z(Ni, Nj, Nv, 2), z(Ni, Nj, Nv, 2), z(Ni, Nj, Nv, 2)
        self.flux_macro_S_D, self.flux_macro_W_D = z(Ni, Nj, 4), z(Ni, Nj, 4)
        self.prim_D, self.aL_D, self.aR_D, self.aT_D = z(Ni, Nj, 4), z(Ni, Nj, 4), z(Ni, Nj, 4), z(Ni, Nj, 4)
        self.faceQ_D, self.Mxi_D = z(Ni, Nj, 2), z(Ni, Nj, 3)
        wl = max(self.ni, self.nj)
        self.wall_len = wl
        self.wall_prop_D = z(wl, 4, 4)
        cover = np.zeros((wl, 4, 4))
        for bci, bc in enumerate(self.bc_list):
            cover[:, bci, 0] = bc.get("cover_initial", 0.0)
        self.wall_cover_D = t(cover)
        self.wall_fluxes_D = z(wl, 4, 8)
        self.wall_dist_D = z(wl, Nv, 2)
        self.para_D = z(wl, 4, 4)
        macro, Q = fill_arrays(spec)
        self.macro_D, self.Q_D = t(macro), t(Q)
        self.time_step_D = z(self.ni, self.nj)
        self.max_freq_D = z(1)
        self.residual_D = z(self.ni, self.nj, 4)
        self.bc_mdot_D = z(wl, 4)
        self.flag_D = z(2)
        self.max_dt = 0.0
        self.residual = np.full(4, 1e10)
        self.bc_mdot = 0.0
        Ls = geom["side_length"]
        self.face_lengths = [Ls[G:-G, -G, 0], Ls[-G, G:-G, 1], Ls[G:-G, G, 0], Ls[G, G:-G, 1]]

    # ------------------------------------------------------------------ init
    def initFunctions(self, restart=None):
        """ugks_block.py:258-432.  restart: this block's entry of a loaded
        checkpoint (macro, Q as saved, f or None): macro and Q are taken as
        saved (Q without conversion, as the reference loads it), and f too
        when present; otherwise f := fEQ(macro, Q) and macro, Q re-taken from
        f."""
        gs, ws = _m_tuple((self.ni, self.nj, 1), (1, 1, 1))
        init_f = True
        if restart is not None:
            self.sim.time = float(restart["time"])
            self.macro_D.copy_(self._t(restart["macro"]))
            self.Q_D.copy_(self._t(restart["Q"]))
            if restart["f"] is not None:
                self.f_D.copy_(self._t(restart["f"]))
                init_f = False
        if init_f:
            self.prg.initFunctions(self.queue, gs, ws, self.f_D, self.macro_D, self.Q_D)
            self.prg.calcMacro(self.queue, gs, ws, self.f_D, self.macro_D)
            self.prg.calcQ(self.queue, gs, ws, self.f_D, self.macro_D, self.Q_D)
        self.parametricBC(force=True)

    def _t(self, a):
        import torch
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(self.f_D.device)

    def parametricBC(self, force=False):
        if force:
            self.prg.paraBC(self.queue, (self.wall_len, 1), (1, 1), self.para_D, self.wall_prop_D,
                            float(self.sim.time))

    # ------------------------------------------------------------------ ghosts
    def updateBC(self):
        for face, bc in enumerate(self.bc_list):
            g = (self.ni, self.ghost, 1) if face in (D.NORTH, D.SOUTH) else (self.ghost, self.nj, 1)
            t = bc["type"]
            q = self.queue
            if t in (D.ADJACENT, D.PERIODIC):
                ob = self.sim.blocks[bc["other_block"]]
                self.prg.edgeExchange(q, g, None, self.f_D, self.xy_D, face, ob.f_D, ob.xy_D, ob.Ni,
                                      ob.Nj, bc["other_face"], bc.get("orientation", 1),
                                      bc.get("flip", D.NO_FLIP))
            elif t == D.EXTRAPOLATE_OUT:
                self.prg.edgeExtrapolate(q, g, None, self.f_D, face)
            elif t == D.CONSTANT:
                self.prg.edgeConstant(q, g, None, self.f_D, face, self.wall_prop_D)
            elif t == D.REFLECT:
                self.prg.edgeMirror(q, g, None, self.f_D, face)
            elif t == D.BOUNCE_BACK:
                self.prg.edgeBounceBack(q, g, None, self.f_D, face)
            elif t in (D.DIFFUSE, D.ADSORBING):
                self.prg.edgeConstGrad(q, g, None, self.f_D, face)
            elif t == D.INFLOW:
                self.prg.edgeInflow(q, g, None, self.f_D, face, self.normal_D, self.macro_D, self.Q_D,
                                    self.wall_prop_D)
            elif t == D.OUTFLOW:
                self.prg.edgeOutflow(q, g, None, self.f_D, face, self.normal_D, self.macro_D, self.Q_D,
                                     self.wall_prop_D)

    # ------------------------------------------------------------------ flags
    def get_flag(self):
        flag = self.flag_D.cpu().numpy()
        err = False
        if flag[0] in (1.0, 1.1, 1.2, 1.3):
            err = True
            print("ERROR: NaN encountered", file=sys.stderr)
        elif flag[0] in (2.0, 3.0):
            self.max_dt = min(self.max_dt, flag[1])
        elif flag[0] == 4.0:
            err = True
            print("ERROR: pressure / temperature outside adsorption isotherm data", file=sys.stderr)
        return err

    def reset_flag(self):
        self.flag_D.zero_()

    # ------------------------------------------------------------------ flux
    def wall_flux(self, bc, wall, gsize, flux, flux_macro, dt):
        q = self.queue
        if bc["type"] == D.DIFFUSE:
            self.prg.accommodatingWallDist(q, gsize, None, self.normal_D, wall, self.wall_prop_D, flux, dt)
        else:
            self.reset_flag()
            self.prg.adsorbingWall_P1(q, gsize, None, self.normal_D, wall, self.wall_prop_D,
                                      self.wall_cover_D, self.wall_dist_D, flux, self.macro_D, dt,
                                      self.flag_D)
            if self.get_flag():
                return True
            # re-emission by reflect_type (ugks_block.py:952-969; 'S' unless 'CL' or 'D')
            rtype = bc.get("reflect_type", "S")
            p2 = (self.prg.adsorbingWallCL_P2 if rtype == "CL" else
                  self.prg.adsorbingWallD_P2 if rtype == "D" else self.prg.adsorbingWallS_P2)
            p2(q, gsize, None, self.normal_D, wall, self.wall_prop_D, self.wall_cover_D, self.wall_dist_D,
               flux, self.macro_D, dt)
        self.prg.wallFlux(q, gsize, None, self.normal_D, self.length_D, wall, flux, flux_macro, dt)
        self.prg.wallMassEnergyFluxes(q, gsize, None, self.normal_D, self.length_D, self.area_D, wall,
                                      flux, self.wall_fluxes_D, dt)
        return False

    def _direction(self, d, dt):
        ni, nj, q = self.ni, self.nj, self.queue
        flux = self.flux_f_S_D if d == D.S_DIR else self.flux_f_W_D
        fm = self.flux_macro_S_D if d == D.S_DIR else self.flux_macro_W_D
        gsize = (ni, nj + 1, 1) if d == D.S_DIR else (ni + 1, nj, 1)
        self.prg.iFace(q, gsize, None, self.f_D, flux, self.sigma_D, self.centre_D, self.side_D,
                       self.normal_D, d)
        off_top = off_bot = 0
        top, bot = (D.NORTH, D.SOUTH) if d == D.S_DIR else (D.EAST, D.WEST)
        wsize = (ni, 1, 1) if d == D.S_DIR else (1, nj, 1)
        for wall, is_top in ((top, True), (bot, False)):
            bc = self.bc_list[wall]
            if bc["type"] in (D.DIFFUSE, D.ADSORBING):
                if is_top:
                    off_top = 1
                else:
                    off_bot = 1
                self.wall_flux(bc, wall, wsize, flux, fm, dt)  # error return ignored (ugks_block.py:1084)
        shrink = off_top + off_bot
        g = (ni, nj + 1 - shrink, 1) if d == D.S_DIR else (ni + 1 - shrink, nj, 1)
        self.prg.getFaceCons(q, g, None, flux, self.normal_D, d, self.prim_D, off_bot, off_top)
        self.prg.getAL(q, g, None, self.f_D, self.normal_D, d, self.aL_D, off_bot, off_top)
        self.prg.getAR(q, g, None, self.f_D, self.normal_D, d, self.aR_D, off_bot, off_top)
        self.prg.getPLR(q, g, None, self.centre_D, self.side_D, d, self.prim_D, self.aL_D, self.aR_D,
                        off_bot, off_top)
        self.prg.initMacroFlux(q, g, None, fm, d, dt, self.prim_D, self.aL_D, self.aR_D, self.aT_D,
                               self.Mxi_D, off_bot, off_top)
        self.prg.calcFaceQ(q, g, None, flux, self.prim_D, self.normal_D, self.faceQ_D, d, off_bot, off_top)
        self.prg.macroFlux(q, g, None, flux, self.sigma_D, fm, self.normal_D, self.length_D, d, dt,
                           self.prim_D, self.faceQ_D, off_bot, off_top)
        self.prg.distFlux(q, g, None, flux, self.sigma_D, self.normal_D, self.length_D, d, dt,
                          self.prim_D, self.aL_D, self.aR_D, self.aT_D, self.Mxi_D, self.faceQ_D,
                          off_bot, off_top)

    def UGKS_flux(self):
        dt = float(self.sim.dt)
        self._direction(D.S_DIR, dt)
        self._direction(D.W_DIR, dt)
        return False

    # ------------------------------------------------------------------ update
    def UGKS_update(self, get_residual=False):
        q = self.queue
        gs = (self.ni, self.nj, 1)
        self.prg.calcQ(q, gs, None, self.f_D, self.macro_D, self.Q_D)
        self.prg.updateMacro(q, (self.ni, self.nj), None, self.flux_macro_S_D, self.flux_macro_W_D,
                             self.area_D, self.macro_D, self.residual_D)
        self.reset_flag()
        self.prg.UGKS_update(q, gs, None, self.f_D, self.flux_f_S_D, self.flux_f_W_D, self.area_D,
                             self.macro_D, self.Q_D, self.residual_D, float(self.sim.dt), self.flag_D)
        if self.get_flag():
            return True
        if get_residual:
            self.get_BC_mdot()
            self.prg.getResidual(q, (self.ni, self.nj), None, self.macro_D, self.residual_D)
            sum_res = self.residual_D.sum(dim=(0, 1)).cpu().numpy()
            sum_avg = self.macro_D.abs().sum(dim=(0, 1)).cpu().numpy()
            self.residual = np.sqrt(self.ni * self.nj * sum_res) / (sum_avg + sys.float_info.min)
            self.residual[self.residual <= 0.0] = 1.0
        return False

    def get_BC_mdot(self):
        got = False
        for face, bc in enumerate(self.bc_list):
            if bc["type"] in (D.EXTRAPOLATE_OUT, D.INFLOW, D.OUTFLOW, D.CONSTANT):
                n = self.ni if face in (D.NORTH, D.SOUTH) else self.nj
                self.prg.edgeMassFlow(self.queue, (n, 1), None, self.macro_D, self.normal_D, self.length_D,
                                      self.bc_mdot_D, face)
                got = True
        self.bc_mdot = float(self.bc_mdot_D.sum().cpu()) if got else 0.0

    # ------------------------------------------------------------------ dt
    def getDT(self):
        import ctypes as C
        from . import _lib
        self.prg.clFindDT(self.queue, (self.ni, self.nj), None, self.xy_D, self.area_D, self.macro_D,
                          self.time_step_D, float(self.sim.Kn_eff))
        from .kernel_program import _stream_ptr
        _lib.check(_lib.lib().ugks_array_max(self.time_step_D.data_ptr(), self.time_step_D.numel(),
                                             self.max_freq_D.data_ptr(), _stream_ptr(self.queue)),
                   "ugks_array_max")
        self.max_dt = self.sim.CFL / float(self.max_freq_D.cpu())

    # ------------------------------------------------------------------ host views
    def block_mass(self):
        G = self.ghost
        macro = self.macro_D.cpu().numpy()
        cover = self.wall_cover_D.cpu().numpy()
        bulk = float(np.sum(self.area_H[G:-G, G:-G] * macro[:, :, 0]))
        n = [self.ni, self.nj, self.ni, self.nj]
        ads = sum(float(np.sum(cover[0:n[f], f, 0] * bc.get("S_T", 1.0) * self.face_lengths[f]))
                  for f, bc in enumerate(self.bc_list))
        return bulk, ads
