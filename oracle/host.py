"""Oracle host sequence: Python restatement of the pyUGKS time-step driver.

TEST INFRASTRUCTURE ONLY.  Restates, over numpy arrays, the launch sequence of

* ``UGKSim.__init__`` / ``one_step`` / ``updateTimeStep`` / ``updateAllBC``
  (``ugks_sim.py:52-115, 274-321, 407-501``);
* ``UGKSBlock.initFunctions`` / ``updateBC`` / ``wall_flux`` / ``UGKS_flux`` /
  ``UGKS_update`` / ``getDT`` / ``block_mass`` (``ugks_block.py:258-432,
  621-665, 930-983, 1049-1329, 1415-1433, 1598-1623``),

driving either oracle program (``programs.RefProgram``: the reference kernels
compiled for the CPU, or ``programs.PortProgram``: the C restatement).
"""
from __future__ import annotations

import sys

import numpy as np

import programs as pg
import ugks_setup as us

NORTH, EAST, SOUTH, WEST = us.NORTH, us.EAST, us.SOUTH, us.WEST
S_DIR, W_DIR = 0, 1


class OracleBlock:
    def __init__(self, sim, bid, block, geom, prog):
        self.sim, self.id, self.spec, self.prg = sim, bid, block, prog
        c = sim.const
        self.G = G = c.ghost
        self.ni, self.nj = block["ni"], block["nj"]
        self.Ni, self.Nj = self.ni + 2 * G, self.nj + 2 * G
        self.Nv = c.Nv
        self.bc_list = block["bc"]
        self.xy = np.ascontiguousarray(geom["xy"])
        self.area = np.ascontiguousarray(geom["area"])
        self.centre = np.ascontiguousarray(geom["centre"])
        self.side = np.ascontiguousarray(geom["mid_side"])
        self.normal = np.ascontiguousarray(geom["normal"])
        self.length = np.ascontiguousarray(geom["side_length"])
        Ni, Nj, Nv = self.Ni, self.Nj, self.Nv
        z = lambda *s: np.zeros(s)
        self.f = z(Ni, Nj, Nv, 2)
        self.flux_f_S, self.flux_f_W, self.sigma = z(Ni, Nj, Nv, 2), z(Ni, Nj, Nv, 2), z(Ni, Nj, Nv, 2)
        self.flux_macro_S, self.flux_macro_W = z(Ni, Nj, 4), z(Ni, Nj, 4)
        self.prim, self.aL, self.aR, self.aT = z(Ni, Nj, 4), z(Ni, Nj, 4), z(Ni, Nj, 4), z(Ni, Nj, 4)
        self.faceQ, self.Mxi = z(Ni, Nj, 2), z(Ni, Nj, 3)
        wl = max(self.ni, self.nj)
        self.wall_len = wl
        self.wall_prop = z(wl, 4, 4)
        self.wall_cover = z(wl, 4, 4)
        for bci, bc in enumerate(self.bc_list):
            self.wall_cover[:, bci, 0] = bc.get("cover_initial", 0.0)
        self.wall_fluxes = z(wl, 4, 8)
        self.wall_dist = z(wl, Nv, 2)
        self.para = z(wl, 4, 4)
        self.macro, self.Q = us.initial_macro(block)
        self.time_step = z(self.ni, self.nj)
        self.residual_buf = z(self.ni, self.nj, 4)
        self.bc_mdot_buf = z(wl, 4)
        self.flag = z(2)
        self.max_dt = 0.0
        self.residual = np.full(4, 1e10)
        self.bc_mdot = 0.0
        self.face_lengths = [self.length[G:-G, -G, 0], self.length[-G, G:-G, 1],
                             self.length[G:-G, G, 0], self.length[G, G:-G, 1]]

    # ugks_block.py:258-432 (fresh start: equilibrium f, macro re-taken from f)
    def init_functions(self):
        g = (self.ni, self.nj)
        self.prg.initFunctions(g, self.f, self.macro, self.Q)
        self.prg.calcMacro(g, self.f, self.macro)
        self.prg.calcQ(g, self.f, self.macro, self.Q)
        self.prg.paraBC((self.wall_len, 1), self.para, self.wall_prop, float(self.sim.time))

    # ugks_block.py:274-300, 347-349, 411-432: macro and Q as saved (Q is the
    # external heat flux the file holds, loaded without conversion); f as
    # saved, or fEQ(macro, Q) with macro and Q then re-taken from f
    def init_functions_restart(self, data):
        self.sim.time = float(data["time"])
        self.macro[:] = data["macro"]
        self.Q[:] = data["Q"]
        if data["f"] is not None:
            self.f[:] = data["f"]
        else:
            g = (self.ni, self.nj)
            self.prg.initFunctions(g, self.f, self.macro, self.Q)
            self.prg.calcMacro(g, self.f, self.macro)
            self.prg.calcQ(g, self.f, self.macro, self.Q)
        self.prg.paraBC((self.wall_len, 1), self.para, self.wall_prop, float(self.sim.time))

    # the datasets save_hdf writes (ugks_block.py:1441-1595), with Q from
    # updateHost: calcQ of the current f and macro, in place, then times
    # (4 + K) / 5 (ugks_block.py:1376-1386)
    def save_data(self, with_f=True):
        self.prg.calcQ((self.ni, self.nj), self.f, self.macro, self.Q)
        return dict(macro=self.macro.copy(), Q_ext=self.Q * ((4.0 + self.sim.const.K) / 5.0),
                    wall_prop=self.wall_prop.copy(), wall_cover=self.wall_cover.copy(),
                    wall_fluxes=self.wall_fluxes.copy(), f=self.f.copy() if with_f else None)

    # getInternal (clKernel.c:314-375)
    def internal_data(self):
        txyz, stress = np.zeros((self.ni, self.nj, 4)), np.zeros((self.ni, self.nj, 4))
        self.prg.getInternal((self.ni, self.nj), self.f, txyz, stress)
        return txyz, stress[:, :, 0:3]

    # get_interface_distribution (ugks_block.py:985-1047), into scratch arrays
    def interface_distribution(self):
        G, Ni, Nj = self.G, self.Ni, self.Nj
        face, sigma = np.zeros_like(self.f), np.zeros_like(self.f)
        self.prg.iFace((self.ni, self.nj + 1), self.f, face, sigma, self.centre, self.side, self.normal, S_DIR)
        out = {"N": face[G:Ni - G, Nj - G].copy(), "S": face[G:Ni - G, G].copy()}
        face[:] = 0.0
        self.prg.iFace((self.ni + 1, self.nj), self.f, face, sigma, self.centre, self.side, self.normal, W_DIR)
        out["E"] = face[Ni - G, G:Nj - G].copy()
        out["W"] = face[G, G:Nj - G].copy()
        return out

    # ugks_block.py:621-665
    def update_bc(self):
        for face, bc in enumerate(self.bc_list):
            g = (self.ni, self.G) if face in (NORTH, SOUTH) else (self.G, self.nj)
            t = bc["type"]
            if t in (us.ADJACENT, us.PERIODIC):
                ob = self.sim.blocks[bc["other_block"]]
                self.prg.edgeExchange(g, self.f, self.xy, face, ob.f, ob.xy, ob.Ni, ob.Nj,
                                      bc["other_face"], bc.get("orientation", 1), bc.get("flip", 0))
            elif t == us.EXTRAPOLATE_OUT:
                self.prg.edgeExtrapolate(g, self.f, face)
            elif t == us.CONSTANT:
                self.prg.edgeConstant(g, self.f, face, self.wall_prop)
            elif t == us.REFLECT:
                self.prg.edgeMirror(g, self.f, face)
            elif t == us.BOUNCE_BACK:
                self.prg.edgeBounceBack(g, self.f, face)
            elif t in (us.DIFFUSE, us.ADSORBING):
                self.prg.edgeConstGrad(g, self.f, face)
            elif t == us.INFLOW:
                self.prg.edgeInflow(g, self.f, face, self.normal, self.macro, self.Q, self.wall_prop)
            elif t == us.OUTFLOW:
                self.prg.edgeOutflow(g, self.f, face, self.normal, self.macro, self.Q, self.wall_prop)

    # ugks_block.py:930-983
    def wall_flux(self, bc, wall, gsize, flux, flux_macro, dt):
        if bc["type"] == us.DIFFUSE:
            self.prg.accommodatingWallDist(gsize, self.normal, wall, self.wall_prop, flux, dt)
        else:
            self.flag[:] = 0
            self.prg.adsorbingWall_P1(gsize, self.normal, wall, self.wall_prop, self.wall_cover,
                                      self.wall_dist, flux, self.macro, dt, self.flag)
            if self.flag[0] == 4.0:
                return True
            # re-emission by reflect_type (ugks_block.py:952-969; 'S' unless 'CL' or 'D')
            rtype = bc.get("reflect_type", "S")
            p2 = (self.prg.adsorbingWallCL_P2 if rtype == "CL" else
                  self.prg.adsorbingWallD_P2 if rtype == "D" else self.prg.adsorbingWallS_P2)
            p2(gsize, self.normal, wall, self.wall_prop, self.wall_cover, self.wall_dist, flux, self.macro, dt)
        self.prg.wallFlux(gsize, self.normal, self.length, wall, flux, flux_macro, dt)
        self.prg.wallMassEnergyFluxes(gsize, self.normal, self.length, self.area, wall, flux,
                                      self.wall_fluxes, dt)
        return False

    def _direction(self, d, dt):
        ni, nj = self.ni, self.nj
        flux = self.flux_f_S if d == S_DIR else self.flux_f_W
        fm = self.flux_macro_S if d == S_DIR else self.flux_macro_W
        gsize = (ni, nj + 1) if d == S_DIR else (ni + 1, nj)
        self.prg.iFace(gsize, self.f, flux, self.sigma, self.centre, self.side, self.normal, d)
        off_top = off_bot = 0
        top, bot = (NORTH, SOUTH) if d == S_DIR else (EAST, WEST)
        wsize = (ni, 1) if d == S_DIR else (1, nj)
        for wall, which in ((top, "top"), (bot, "bot")):
            bc = self.bc_list[wall]
            if bc["type"] in (us.DIFFUSE, us.ADSORBING):
                if which == "top":
                    off_top = 1
                else:
                    off_bot = 1
                # the reference ignores the wall's error return here (ugks_block.py:1084)
                self.wall_flux(bc, wall, wsize, flux, fm, dt)
        shrink = off_top + off_bot
        g = (ni, nj + 1 - shrink) if d == S_DIR else (ni + 1 - shrink, nj)
        self.prg.getFaceCons(g, flux, self.normal, d, self.prim, off_bot, off_top)
        self.prg.getAL(g, self.f, self.normal, d, self.aL, off_bot, off_top)
        self.prg.getAR(g, self.f, self.normal, d, self.aR, off_bot, off_top)
        self.prg.getPLR(g, self.centre, self.side, d, self.prim, self.aL, self.aR, off_bot, off_top)
        self.prg.initMacroFlux(g, fm, d, dt, self.prim, self.aL, self.aR, self.aT, self.Mxi,
                               off_bot, off_top)
        self.prg.calcFaceQ(g, flux, self.prim, self.normal, self.faceQ, d, off_bot, off_top)
        self.prg.macroFlux(g, flux, self.sigma, fm, self.normal, self.length, d, dt, self.prim,
                           self.faceQ, off_bot, off_top)
        self.prg.distFlux(g, flux, self.sigma, self.normal, self.length, d, dt, self.prim,
                          self.aL, self.aR, self.aT, self.Mxi, self.faceQ, off_bot, off_top)
        return False

    # ugks_block.py:1049-1260
    def ugks_flux(self, dt):
        return self._direction(S_DIR, dt) or self._direction(W_DIR, dt)

    # ugks_block.py:1262-1329
    def ugks_update(self, dt, get_residual=False):
        g = (self.ni, self.nj)
        self.prg.calcQ(g, self.f, self.macro, self.Q)
        self.prg.updateMacro(g, self.flux_macro_S, self.flux_macro_W, self.area, self.macro,
                             self.residual_buf)
        self.flag[:] = 0
        self.prg.UGKS_update(g, self.f, self.flux_f_S, self.flux_f_W, self.area, self.macro,
                             self.Q, self.residual_buf, dt, self.flag)
        if self.flag[0] == 1.0:
            return True
        if get_residual:
            self.get_bc_mdot()
            self.prg.getResidual(g, self.macro, self.residual_buf)
            sum_res = np.sum(np.sum(self.residual_buf, axis=0), axis=0)
            sum_avg = np.sum(np.sum(np.abs(self.macro), axis=0), axis=0)
            self.residual = np.sqrt(self.ni * self.nj * sum_res) / (sum_avg + sys.float_info.min)
            self.residual[self.residual <= 0.0] = 1.0
        return False

    # ugks_block.py:889-924
    def get_bc_mdot(self):
        got = False
        for face, bc in enumerate(self.bc_list):
            if bc["type"] in (us.EXTRAPOLATE_OUT, us.INFLOW, us.OUTFLOW, us.CONSTANT):
                n = self.ni if face in (NORTH, SOUTH) else self.nj
                self.prg.edgeMassFlow((n, 1), self.macro, self.normal, self.length,
                                      self.bc_mdot_buf, face)
                got = True
        self.bc_mdot = float(np.sum(self.bc_mdot_buf)) if got else 0.0

    # ugks_block.py:1415-1433
    def get_dt(self):
        self.prg.clFindDT((self.ni, self.nj), self.xy, self.area, self.macro, self.time_step,
                          self.sim.const.Kn_eff_host)
        self.max_dt = self.sim.const.CFL / np.max(self.time_step)

    # ugks_block.py:1598-1623 (non-dimensional: reference values of 1)
    def block_mass(self):
        G = self.G
        bulk = float(np.sum(self.area[G:-G, G:-G] * self.macro[:, :, 0]))
        ads = 0.0
        n = [self.ni, self.nj, self.ni, self.nj]
        for face, bc in enumerate(self.bc_list):
            ads += float(np.sum(self.wall_cover[0:n[face], face, 0] * bc.get("S_T", 1.0) *
                                self.face_lengths[face]))
        return bulk, ads


class OracleSim:
    """``UGKSim`` restated for the time-step path."""

    def __init__(self, case: dict, backend: str = "port", threads: int | None = None,
                 restart: dict | None = None):
        """restart: a loaded checkpoint ({'final_step', 'blocks': [dt, time,
        macro, Q, f or None]}); UGKSim.restart (ugks_sim.py:824-840) sets the
        step, UGKSBlock.initFunctions (ugks_block.py:274-300) the fields."""
        self.case = case
        self.const = us.Constants(case)
        self.time = 0.0
        self.dt = 0.0
        self.step = 0 if restart is None else int(restart["final_step"])
        self.force_time = False
        geoms = us.block_geometry(case, self.const.ghost)
        self.blocks = []
        for bid, (b, g) in enumerate(zip(case["blocks"], geoms)):
            if backend == "ref":
                prog = pg.RefProgram(self.const, b, bid, threads=threads)
            elif backend == "port":
                prog = pg.PortProgram(self.const, b, bid)
            else:
                raise ValueError(backend)
            self.blocks.append(OracleBlock(self, bid, b, g, prog))
        self.is_open = any(bc["type"] in (us.EXTRAPOLATE_OUT, us.INFLOW, us.OUTFLOW, us.CONSTANT)
                           for b in case["blocks"] for bc in b["bc"])
        for k, blk in enumerate(self.blocks):
            if restart is None:
                blk.init_functions()
            else:
                blk.init_functions_restart(restart["blocks"][k])
        self.update_all_bc()
        self.calc_time_step()
        self.update_time_step(limit=False)
        bulk, ads = self.total_mass()
        self.initial_mass_total = bulk + ads
        self.global_residual = None
        self.flux_passes = 0

    def update_all_bc(self):
        for b in self.blocks:
            b.update_bc()

    def calc_time_step(self):
        for b in self.blocks:
            b.get_dt()

    # ugks_sim.py:285-311
    def update_time_step(self, limit=True):
        if self.force_time:
            return
        dt_old = self.dt
        dt_new = min(b.max_dt for b in self.blocks)
        if dt_old != dt_new:
            if (dt_new > (1.0 + self.const.delta_dt) * dt_old) and limit:
                dt_new = (1.0 + self.const.delta_dt) * dt_old
            self.dt = dt_new

    def total_mass(self):
        bulk = ads = 0.0
        for b in self.blocks:
            x, y = b.block_mass()
            bulk += x
            ads += y
        return bulk, ads

    # ugks_sim.py:407-501
    def one_step(self, get_dt=True, get_res=False):
        dt_old = 0.0
        count = 0
        while (self.dt != dt_old) and (count < 2):
            dt_old = self.dt
            for b in self.blocks:
                if b.ugks_flux(self.dt):
                    return True
            self.flux_passes += 1
            self.update_time_step()
            count += 1
        if count > 1:
            if self.step == 1:
                raise RuntimeError("Overshot on first iteration, decrease time step")
            get_dt = True
        for b in self.blocks:
            if b.ugks_update(self.dt, get_res):
                return True
        if get_dt:
            self.calc_time_step()
            self.update_time_step()
        if get_res:
            res = sum(b.residual for b in self.blocks) / len(self.blocks)
            mdot = sum(b.bc_mdot for b in self.blocks)
            if self.is_open:
                res = np.append(res, [np.nan if mdot == 0.0 else abs(mdot)])
                bulk, ads = self.total_mass()
                dm = abs((self.initial_mass_total - (bulk + ads)) / self.initial_mass_total)
                res = np.append(res, [dm if dm > 0.0 else np.nan])
            self.global_residual = res
        self.time += self.dt
        self.step += 1
        self.update_all_bc()
        return False

    def run(self, nsteps, get_res_every=0):
        for _ in range(nsteps):
            get_res = bool(get_res_every) and ((self.step + 1) % get_res_every == 0)
            if self.one_step(True, get_res):
                raise FloatingPointError("NaN flagged at step %d" % self.step)

    # ---- comparisons -----------------------------------------------------
    def fields(self):
        """Interior macroscopic fields per block: rho, U, V, T, qx, qy."""
        out = []
        for b in self.blocks:
            g = (b.ni, b.nj)
            Q = np.zeros_like(b.Q)
            b.prg.calcQ(g, b.f, b.macro, Q)
            out.append(dict(rho=b.macro[:, :, 0].copy(), U=b.macro[:, :, 1].copy(),
                            V=b.macro[:, :, 2].copy(), T=1.0 / b.macro[:, :, 3],
                            qx=Q[:, :, 0].copy(), qy=Q[:, :, 1].copy()))
        return out

    def interior_f(self):
        return [b.f[b.G:-b.G, b.G:-b.G].copy() for b in self.blocks]
