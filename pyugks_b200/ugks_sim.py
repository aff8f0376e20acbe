"""UGKSim: the time loop over the blocks of one simulation.

Python-3 restatement of pyUGKS's ``UGKSim`` (``ugks_sim.py:30-1300``) for the
time-step path: start-up (``__init__``, ``ugks_sim.py:52-115``), dt control
(``calcTimeStep`` / ``updateTimeStep``, ``274-311``), ghost update
(``updateAllBC``, ``313-321``), one step (``one_step``, ``407-501``) and the
run loop's residual and NaN exits (``run``, ``503-710``).  Each step issues the
reference's per-kernel launch sequence through ``KernelProgram``; for the
fused single-launch-per-phase step of many blocks and solves at once use
``pyugks_b200.fused.FusedSolver``.
"""
from __future__ import annotations

import numpy as np

from . import checkpoint
from . import defs as D
from .desc import VelocityTables
from .problem import Constants, geometry
from .ugks_block import UGKSBlock


class UGKSim:
    def __init__(self, case: dict, device="cuda", queue=None, restart=None, device_geometry=False):
        """restart: checkpoint path (or the dict of checkpoint.read) to resume
        from, as the reference's ``gdata.restart`` (``restart``,
        ugks_sim.py:824-840).  device_geometry: build the block geometry with
        the xyExchange / xyExtrapolate / cellGeom kernels on the device, as the
        reference's initGeom does, instead of on the host."""
        import torch
        self.case = case
        self.const = Constants(case)
        self.device = torch.device(device)
        self.queue = queue
        self.CFL = float(case["CFL"])
        self.delta_dt = float(case.get("delta_dt", 1.0))
        self.Kn_eff = float(case["Kn_eff"])
        self.dt = 0.0
        self.time = 0.0
        if restart is not None and not isinstance(restart, dict):
            restart = checkpoint.read(restart)
        self.step = 0 if restart is None else int(restart["final_step"])
        self.force_time = False
        self.tabs = VelocityTables(self.const, self.device)
        if device_geometry:
            from .geometry import device_geometry as _dg
            geoms = _dg(case, device, queue)
        else:
            geoms = geometry(case, self.const.ghost)
        self.blocks = [UGKSBlock(self, k, b, g, self.tabs, self.device, queue)
                       for k, (b, g) in enumerate(zip(case["blocks"], geoms))]
        self.is_open = any(bc["type"] in (D.EXTRAPOLATE_OUT, D.INFLOW, D.OUTFLOW, D.CONSTANT)
                           for b in case["blocks"] for bc in b["bc"])
        for k, b in enumerate(self.blocks):
            b.initFunctions(None if restart is None else restart["blocks"][k])
        self.updateAllBC()
        self.calcTimeStep()
        self.updateTimeStep(limit=False)
        bulk, ads = self.total_mass()
        self.initial_mass_total = bulk + ads
        self.global_residual = None

    def updateAllBC(self):
        for b in self.blocks:
            b.updateBC()

    def calcTimeStep(self):
        for b in self.blocks:
            b.getDT()

    def updateTimeStep(self, limit=True):
        if self.force_time:
            return
        dt_old = self.dt
        dt_new = min(b.max_dt for b in self.blocks)
        if dt_old != dt_new:
            if (dt_new > (1.0 + self.delta_dt) * dt_old) and limit:
                dt_new = (1.0 + self.delta_dt) * dt_old
            self.dt = dt_new

    def total_mass(self):
        bulk = ads = 0.0
        for b in self.blocks:
            x, y = b.block_mass()
            bulk += x
            ads += y
        return bulk, ads

    def one_step(self, get_dt=True, get_res=False):
        """ugks_sim.py:407-501.  Returns True when a block flagged an error."""
        dt_old = 0.0
        count = 0
        while (self.dt != dt_old) and (count < 2):
            dt_old = self.dt
            for b in self.blocks:
                if b.UGKS_flux():
                    return True
            self.updateTimeStep()
            count += 1
        if count > 1:
            if self.step == 1:
                raise RuntimeError("Overshot on first iteration, decrease time step")
            get_dt = True
        for b in self.blocks:
            if b.UGKS_update(get_res):
                return True
        if get_dt:
            self.calcTimeStep()
            self.updateTimeStep()
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
        self.updateAllBC()
        return False

    def run(self, max_step: int, residual_count: int = 0, min_residual: float = 0.0, res_drop: float = np.inf,
            residual_start: int = 0, slope_start: float = np.inf, min_slope: float = 0.0,
            max_time: float = np.inf):
        """The run loop of UGKSim.run (ugks_sim.py:503-710) without its I/O:
        step until max_step, a NaN, max_time, or one of the residual exits of
        diagnostics.ResidualMonitor when residual_count > 0 (a residual every
        residual_count steps).  The last step is shortened to land on
        max_time, as the reference does.  Returns the reason it stopped; the
        residual history is kept in self.monitor."""
        from .diagnostics import ResidualMonitor
        self.monitor = ResidualMonitor(min_residual, res_drop, residual_start, slope_start, min_slope)
        while self.step < max_step:
            get_res = residual_count > 0 and ((self.step + 1) % residual_count == 0)
            if self.one_step(True, get_res):
                return "nan"
            if self.time >= max_time:
                return "time limit reached"
            if get_res:
                why = self.monitor.record(self.step, self.global_residual)
                if why:
                    return why
            if (max_time - self.time) < self.dt:
                self.dt = max_time - self.time
                self.force_time = True
        return "max_step"

    # ------------------------------------------------------------------ host views
    def fields(self):
        """Interior rho, U, V, T, qx, qy per block (Q re-taken from f)."""
        out = []
        for b in self.blocks:
            import torch
            Q = torch.zeros_like(b.Q_D)
            b.prg.calcQ(self.queue, (b.ni, b.nj, 1), None, b.f_D, b.macro_D, Q)
            m = b.macro_D.cpu().numpy()
            q = Q.cpu().numpy()
            out.append(dict(rho=m[:, :, 0], U=m[:, :, 1], V=m[:, :, 2], T=1.0 / m[:, :, 3],
                            qx=q[:, :, 0], qy=q[:, :, 1]))
        return out

    def internal_data(self):
        """Per block (Txyz [ni, nj, 4], stress [ni, nj, 3]) from getInternal."""
        from .diagnostics import internal_data
        return [internal_data(b.prg, b.f_D, b.ni, b.nj, self.queue) for b in self.blocks]

    def interface_distribution(self):
        """Per block the reconstructed distribution at its four walls
        (get_interface_distribution, ugks_block.py:985-1047)."""
        from .diagnostics import interface_distribution
        return [interface_distribution(b.prg, b.f_D, b.centre_D, b.side_D, b.normal_D, b.ni, b.nj, b.ghost,
                                       self.queue) for b in self.blocks]

    def save_checkpoint(self, path: str, save_f: bool = True):
        """saveHDF5 + close_HDF5 (ugks_sim.py:1022-1096) into one .npz:
        per block the fields with Q re-taken from f as updateHost does
        (ugks_block.py:1376-1386), wall data and optionally f."""
        import torch
        blocks = []
        for k, b in enumerate(self.blocks):
            b.prg.calcQ(self.queue, (b.ni, b.nj, 1), None, b.f_D, b.macro_D, b.Q_D)
            q = b.Q_D.cpu().numpy()
            blocks.append(checkpoint.block_datasets(
                k, self.dt, self.time, b.macro_D.cpu().numpy(), checkpoint.external_heat_flux(q, self.const.K),
                b.wall_prop_D.cpu().numpy(), b.wall_cover_D.cpu().numpy(), b.wall_fluxes_D.cpu().numpy(),
                b.f_D.cpu().numpy() if save_f else None))
        meta = dict(Nv=self.const.Nv, K=self.const.K, CFL=self.CFL, quad=self.const.vgrid.quad,
                    weight=self.const.vgrid.weight)
        checkpoint.write(path, self.step, blocks, meta)

    def interior_f(self):
        return [b.f_D[b.ghost:-b.ghost, b.ghost:-b.ghost].cpu().numpy() for b in self.blocks]
