"""Diagnostics of a solve: directional temperatures and stress
(getInternal), the reconstructed distribution at the walls
(UGKSBlock.get_interface_distribution) and the run loop's residual-based
stop rules (UGKSim.run / analyse_residual).
"""
from __future__ import annotations

import numpy as np

from . import defs as D
from .kernel_program import KernelProgram


def internal_data(prg: KernelProgram, f, ni: int, nj: int, queue=None):
    """getInternal (clKernel.c:314-375) of one block: per interior cell
    Txyz = (Tx, Ty, Tz, T) and stress (tau_xx, tau_xy, tau_yy), as numpy
    (what updateHost keeps when internal data is saved, ugks_block.py:1493-1508)."""
    import torch
    f64 = f if f.dtype == torch.float64 else f.double()
    txyz = torch.zeros((ni, nj, 4), dtype=torch.float64, device=f.device)
    stress = torch.zeros((ni, nj, 4), dtype=torch.float64, device=f.device)
    prg.getInternal(queue, (ni, nj, 1), None, f64.contiguous(), txyz, stress)
    return txyz.cpu().numpy(), stress.cpu().numpy()[:, :, 0:3]


def interface_distribution(prg: KernelProgram, f, centre, mid_side, normal, ni: int, nj: int, G: int,
                           queue=None):
    """get_interface_distribution (ugks_block.py:985-1047): iFace into
    scratch copies of the face arrays, then the rows of the four walls:
    {'N': [ni, Nv, 2], 'E': [nj, Nv, 2], 'S': ..., 'W': ...}."""
    import torch
    f64 = (f if f.dtype == torch.float64 else f.double()).contiguous()
    Ni, Nj = ni + 2 * G, nj + 2 * G
    face = torch.zeros_like(f64)
    sigma = torch.zeros_like(f64)
    prg.iFace(queue, (ni, nj + 1, 1), None, f64, face, sigma, centre, mid_side, normal, D.S_DIR)
    fs = face.cpu().numpy()
    out = {"N": fs[G:Ni - G, Nj - G].copy(), "S": fs[G:Ni - G, G].copy()}
    face.zero_()
    prg.iFace(queue, (ni + 1, nj, 1), None, f64, face, sigma, centre, mid_side, normal, D.W_DIR)
    fw = face.cpu().numpy()
    out["E"] = fw[Ni - G, G:Nj - G].copy()
    out["W"] = fw[G, G:Nj - G].copy()
    return out


class ResidualMonitor:
    """The residual exit rules of UGKSim.run (ugks_sim.py:604-645) with the
    slope analysis of analyse_residual (ugks_sim.py:722-811):

    * minimum residual: every component <= min_residual;
    * residual drop: from step residual_start, every component dropped by
      res_drop from its first recorded value;
    * stabilised residual: from step slope_start, the slope of the
      Butterworth-filtered log10 residual against log10 step is below
      min_slope for every component at two consecutive records.

    ``record(step, residual)`` returns the reason to stop, or None.
    """

    def __init__(self, min_residual=0.0, res_drop=np.inf, residual_start=0, slope_start=np.inf,
                 min_slope=0.0):
        self.min_residual = min_residual
        self.res_drop = res_drop
        self.residual_start = residual_start
        self.slope_start = slope_start
        self.min_slope = min_slope
        self.steps = []
        self.history = []
        self.below = 0
        self.initial = None
        self.last_slope = None

    def slopes(self, step):
        """analyse_residual's slopes (without the plots), or inf before slope_start."""
        if step < self.slope_start:
            return np.inf
        from scipy import signal
        res_x = np.log10(np.asarray(self.steps, dtype=np.float64))
        res_y = np.log10(np.asarray(self.history, dtype=np.float64))
        dx = np.min(np.diff(res_x))
        sample_x = np.arange(res_x[0], res_x[-1] + dx, dx)
        n = len(res_x)
        A, B = signal.butter(2, 1.0 / n ** 0.8, output="ba")
        out = []
        for i in range(res_y.shape[1]):
            ry = res_y[:, i]
            mask = np.isfinite(ry)
            sample_y = np.interp(sample_x, res_x[mask], ry[mask])
            filt = signal.filtfilt(A, B, sample_y)
            out.append(np.abs(np.diff(filt) / dx)[-1])
        return out

    def record(self, step: int, residual) -> str | None:
        residual = np.asarray(residual, dtype=np.float64)
        self.steps.append(step)
        self.history.append(residual)
        slope = self.slopes(step)
        self.last_slope = slope
        if step >= self.slope_start:
            self.below = self.below + 1 if np.all(np.array(slope) < self.min_slope) else 0
            if self.below >= 2:
                return "residual stabilised"
        if step >= self.residual_start:
            if self.initial is None:
                self.initial = residual
            else:
                if np.all(self.initial / residual >= self.res_drop):
                    return "residual reduction limit reached"
            if np.all(residual <= self.min_residual):
                return "minimum residual reached"
        return None
