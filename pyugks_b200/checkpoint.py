"""Checkpoint files: save a solve and restart it.

pyUGKS writes one HDF5 file per saved step (``UGKSim.saveHDF5`` /
``UGKSBlock.save_hdf``, ugks_sim.py:1022-1063, ugks_block.py:1435-1595) and a
global file with ``final_step`` (ugks_sim.py:1065-1096); a restart reads the
last saved step back (``UGKSim.restart``, ugks_sim.py:824-840, and
``UGKSBlock.initFunctions``, ugks_block.py:274-300).  h5py is not available
here, so the same datasets are stored in one ``.npz`` per checkpoint, each key
being the HDF5 path of the dataset:

    final_step, Nb, Nv, K, CFL, quad, weight
    block_<id>/dt, block_<id>/time
    block_<id>/rho, block_<id>/UV, block_<id>/T       [ni, nj], [ni, nj, 2], [ni, nj]
    block_<id>/Q                                     [ni, nj, 2], external heat flux
    block_<id>/f                                     [Ni, Nj, Nv, 2], ghosts included (optional)
    block_<id>/wall/<N|E|S|W>/<rho|U|V|T|cover|reflected|adsorbed|desorbed|
                               mass_in|mass_out|mom_n_in|mom_n_out|mom_t_in|
                               mom_t_out|nrg_in|nrg_out>

Reference behaviour kept on purpose:

* ``Q`` is saved as calcQ of the current f and macro times (4 + K) / 5
  (``updateHost``, ugks_block.py:1376-1386) and is loaded back unscaled
  (ugks_block.py:281-285); it only feeds the start-up ghost cells of inflow /
  outflow boundaries and, without saved f, the start-up equilibrium;
* without ``f`` the restart starts from fEQ(macro, Q), with the macro then
  re-taken from the discrete f (ugks_block.py:288-292, 411-429);
* wall coverage is not restored: it restarts from ``cover_initial``;
* dt is recomputed from the restored macro (calcTimeStep + updateTimeStep
  without the growth limit, ugks_sim.py:85-92), and the step counter resumes at
  ``final_step``.
"""
from __future__ import annotations

import numpy as np

FACES = ("N", "E", "S", "W")
WALL_FLUX_NAMES = ("mass_in", "mass_out", "mom_n_in", "mom_n_out", "mom_t_in", "mom_t_out",
                   "nrg_in", "nrg_out")


def block_datasets(bid: int, dt: float, time: float, macro: np.ndarray, Q_ext: np.ndarray,
                   wall_prop: np.ndarray, wall_cover: np.ndarray, wall_fluxes: np.ndarray,
                   f: np.ndarray | None = None) -> dict:
    """The datasets of one block (save_hdf, ugks_block.py:1441-1595).
    macro is [ni, nj, 4] (rho, U, V, 1/T); Q_ext the external heat flux."""
    ni, nj = macro.shape[:2]
    p = "block_%d/" % bid
    out = {p + "dt": np.float64(dt), p + "time": np.float64(time),
           p + "rho": macro[:, :, 0].copy(), p + "UV": macro[:, :, 1:3].copy(),
           p + "Q": np.asarray(Q_ext, dtype=np.float64).copy(), p + "T": 1.0 / macro[:, :, 3]}
    for fid, face in enumerate(FACES):
        n = ni if face in ("N", "S") else nj
        w = p + "wall/%s/" % face
        out[w + "rho"] = wall_prop[:n, fid, 0].copy()
        out[w + "U"] = wall_prop[:n, fid, 1].copy()
        out[w + "V"] = wall_prop[:n, fid, 2].copy()
        with np.errstate(divide="ignore"):
            out[w + "T"] = 1.0 / wall_prop[:n, fid, 3]
        for k, name in enumerate(("cover", "reflected", "adsorbed", "desorbed")):
            out[w + name] = wall_cover[:n, fid, k].copy()
        for k, name in enumerate(WALL_FLUX_NAMES):
            out[w + name] = wall_fluxes[:n, fid, k].copy()
    if f is not None:
        out[p + "f"] = f
    return out


def write(path: str, final_step: int, blocks: list, meta: dict | None = None):
    """Write one checkpoint: ``blocks`` are dicts from block_datasets."""
    data = {"final_step": np.int64(final_step), "Nb": np.int64(len(blocks))}
    for k, v in (meta or {}).items():
        data[k] = np.asarray(v)
    for b in blocks:
        data.update(b)
    np.savez(path, **data)


def read(path: str) -> dict:
    """Load a checkpoint: {'final_step', 'blocks': [per block: dt, time,
    macro [ni, nj, 4], Q (as saved), f (or None)], plus the global keys}."""
    with np.load(path) as z:
        keys = set(z.files)
        out = {k: z[k] for k in keys if "/" not in k}
        out["final_step"] = int(z["final_step"])
        nb = int(z["Nb"])
        blocks = []
        for bid in range(nb):
            p = "block_%d/" % bid
            rho, UV, T = z[p + "rho"], z[p + "UV"], z[p + "T"]
            macro = np.empty(rho.shape + (4,))
            macro[:, :, 0] = rho
            macro[:, :, 1:3] = UV
            macro[:, :, 3] = 1.0 / T
            blocks.append(dict(dt=float(z[p + "dt"]), time=float(z[p + "time"]), macro=macro,
                               Q=np.array(z[p + "Q"]), f=np.array(z[p + "f"]) if p + "f" in keys else None))
        out["blocks"] = blocks
    return out


def external_heat_flux(Q_int: np.ndarray, K: float) -> np.ndarray:
    """Internal to external heat flux as updateHost writes it
    (ugks_block.py:1386)."""
    return Q_int * ((4.0 + K) / 5.0)
