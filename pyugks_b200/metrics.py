"""Structured metrics as JSON lines.

The reference prints progress to stdout and keeps a residual history in
memory (`ugks_data.py:91-104`, `ugks_sim.py:463-488`); its only timing is a
wall clock around the run (`ugks_sim.py:171-185`, `690`).  Here every record
is one JSON object per line, so that a run can be followed or compared by
machine:

* ``solver_step`` -- per solve of a FusedSolver: completed steps, simulated
  time, dt, the four residuals, the status word, the bulk mass and its drift
  from the solve's first record, and, given the device time of the steps
  since the last record, the cell-velocity updates per second;
* ``request`` -- a served request: arrival, admission, completion, latency,
  steps, stop reason and its cell-velocity work;
* ``tick`` -- the serving loop after a tick: running solves, backlog, memory
  admitted against the budget;
* any other kind through ``write``.

Records carry the wall-clock time ``t`` and the log's fixed context (the
workload, precision, ...).
"""
from __future__ import annotations

import json
import os
import time


class MetricsLog:
    def __init__(self, path, **context):
        """Append JSON lines to `path` (a file name or an open text file)."""
        self._own = isinstance(path, (str, os.PathLike))
        self._fh = open(path, "a") if self._own else path
        self.context = dict(context)
        self._mass0 = {}
        self._last = {}

    def close(self):
        if self._own:
            self._fh.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def write(self, kind: str, **fields):
        rec = {"t": time.time(), "kind": kind}
        rec.update(self.context)
        rec.update(fields)
        self._fh.write(json.dumps(rec, default=_plain) + "\n")
        self._fh.flush()
        return rec

    # ------------------------------------------------------------ records
    def solver_step(self, solver, device_ms: float | None = None):
        """One record per solve of `solver` (synchronises).  device_ms: the
        device time of the steps taken since this log's last record of the
        same solver, for the throughput figure."""
        states = solver.solve_state()
        out = []
        for k, st in enumerate(states):
            mass = bulk_mass(solver, k)
            key = (id(solver), k)
            m0 = self._mass0.setdefault(key, mass)
            steps_before = self._last.get(key, st["steps"])
            rec = dict(solve=k, step=st["steps"], time=st["time"], dt=st["dt"], residual=st["residual"],
                       status=st["status"], mass=mass, mass_drift=(mass - m0) / m0 if m0 else 0.0)
            if device_ms and st["steps"] > steps_before:
                from .configs import workload_size
                work = workload_size(solver.cases[k]) * (st["steps"] - steps_before)
                rec["cell_vel_per_s"] = work / (device_ms / 1e3)
            self._last[key] = st["steps"]
            out.append(self.write("solver_step", **rec))
        return out

    def request(self, r):
        """A completed serving.Request."""
        return self.write("request", id=r.id, arrival=r.arrival, admitted=r.admitted, finished=r.finished,
                          latency=(r.finished - r.arrival) if r.finished is not None else None, steps=r.steps,
                          reason=r.reason, units_per_step=r.units, work=r.steps * r.units)

    def tick(self, now: float, running: int, backlog: int, used_bytes: float, budget_bytes: float, units: int):
        return self.write("tick", now=now, running=running, backlog=backlog, used_bytes=used_bytes,
                          budget_bytes=budget_bytes, units=units)


def bulk_mass(solver, solve: int = 0) -> float:
    """Sum of rho * area over the interior cells of one solve of a FusedSolver
    (on the device; one scalar comes back)."""
    total = None
    for bi in solver.solve_block_ids(solve):
        b = solver.blocks[bi]
        G = b.G
        m = (b.macro[:, :, 0] * b.area[G:-G, G:-G]).sum()
        total = m if total is None else total + m
    return float(total) if total is not None else 0.0


def read(path):
    """The records of a JSON-lines file."""
    with open(path) as fh:
        return [json.loads(line) for line in fh if line.strip()]


def _plain(x):
    try:
        import numpy as np
        if isinstance(x, np.generic):
            return x.item()
        if isinstance(x, np.ndarray):
            return x.tolist()
    except ImportError:  # pragma: no cover
        pass
    return str(x)
