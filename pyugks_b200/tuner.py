"""Launch-shape autotuner for the fused step.

The reference tunes its OpenCL launch sizes at start-up: ``set_opt_list``
builds the candidate work-group sizes and ``run_optimisation`` times a few
steps with each, rejects outliers and keeps the fastest
(``ugks_sim.py:128-169, 336-405``).  Here the candidates are the launch shapes
compiled into the library:

* the face pass runs one launch per *segment* (a run of blocks with one flux
  method and one velocity grid, ``ugks_fused_layout``), and each segment can
  use any of four shapes, threads per face CTA x CTAs per SM
  (``ugks_fused_sizes.seg_variant`` 1..4, ``ugks_fused.cu`` FaceShape);
* the cell pass runs with 2 or 3 CTAs of 8 warps per SM (``cell_variant``).

``tune`` times the candidates on a scratch copy of a solver's table (so the
solver itself does not advance), one segment at a time with the others
fixed, taking the median of a few repeats; the cell pass last.  The choice is
cached per (GPU, precision, flux method, velocity count, library version) in a
JSON file (``$UGKS_TUNE_CACHE``, else ``~/.cache/pyugks_b200/launch_shapes.json``)
written under a file lock, so later solvers of the same kind take it without
timing.  A shape changes only the order of per-face sums: results agree to
round-off across shapes.
"""
from __future__ import annotations

import ctypes as C
import fcntl
import json
import os
import statistics
import threading

from . import _lib

_LOCK = threading.Lock()
FACE_SHAPES = (1, 2, 3, 4)
CELL_SHAPES = (2, 3)


def cache_path() -> str:
    return os.environ.get("UGKS_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "pyugks_b200", "launch_shapes.json"))


def _gpu_name(device) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def face_key(gpu: str, precision: str, method: int, nv: int) -> str:
    return "%s|%s|%s|face|m%d|nv%d" % (gpu, _lib.lib().ugks_version().decode(), precision, method, nv)


def cell_key(gpu: str, precision: str, max_nv: int) -> str:
    return "%s|%s|%s|cell|nv%d" % (gpu, _lib.lib().ugks_version().decode(), precision, max_nv)


def load_cache(path: str | None = None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as fh:
            fcntl.flock(fh, fcntl.LOCK_SH)
            try:
                return json.load(fh)
            finally:
                fcntl.flock(fh, fcntl.LOCK_UN)
    except (OSError, ValueError):
        return {}


def update_cache(entries: dict, path: str | None = None) -> dict:
    """Merge entries into the cache file under an exclusive lock (a sibling
    lock file, so that readers never see a half-written file) and return the
    merged cache."""
    path = path or cache_path()
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with _LOCK, open(path + ".lock", "w") as lk:
        fcntl.flock(lk, fcntl.LOCK_EX)
        try:
            cache = load_cache(path)
            cache.update(entries)
            tmp = "%s.%d.tmp" % (path, os.getpid())
            with open(tmp, "w") as fh:
                json.dump(cache, fh, indent=1, sort_keys=True)
            os.replace(tmp, path)
            return cache
        finally:
            fcntl.flock(lk, fcntl.LOCK_UN)


def segments(sizes):
    """(index, flux method, velocity count) of every face-pass segment."""
    return [(k, sizes.seg_method[k], sizes.seg_max_nv[k]) for k in range(sizes.n_segments)
            if sizes.seg_count[k] > 0]


def apply(solver, choices: dict):
    """Set the solver's launch shapes from {"face": {k: variant}, "cell": variant}."""
    for k, v in choices.get("face", {}).items():
        solver.sizes.seg_variant[int(k)] = int(v)
    solver.sizes.cell_variant = int(choices.get("cell", 0))


def cached_choices(solver, cache: dict | None = None):
    """The cached shapes for every segment of this solver, or None when any
    is missing."""
    cache = load_cache() if cache is None else cache
    gpu = _gpu_name(solver.device)
    face = {}
    for k, m, nv in segments(solver.sizes):
        v = cache.get(face_key(gpu, solver.precision, m, nv))
        if v is None:
            return None
        face[k] = v
    cell = cache.get(cell_key(gpu, solver.precision, solver.sizes.max_nv))
    if cell is None:
        return None
    return {"face": face, "cell": cell}


def _time_phase(solver, phase, steps, repeats):
    """Median over repeats of the mean device time of one phase of the step
    (0: face pass, 1: cell pass), from the step's own phase events."""
    import torch
    L = solver.lib
    mixed = 0 if solver.precision == "fp64" else 1
    stream = torch.cuda.current_stream(solver.device)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(8)] for _ in range(steps)]
    for row in ev:
        for e in row:
            e.record(stream)
    torch.cuda.synchronize(solver.device)
    handles = [(_lib.vp * 8)(*[e.cuda_event for e in row]) for row in ev]
    out = []
    for _ in range(repeats):
        for k in range(steps):
            _lib.check(L.ugks_step_profiled(mixed, solver.table.data_ptr(), solver.nblocks, C.byref(solver.sizes),
                                            solver.solves.data_ptr(), solver.nsolves, handles[k],
                                            stream.cuda_stream), "ugks_step_profiled")
        torch.cuda.synchronize(solver.device)
        a, b = (0, 1) if phase == 0 else (4, 5)
        out.append(statistics.mean(ev[k][a].elapsed_time(ev[k][b]) for k in range(steps)))
    return statistics.median(out)


def tune(solver, steps: int = 3, repeats: int = 3, use_cache: bool = True, write_cache: bool = True):
    """Pick the launch shapes for `solver` (a FusedSolver) and apply them.
    Returns {"face": {segment: variant}, "cell": variant, "timed": bool,
    "times_ms": {...}}; with use_cache and every key cached, nothing is timed."""
    from .fused import FusedSolver
    gpu = _gpu_name(solver.device)
    if use_cache:
        got = cached_choices(solver)
        if got is not None:
            apply(solver, got)
            return dict(got, timed=False, times_ms={})
    scratch = FusedSolver(solver.cases, precision=solver.precision, device=solver.device)
    scratch.step(1)  # sets the kernel attributes; a first step for warm caches
    times = {}
    face = {}
    for k, m, nv in segments(scratch.sizes):
        best, best_t = None, None
        for v in FACE_SHAPES:
            scratch.sizes.seg_variant[k] = v
            t = _time_phase(scratch, 0, steps, repeats)
            times["face%d_v%d" % (k, v)] = t
            if best_t is None or t < best_t:
                best, best_t = v, t
        scratch.sizes.seg_variant[k] = best
        face[k] = best
    cell, cell_t = None, None
    for v in CELL_SHAPES:
        scratch.sizes.cell_variant = v
        t = _time_phase(scratch, 1, steps, repeats)
        times["cell_v%d" % v] = t
        if cell_t is None or t < cell_t:
            cell, cell_t = v, t
    del scratch
    choices = {"face": face, "cell": cell}
    if write_cache:
        entries = {face_key(gpu, solver.precision, m, nv): face[k] for k, m, nv in segments(solver.sizes)}
        entries[cell_key(gpu, solver.precision, solver.sizes.max_nv)] = cell
        update_cache(entries)
    apply(solver, choices)
    return dict(choices, timed=True, times_ms=times)
