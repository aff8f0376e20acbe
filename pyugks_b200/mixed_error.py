"""Error of the mixed-precision step against the plain FP64 step.

Runs the same solves with f and the face fluxes stored in FP64 and in FP32
(moments, conserved update, relaxation and dt stay FP64 in both) and reports,
per solve, the relative L2 and Linf errors of density, velocity, temperature
and heat flux (velocity and heat flux as 2-vectors):

    L2   = ||a - b||_2 / ||b||_2        over all interior cells of the solve
    Linf = max |a - b| / max |b|

    python -m pyugks_b200.mixed_error --workload multiblock --steps 200
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def _stack(fields, key):
    return np.concatenate([np.ravel(f[key]) for f in fields])


def errors(fa, fb):
    """fa: mixed, fb: FP64 -- lists of per-block field dicts of one solve."""
    out = {}
    for name, keys in (("rho", ("rho",)), ("T", ("T",)), ("UV", ("U", "V")), ("q", ("qx", "qy"))):
        a = np.stack([_stack(fa, k) for k in keys], -1)
        b = np.stack([_stack(fb, k) for k in keys], -1)
        d = np.linalg.norm(a - b, axis=-1)
        nb = np.linalg.norm(b, axis=-1)
        out[name] = {"L2": float(np.sqrt(np.sum(d * d)) / max(np.sqrt(np.sum(nb * nb)), 1e-300)),
                     "Linf": float(np.max(d) / max(np.max(nb), 1e-300))}
    return out


def compare(cases, steps, device="cuda"):
    from .fused import FusedSolver
    hi = FusedSolver(cases, precision="fp64", device=device)
    lo = FusedSolver(cases, precision="mixed", device=device)
    hi.step(steps)
    lo.step(steps)
    return [errors(lo.fields(k), hi.fields(k)) for k in range(len(cases))]


def main():
    import sys
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bench import workload
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="multiblock")
    ap.add_argument("--steps", type=int, default=200)
    args = ap.parse_args()
    cases, desc = workload(args.workload)
    res = compare(cases, args.steps)
    worst = {k: {m: max(r[k][m] for r in res) for m in ("L2", "Linf")} for k in res[0]}
    print(json.dumps({"workload": desc, "steps": args.steps, "solves": len(res), "worst": worst}))


if __name__ == "__main__":
    main()
