#!/usr/bin/env python
"""Benchmark of the UGKS time step: cell-velocity updates per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|mixed] [--workload multiblock|cavity|channel|batched]

Prints one JSON line.  A step is one ``UGKSim.one_step`` over every block of
the workload; the metric counts interior cell x velocity points updated per
second (ghost cells not counted).

Default workload: the 128x128 lid-driven cavity in 2x2 blocks of 64x64 cells,
33x33 = 1089 velocities on [-5,5]^2, WENO5, Kn 0.01, plain FP64 — 17.8 M
cell-velocity points per step.  Its f and face-flux arrays (about 1 GB in FP64)
are far larger than the 126 MB L2, so no flush is needed between steps.

``--impl ours`` (default): the fused CUDA step on each GPU.  ``value`` is
device time with the state resident in HBM (CUDA events on the launch stream);
``e2e`` goes through the same public call with host buffers: the initial state
is copied from pinned host memory inside the timed region, each step's solve
record (dt, time, status) is copied back asynchronously, and the final
macroscopic fields are read back.  ``roofline`` times the dominant kernels
(the face pass) live with two events around them in every timed step; the
other phases' times come from a second pass of as many steps with an event
between every phase, run after the timed region (events between all the
phases cost the timed step about 20 us).

``--impl reference``: the reference's own kernels compiled for the CPU
(oracle/_ref, OpenMP over the host cores) driven by the reference's step
sequence, on the same workload; rank 0 only.

Several GPUs (torchrun): the path has no data exchange between independent
solves, so every rank runs its own replica (weak scaling); the reported time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from pyugks_b200 import configs  # noqa: E402

METRIC = "cell-velocity updates/s"
UNIT = "cell*velocity/s"
BYTES_PER_UPDATE = {"fp64": 32, "mixed": 16}  # read + write of (h, b) per cell-velocity


def workload(name: str):
    if name == "multiblock":
        case = configs.cavity_multiblock(nb=2, n=64, m=32, vlim=5.0, flux_method="WENO5", Kn=0.01,
                                         CFL=configs.WORKLOAD_CFL)
        desc = ("lid-driven cavity 128x128 as 2x2 blocks of 64x64 cells, 33x33 velocities on "
                "[-5,5]^2 (Nv=1089), WENO5, Kn 0.01, CFL 0.2")
        return [case], desc
    if name == "cavity":
        case = configs.cavity(n=32, m=24, vlim=4.0)
        return [case], "lid-driven cavity 32x32, 25x25 velocities on [-4,4]^2 (Nv=625), vanLeer, Kn 0.075"
    if name == "channel":
        case = configs.channel(nblocks=4, n=64, m=32, Kn=0.05, CFL=configs.WORKLOAD_CFL)
        return [case], ("adsorbing channel 256x64 in 4 blocks, 33x33 velocities on [-5,5]^2, WENO5, "
                        "Kn 0.05, inlet rho 1.2 / outlet rho 1.0, CFL 0.2")
    if name == "batched":
        cases = configs.batched_cavities(64, seed=1)
        return cases, "64 independent cavities, n in {24..128}, m in {16..48}, seed 1"
    raise ValueError(name)


def units_per_step(cases) -> int:
    return sum(configs.workload_size(c) for c in cases)


# ---------------------------------------------------------------------------
def sample_clocks(stop_file, out_file):
    cmd = ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
           "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
           "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
           "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"]
    try:
        return subprocess.Popen(cmd, stdout=open(out_file, "w"), stderr=subprocess.DEVNULL)
    except (FileNotFoundError, OSError):
        return None


def parse_clocks(path, gpu_index):
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        with open(path) as fh:
            for line in fh:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9 or p[0] != str(gpu_index):
                    continue
                try:
                    sm.append(float(p[1]))
                    mx = float(p[2])
                except ValueError:
                    continue
                for nm, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
    except OSError:
        pass
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
            "reasons": sorted(reasons), "samples": len(sm)}


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def read_traffic(kernel: str, workload_name: str, precision: str):
    """DRAM bytes per launch recorded from an ncu capture in profiles/."""
    path = os.path.join(ROOT, "profiles", "%s_%s_%s.md" % (kernel, workload_name, precision))
    try:
        with open(path) as fh:
            for line in fh:
                if line.startswith("traffic_bytes_per_launch:"):
                    return int(float(line.split(":", 1)[1]))
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
def cpu_reference(cases, steps, warmup, threads=None, time_budget=None):
    """Time the reference kernels compiled for the CPU (or the C restatement
    if they are unavailable) on the workload.  Returns (units/s, kind, cores,
    steps timed)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import host  # the checker / CPU baseline only
    import programs
    import ugks_setup
    threads = threads or os.cpu_count()
    kind = "reference"
    for case in cases:
        c = ugks_setup.Constants(case)
        if not all(programs.reference_available(c, b, k) for k, b in enumerate(case["blocks"])):
            kind = "port"
    sims = [host.OracleSim(case, "ref" if kind == "reference" else "port", threads=threads)
            for case in cases]
    for _ in range(warmup):
        for s in sims:
            s.one_step()
    t0 = time.perf_counter()
    done = 0
    for _ in range(steps):
        for s in sims:
            s.one_step()
        done += 1
        if time_budget and time.perf_counter() - t0 > time_budget:
            break
    el = time.perf_counter() - t0
    return units_per_step(cases) * done / el, kind, (threads if kind == "reference" else 1), done


def run_reference(args, rank, world):
    if rank != 0:
        return
    cases, desc = workload(args.workload)
    val, kind, cores, done = cpu_reference(cases, args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": done, "warmup": args.warmup, "ms_per_step": units_per_step(cases) / val * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": desc, "precision": "fp64", "units_per_step": units_per_step(cases)},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": "%d full steps of the workload after %d warm-up steps" % (done, args.warmup)},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_ours(args, rank, world, dist):
    import torch
    from pyugks_b200 import _lib
    from pyugks_b200.fused import FusedSolver

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cases, desc = workload(args.workload)
    units = units_per_step(cases)
    stream = torch.cuda.Stream(dev)
    with torch.cuda.stream(stream):
        solver = FusedSolver(cases, precision=args.precision, device=dev, stream=stream)
        L = solver.lib
        mixed = 1 if args.precision == "mixed" else 0
        # warm-up
        solver.step(args.warmup)
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        # ---- device-resident timing: the face pass (the dominant kernels)
        # bracketed by events in every timed step; the other phases in a
        # second, profiled pass of as many steps after the timed region (every
        # event recorded between launches costs the stream a few microseconds)
        def make_events(n):
            rows = [[torch.cuda.Event(enable_timing=True) for _ in range(n)] for _ in range(args.steps)]
            for row in rows:  # torch creates the CUDA event at its first record
                for e in row:
                    e.record(stream)
            return rows
        evs = make_events(2)
        pevs = make_events(8)
        torch.cuda.synchronize(dev)
        handles = [(_lib.vp * 8)(row[0].cuda_event, row[1].cuda_event) for row in evs]
        phandles = [(_lib.vp * 8)(*[e.cuda_event for e in row]) for row in pevs]
        clock_file = os.path.join("/tmp", "ugks_clocks_%d_%d.csv" % (os.getpid(), rank))
        smi = sample_clocks(None, clock_file)
        time.sleep(0.3)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        start.record(stream)
        for k in range(args.steps):
            _lib.check(L.ugks_step_profiled(mixed, solver.table.data_ptr(), solver.nblocks,
                                            C.byref(solver.sizes), solver.solves.data_ptr(),
                                            solver.nsolves, handles[k], stream.cuda_stream),
                       "ugks_step_profiled")
        end.record(stream)
        torch.cuda.synchronize(dev)
        if smi is not None:
            smi.terminate()
            smi.wait()
        ms = start.elapsed_time(end)
        face = [evs[k][0].elapsed_time(evs[k][1]) for k in range(args.steps)]
        for k in range(args.steps):
            _lib.check(L.ugks_step_profiled(mixed, solver.table.data_ptr(), solver.nblocks,
                                            C.byref(solver.sizes), solver.solves.data_ptr(),
                                            solver.nsolves, phandles[k], stream.cuda_stream),
                       "ugks_step_profiled")
        torch.cuda.synchronize(dev)
        retry = [pevs[k][2].elapsed_time(pevs[k][3]) for k in range(args.steps)]
        cell = [pevs[k][4].elapsed_time(pevs[k][5]) for k in range(args.steps)]
        ghost = [pevs[k][6].elapsed_time(pevs[k][7]) for k in range(args.steps)]
        face_profiled = [pevs[k][0].elapsed_time(pevs[k][1]) for k in range(args.steps)]
        state = solver.solve_state()
        if any(s["status"] != 0 for s in state):
            raise RuntimeError("solver status %s" % [s["status"] for s in state])
        # ---- end to end through the public call with host buffers
        e2e = run_e2e(solver, args, stream, dev, units)
    t_max, e2e_ms = max_over_ranks([ms, e2e["ms"]], dist, dev)
    if rank != 0:
        return
    value = job_throughput(units, args.steps, world, t_max)
    kernels = {"face_pass": statistics.mean(face), "cell_pass": statistics.mean(cell),
               "ghost_pass": statistics.mean(ghost), "retry_face_pass": statistics.mean(retry),
               "face_pass_profiled": statistics.mean(face_profiled),
               "source": "face_pass: the timed steps (2 events each); the rest: %d profiled steps "
                         "after them (8 events each)" % args.steps}
    dom = max(("face_pass", "cell_pass"), key=lambda k: kernels[k])
    peak, peak_kind = read_peaks()
    bpu = BYTES_PER_UPDATE[args.precision]
    achieved = bpu * units / (kernels[dom] / 1e3) / 1e9
    clocks = parse_clocks(clock_file, local)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        # mixed: FP32 per-velocity face fluxes, FP64 sums, cell update and relaxation
        "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
        "config": {"workload": desc, "precision": args.precision, "units_per_step": units,
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "working set > 126 MB L2 (f and face fluxes %.2f GB), no flush"
                         % (solver_bytes(solver) / 1e9)},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": read_traffic(dom, args.workload, args.precision),
                     "bytes_per_unit": bpu, "kernel_ms": kernels,
                     "step_frac": bpu * units / (t_max / args.steps / 1e3) / 1e9 / peak},
        "e2e": {"value": job_throughput(units, args.steps, world, e2e_ms), "unit": UNIT,
                "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]},
        "gpu_launches": solver.launches_per_step() * args.steps,
        "clocks": clocks,
    }
    if world == 1 and args.workload == "multiblock" and args.precision == "fp64" and not args.no_comparisons:
        # the comparison records: batched mixed precision and serving
        # against the plain FP64 method, measured in the same run
        for key, fn in (("batched_mixed", batched_record), ("serving", serving_record)):
            try:
                line[key] = fn()
            except Exception as exc:  # the main line is printed regardless
                line[key] = {"error": "%s: %s" % (type(exc).__name__, exc)}
    if world == 1 and not args.no_cpu_baseline:
        budget = float(os.environ.get("UGKS_CPU_BASELINE_SECONDS", "20"))
        val, kind, cores, done = cpu_reference(cases, steps=50, warmup=1, time_budget=budget)
        line["cpu_baseline"] = {"value": val, "unit": UNIT, "cores": cores, "kind": kind,
                                "sample": "%d full steps of the workload (time budget %.0f s) after 1 warm-up"
                                          % (done, budget)}
    if args.metrics:
        from pyugks_b200.metrics import MetricsLog
        with MetricsLog(args.metrics, workload=args.workload, precision=args.precision) as log:
            log.write("bench", **line)
    print(json.dumps(line), flush=True)


def max_over_ranks(values, dist, device=None):
    """Max over all ranks of a few local timings (each rank times its own
    replica; the job's time is the slowest rank's)."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def job_throughput(units_per_step, steps, world, t_max_ms):
    """Whole-job cell-velocity updates per second: every rank advances its own
    replica of the workload by `steps` steps in at most t_max_ms."""
    return world * units_per_step * steps / (t_max_ms / 1e3)


def solver_bytes(solver):
    return sum(b.f.numel() * b.f.element_size() * 3 for b in solver.blocks)


def run_e2e(solver, args, stream, dev, units):
    """Host-buffer run: initial state H2D (pinned) + K steps with an async D2H
    of each step's solve record + final D2H of the macroscopic fields."""
    import torch
    host_state = [(b.f.detach().cpu().pin_memory(), b.macro.detach().cpu().pin_memory(),
                   b.Q.detach().cpu().pin_memory()) for b in solver.blocks]
    rec = torch.empty((args.steps, solver.solves.numel()), dtype=torch.uint8).pin_memory()
    fields = [torch.empty_like(b.macro, device="cpu").pin_memory() for b in solver.blocks]
    h2d = sum(x.numel() * x.element_size() for t in host_state for x in t)
    torch.cuda.synchronize(dev)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for b, (f, m, q) in zip(solver.blocks, host_state):
        b.f.copy_(f, non_blocking=True)
        b.macro.copy_(m, non_blocking=True)
        b.Q.copy_(q, non_blocking=True)
    for k in range(args.steps):
        solver.step(1)
        rec[k].copy_(solver.solves, non_blocking=True)
    for b, out in zip(solver.blocks, fields):
        out.copy_(b.macro, non_blocking=True)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    d2h = rec.numel() + sum(x.numel() * x.element_size() for x in fields)
    return {"ms": t0.elapsed_time(t1), "h2d": h2d // args.steps, "d2h": d2h // args.steps}


def batched_record(steps=10, warmup=3):
    """Config 3 (64 independent cavities, seed 1) in one block table, mixed and
    FP64: device-timed throughput of each, and the mixed fields' error against
    the FP64 fields after the same steps (relative L2 / Linf per solve; the
    worst over the 64 solves)."""
    import torch
    from pyugks_b200.fused import FusedSolver
    from pyugks_b200.mixed_error import errors
    cases, desc = workload("batched")
    units = units_per_step(cases)
    out = {"workload": desc, "units_per_step": units, "steps": steps, "warmup": warmup}
    solvers = {}
    out["launch_shapes"] = "tuned for both arms (pyugks_b200.tuner, before the timed steps)"
    for prec in ("mixed", "fp64"):
        s = FusedSolver(cases, precision=prec, tune=True)
        s.step(warmup)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        s.step(steps)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        out[prec] = {"value": units * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
                     "gpu_launches": s.launches_per_step() * steps}
        solvers[prec] = s
    out["ratio_mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    worst = {}
    for k in range(len(cases)):
        e = errors(solvers["mixed"].fields(k), solvers["fp64"].fields(k))
        for name, v in e.items():
            w = worst.setdefault(name, {"L2": 0.0, "Linf": 0.0})
            w["L2"], w["Linf"] = max(w["L2"], v["L2"]), max(w["Linf"], v["Linf"])
    out["mixed_vs_fp64_error"] = {"after_steps": warmup + steps, "worst_over_solves": worst}
    return out


def serving_record(arrival_seconds=2.0, max_steps=2000, tol=1e-6, steps_per_tick=50, metrics=None):
    """A bounded config-5 stream: Poisson arrivals at 20/s (seed 2) over
    arrival_seconds, 70% cavities / 30% adsorbing channels with config 5's
    size and parameter distributions, each run until its density residual is
    below tol or max_steps steps.  Served by continuous batching in mixed
    precision, and by the plain FP64 fused step one solve at a time to the
    same stop rule (first come, first served)."""
    from pyugks_b200.serving import Server, request_stream, serve_one_at_a_time
    reqs = request_stream(seed=2, rate=20.0, duration=arrival_seconds, max_steps=max_steps, tol=tol)
    server = Server(budget_bytes=150e9, precision="mixed", steps_per_tick=steps_per_tick)
    done = server.run(reqs, metrics=metrics)
    lat = np.array([r.finished - r.arrival for r in done])
    batched = {"value": server.units / server.wall, "unit": UNIT, "wall_s": server.wall,
               "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
               "completed": len(done), "converged": sum(r.reason == "converged" for r in done),
               "step_limit": sum(r.reason == "max_steps" for r in done),
               "errors": sum(r.reason == "error" for r in done)}
    arm = serve_one_at_a_time(request_stream(seed=2, rate=20.0, duration=arrival_seconds, max_steps=max_steps,
                                             tol=tol), precision="fp64", steps_per_tick=steps_per_tick)
    la = np.array(arm["latency"])
    fp64 = {"value": arm["value"], "unit": UNIT, "makespan_s": arm["makespan_s"],
            "p50_s": float(np.percentile(la, 50)), "p99_s": float(np.percentile(la, 99)),
            "converged": sum(x == "converged" for x in arm["reasons"]),
            "step_limit": sum(x == "max_steps" for x in arm["reasons"]),
            "errors": sum(x == "error" for x in arm["reasons"])}
    return {"stream": "%d requests: Poisson 20/s over %.1f s (seed 2), stop at density residual < %g or %d steps"
                      % (len(reqs), arrival_seconds, tol, max_steps),
            "arrivals": len(reqs), "admitted": len(done), "backlog": len(reqs) - len(done),
            "mixed_batched": batched, "fp64_one_at_a_time": fp64,
            "ratio_throughput": batched["value"] / fp64["value"] if fp64["value"] else None}


def run_serving(args):
    """Config-5 style stream on one GPU: Poisson arrivals (rate 20/s, seed 2)
    for --arrival-seconds, 70% cavities / 30% adsorbing channels with the
    config-5 size distributions, each solve run to density residual < 1e-6 or
    --max-steps, admission by HBM footprint against 150 GB."""
    if args.impl == "reference":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference has no serving loop; its CPU step is timed by the default workload"}))
        return
    log = None
    if args.metrics:
        from pyugks_b200.metrics import MetricsLog
        log = MetricsLog(args.metrics, workload="serving", precision="mixed")
    rec = serving_record(args.arrival_seconds, args.max_steps, metrics=log)
    line = {
        "metric": METRIC, "value": rec["mixed_batched"]["value"], "unit": UNIT, "n_gpus": 1,
        "steps": None, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": "serving stream: " + rec["stream"], "precision": "mixed"},
        "serving": rec,
    }
    if log is not None:
        log.write("bench", **line)
        log.close()
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--workload", default="multiblock",
                    choices=["multiblock", "cavity", "channel", "batched", "serving"])
    ap.add_argument("--arrival-seconds", type=float, default=2.0,
                    help="serving: length of the Poisson arrival window (rate 20/s)")
    ap.add_argument("--max-steps", type=int, default=2000, help="serving: step limit per solve")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--metrics", default=None,
                    help="append JSON-lines records (the bench line; serving: per tick and per request) here")
    ap.add_argument("--no-comparisons", action="store_true",
                    help="skip the batched-mixed and serving sub-records of the default line")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1 and args.impl == "ours":
        import datetime

        import torch.distributed as tdist
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        if args.workload == "serving":
            if rank == 0:
                run_serving(args)
        elif args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
