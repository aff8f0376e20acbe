"""Continuous batching of independent UGKS solves on one GPU.

``SolvePool`` keeps every admitted solve resident in HBM (f, face fluxes,
macro, walls) and advances all of them together with the fused step
(``ugks_step_*``), one launch per phase for the whole pool.  Membership changes
between launches:

* ``admit(case)`` allocates the new solve's arrays, initialises it on a block
  table of its own (``ugks_init_*``), then rebuilds the shared table;
* ``retire(id)`` drops a solve and rebuilds the table;
* solves already in flight are untouched by either (their arrays stay where
  they are and their solve records are carried over), so a solve's result is
  the same alone and in any mix.

``Server`` runs a request stream against a pool: requests are admitted in
arrival order while their HBM footprint fits the budget; every tick advances
the pool by a fixed number of steps, each followed by the reference residual
(``ugks_block.py:1303-1327``) and the stop rule of every solve on the device,
so a solve stops at the step its density residual falls below its tolerance
or it reaches its step limit, and leaves at the end of that tick.
Time-to-converged is measured from arrival to the end of that tick.
``serve_one_at_a_time`` is the comparison arm: the same stream, one solve at
a time, to the same stop rule.
"""
from __future__ import annotations

import ctypes as C
import heapq
import time

import numpy as np

from . import _lib
from . import defs as D
from .fused import FusedSolver


def footprint_bytes(case: dict, precision: str) -> int:
    """HBM bytes a solve keeps resident: f and the two face-flux arrays, plus
    the per-cell and per-face FP64 arrays."""
    from .problem import VelocityGrid
    q = case["quad"]
    nv = VelocityGrid(q).Nv
    G = 3 if case["flux_method"] == "WENO5" else 2
    es = 8 if precision == "fp64" else 4
    total = 0
    for b in case["blocks"]:
        Ni, Nj = b["ni"] + 2 * G, b["nj"] + 2 * G
        total += 3 * Ni * Nj * nv * 2 * es
        total += Ni * Nj * 8 * (4 * 3 + 2 * 2 + 2 * 2 + 1 + 2 + 2 * 2 + 2 + 2 * 6)  # incl. face_geo
        total += max(b["ni"], b["nj"]) * 4 * 8 * (4 + 4 + 8) + max(b["ni"], b["nj"]) * nv * 16
    return total


class _Solve:
    def __init__(self, sid, case, solver):
        self.id = sid
        self.case = case
        self.solver = solver          # its own FusedSolver (arrays + one-solve table)
        self.cells = sum(b["ni"] * b["nj"] for b in case["blocks"])
        self.nv = solver.blocks[0].Nv
        self.record = None            # latest ugks_solve_state (bytes) while in the pool


def _records(raw: bytes, n: int):
    arr = (_lib.SolveState * n).from_buffer_copy(raw)
    return [dict(dt=x.dt, time=x.time, steps=x.steps, status=x.status, stopped=x.stopped, active=x.active,
                 residual=list(x.residual)) for x in arr]


class SolvePool:
    """Admitted solves advanced together, a tick at a time.

    A tick is ``ugks_serve_steps``: per step the fused step, the residual and
    the stop rule of every solve, decided on the device (ugks_stop_check), so
    that a solve stops at the step it meets its rule while the others go on.
    With ``graphs`` the tick is captured once per membership (a CUDA graph of
    all its launches) and replayed until a solve joins or leaves."""

    def __init__(self, precision="fp64", device="cuda", graphs=True):
        import torch
        self.precision = precision
        self.device = torch.device(device)
        self.lib = _lib.lib()
        self.mixed = 0 if precision == "fp64" else 1
        with torch.cuda.device(self.device):
            _lib.check(self.lib.ugks_prepare(self.mixed), "ugks_prepare")
        self.graphs = graphs
        self.solves = {}              # id -> _Solve, admission order
        self._next = 0
        self._table = None
        self._states = None
        self._sizes = None
        self._order = []
        self._dirty = True
        self._graph = None            # (steps per tick, CUDAGraph) of the current membership

    # -------------------------------------------------------------- membership
    def admit(self, case, tol=0.0, max_steps=0, start=10) -> int:
        """Allocate and initialise a solve with its stop rule (density
        residual below tol from `start` steps on, or max_steps steps; 0
        disables either); returns its id."""
        solver = FusedSolver(case, precision=self.precision, device=self.device)
        solver.set_stop_rule(0, tol, max_steps, start)
        sid = self._next
        self._next += 1
        s = _Solve(sid, case, solver)
        s.record = solver.solves.clone()
        self.solves[sid] = s
        self._dirty = True
        return sid

    def retire(self, sid):
        self._sync_records()
        s = self.solves.pop(sid)
        self._dirty = True
        return s

    def _sync_records(self):
        """Copy each solve's state record out of the shared array."""
        if self._states is None or not self._order:
            return
        sz = C.sizeof(_lib.SolveState)
        for k, sid in enumerate(self._order):
            if sid in self.solves:
                self.solves[sid].record = self._states[k * sz:(k + 1) * sz].clone()

    def _rebuild(self):
        import torch
        self._sync_records()
        self._graph = None  # its launches name the old table
        # group by limiter (ugks_fused_layout's rule), then by Nv (one face-pass
        # launch per run), then admission order
        order = sorted(self.solves, key=lambda sid: (D.FLUX_METHODS[self.solves[sid].case["flux_method"]],
                                                     self.solves[sid].nv, sid))
        structs, records = [], []
        for k, sid in enumerate(order):
            s = self.solves[sid]
            first = len(structs)
            for blk in s.solver.blocks:
                x = _lib.FusedBlock.from_buffer_copy(bytes(blk.struct))
                x.solve = k
                for f in range(4):
                    if blk.bc[f]["type"] in (D.ADJACENT, D.PERIODIC):
                        x.bc_block[f] = first + blk.bc[f]["other_block"]
                structs.append(x)
            rec = _lib.SolveState.from_buffer_copy(s.record.cpu().numpy().tobytes())
            rec.first_block = first
            rec.nblocks = len(s.solver.blocks)
            records.append(rec)
        self._order = order
        if not structs:
            self._table = self._states = None
            self._dirty = False
            return
        arr = (_lib.FusedBlock * len(structs))(*structs)
        self._sizes = _lib.FusedSizes()
        rc = self.lib.ugks_fused_layout(arr, len(structs), C.byref(self._sizes))
        if rc != 0:
            raise RuntimeError("ugks_fused_layout: %d" % rc)
        self._nblocks = len(structs)
        self._table = torch.from_numpy(np.frombuffer(bytes(arr), dtype=np.uint8).copy()).to(self.device)
        st = (_lib.SolveState * len(records))(*records)
        self._states = torch.from_numpy(np.frombuffer(bytes(st), dtype=np.uint8).copy()).to(self.device)
        self._dirty = False

    # -------------------------------------------------------------- stepping
    def _serve(self, n, stream):
        _lib.check(self.lib.ugks_serve_steps(self.mixed, self._table.data_ptr(), self._nblocks,
                                             C.byref(self._sizes), self._states.data_ptr(), len(self._order),
                                             n, stream), "ugks_serve_steps")

    def tick(self, n=1):
        """Advance every running solve by up to n steps (asynchronous)."""
        import torch
        if self._dirty:
            self._rebuild()
        if self._table is None:
            return
        if not self.graphs:
            self._serve(n, torch.cuda.current_stream(self.device).cuda_stream)
            return
        if self._graph is None or self._graph[0] != n:
            g = torch.cuda.CUDAGraph()
            cap = torch.cuda.Stream(self.device)
            cap.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.graph(g, stream=cap):
                self._serve(n, cap.cuda_stream)
            torch.cuda.current_stream(self.device).wait_stream(cap)
            self._graph = (n, g)
        self._graph[1].replay()

    def step(self, n=1):
        """Alias of tick (n steps of every running solve)."""
        self.tick(n)

    def states(self, rebuild=True):
        """{id: solve record dict} (synchronises).  With rebuild=False the
        solves admitted since the last tick are left out (they have not
        stepped yet)."""
        if self._dirty and rebuild:
            self._rebuild()
        if self._table is None:
            return {}
        return dict(zip(self._order, _records(self._states.cpu().numpy().tobytes(), len(self._order))))

    def fields(self, sid):
        return self.solves[sid].solver.fields(0)

    def interior_f(self, sid):
        return self.solves[sid].solver.interior_f(0)

    def units_per_step(self):
        return sum(s.cells * s.nv for s in self.solves.values())


class Request:
    def __init__(self, rid, arrival, case, max_steps, tol):
        self.id, self.arrival, self.case = rid, arrival, case
        self.max_steps, self.tol = max_steps, tol
        self.admitted = self.finished = None
        self.steps = 0
        self.reason = None
        self.units = case_units(case)


def case_units(case) -> int:
    """Cell-velocity points of one step of a solve."""
    from .configs import workload_size
    return workload_size(case)


class Server:
    def __init__(self, budget_bytes=150e9, precision="mixed", steps_per_tick=50, device="cuda", graphs=True):
        self.pool = SolvePool(precision, device, graphs=graphs)
        self.budget = budget_bytes
        self.precision = precision
        self.steps_per_tick = steps_per_tick
        self.used = 0
        self.done = []
        self.units = 0

    def run(self, requests, time_limit=None, metrics=None):
        """Serve a list of Request (arrival in seconds from the start).
        Returns the completed requests.

        A tick's steps are launched first; requests that arrived meanwhile are
        then set up (allocation, geometry, initialisation) on a side stream
        while the tick runs, and join the table at the next tick.  A solve
        stops on the device at the step that meets its rule (residual below
        its tolerance, its step limit, or an error status) and leaves at the
        end of that tick.  metrics: a metrics.MetricsLog that gets a record
        per tick and per completed request."""
        import torch
        dev = self.pool.device
        main = torch.cuda.current_stream(dev)
        side = torch.cuda.Stream(device=dev)
        queue = sorted(requests, key=lambda r: r.arrival)
        waiting = []
        active = {}
        t0 = time.perf_counter()
        i = 0

        def arrivals():
            nonlocal i
            now = time.perf_counter() - t0
            while i < len(queue) and queue[i].arrival <= now:
                waiting.append(queue[i])
                i += 1
            return now

        def admit():
            # in arrival order while the footprint fits
            while waiting:
                r = waiting[0]
                need = footprint_bytes(r.case, self.precision)
                if self.used + need > self.budget and active:
                    break
                waiting.pop(0)
                with torch.cuda.stream(side):
                    sid = self.pool.admit(r.case, r.tol, r.max_steps)
                r.admitted, r.need, r.sid = time.perf_counter() - t0, need, sid
                self.used += need
                active[sid] = r

        try:
            while i < len(queue) or waiting or active:
                now = arrivals()
                if time_limit is not None and now > time_limit:
                    break
                admit()
                main.wait_stream(side)
                if not active:
                    if i < len(queue):
                        time.sleep(max(0.0, min(queue[i].arrival - now, 0.05)))
                    continue
                self.pool.tick(self.steps_per_tick)
                arrivals()
                admit()                                      # overlaps the tick
                # the host sync here is also what makes retiring safe: every
                # kernel that reads a retired solve's arrays has finished
                states = self.pool.states(rebuild=False)
                main.wait_stream(side)
                now = time.perf_counter() - t0
                for sid, st in states.items():
                    r = active[sid]
                    self.units += (st["steps"] - r.steps) * r.units
                    r.steps = st["steps"]
                    if st["stopped"]:
                        r.finished, r.reason = now, _lib.STOP_REASONS[st["stopped"]]
                        self.pool.retire(sid)
                        self.used -= r.need
                        del active[sid]
                        self.done.append(r)
                        if metrics is not None:
                            metrics.request(r)
                if metrics is not None:
                    metrics.tick(now, len(active), len(waiting) + len(queue) - i, self.used, self.budget, self.units)
        finally:
            main.wait_stream(side)
        self.wall = time.perf_counter() - t0
        return self.done


def serve_one_at_a_time(requests, precision="fp64", steps_per_tick=50, device="cuda", graphs=True):
    """The comparison arm: the same requests served first come, first served,
    one solve at a time on the fused step, each to the same stop rule, with
    the same tick (steps_per_tick steps, replayed as one CUDA graph when
    graphs) as the batched server.  A request's service time is its solve's
    stepping time on the device (CUDA events around its ticks, the graph's
    capture included; set-up excluded); its completion is max(arrival,
    previous completion) + service, as for a single server working the queue
    in order.  Returns a dict with per-request latencies and the aggregate
    cell-velocity updates per second of service."""
    import torch
    dev = torch.device(device)
    lib = _lib.lib()
    mixed = 0 if precision == "fp64" else 1
    with torch.cuda.device(dev):
        _lib.check(lib.ugks_prepare(mixed), "ugks_prepare")
    clock, units, busy = 0.0, 0, 0.0
    lat, reasons, steps = [], [], []
    stream = torch.cuda.current_stream(dev)
    for r in sorted(requests, key=lambda q: q.arrival):
        pool = SolvePool(precision, dev, graphs=graphs)
        sid = pool.admit(r.case, r.tol, r.max_steps)
        torch.cuda.synchronize(dev)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        while True:
            pool.tick(steps_per_tick)
            st = pool.states(rebuild=False)[sid]  # synchronises
            if st["stopped"]:
                break
        t1.record(stream)
        torch.cuda.synchronize(dev)
        service = t0.elapsed_time(t1) / 1e3
        clock = max(clock, r.arrival) + service
        busy += service
        lat.append(clock - r.arrival)
        reasons.append(_lib.STOP_REASONS[st["stopped"]])
        steps.append(st["steps"])
        units += st["steps"] * r.units
        pool.retire(sid)
        del pool
    return dict(latency=lat, reasons=reasons, steps=steps, units=units, service_s=busy,
                value=units / busy if busy > 0 else 0.0, makespan_s=clock)


def request_stream(seed=2, rate=20.0, duration=600.0, max_steps=20000, tol=1e-6):
    """Poisson arrivals of cavity (p = 0.7, the batched-cavity distributions)
    and adsorbing-channel solves (p = 0.3: 64k x 16k cells, k in {1,2,4},
    m in {16,24,32}, Kn log-uniform on [0.01, 0.5])."""
    from . import configs
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        if rng.random() < 0.7:
            n = int(rng.choice(configs.CAVITY_SIZES))
            m = int(rng.choice(configs.CAVITY_VGRIDS))
            Kn = float(10 ** rng.uniform(np.log10(0.005), 0.0))
            lid = float(rng.uniform(0.05, 0.3))
            Tw = float(rng.uniform(0.8, 1.2))
            scheme = "WENO5" if rng.random() < 0.5 else "vanLeer"
            case = configs.cavity(n=n, m=m, vlim=5.0, flux_method=scheme, Kn=Kn, lid=lid, T_wall=Tw,
                                  CFL=configs.WORKLOAD_CFL)
        else:
            k = int(rng.choice([1, 2, 4]))
            m = int(rng.choice([16, 24, 32]))
            Kn = float(10 ** rng.uniform(np.log10(0.01), np.log10(0.5)))
            case = configs.channel(nblocks=4, n=16 * k, nj=16 * k, m=m, Kn=Kn, CFL=configs.WORKLOAD_CFL)
        out.append(Request(len(out), t, case, max_steps, tol))
    return out
