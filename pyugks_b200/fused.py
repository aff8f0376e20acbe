"""Fused time stepping: every block of every solve in one device-resident table.

``FusedSolver`` owns, as torch CUDA tensors, all per-block state of one or
more solves (a solve = one pyUGKS simulation, possibly multi-block) and
advances them with the fused entry points of libugks_b200.so:

* ``ugks_step_fp64`` / ``ugks_step_mixed``: one ``UGKSim.one_step`` of every
  active solve in five kernel launches plus two tiny dt launches, with dt
  control, the reference's single flux retry, and the ghost update done on
  the device (no host synchronisation inside a step);
* ``ugks_residual``: the reference residual on demand.

``precision="fp64"`` stores f and the face fluxes as double (the plain
method); ``"mixed"`` stores them as FP32 deviations from a reference
Maxwellian of each solve, in velocity pairs along u (``to_pairs``), with moments, the
conserved update, the relaxation and dt in FP64.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from . import checkpoint
from . import defs as D
from .desc import fill_walls
from .problem import Constants, VelocityGrid, fill_arrays, geometry


def _torch():
    import torch
    return torch


# ---------------------------------------------------------------------------
# mixed precision: deviations from a reference Maxwellian in velocity pairs
# ---------------------------------------------------------------------------
def reference_state(case):
    """(rho0, T0) of a solve's reference Maxwellian: the mean fill density, and
    the wall temperature the gas relaxes to (mean over its diffuse and
    adsorbing faces; the fill temperature when it has none)."""
    rho, cells, tw = 0.0, 0, []
    for b in case["blocks"]:
        n = b["ni"] * b["nj"]
        rho += float(np.mean(np.broadcast_to(np.asarray(b["fill"].get("D", 1.0), dtype=np.float64),
                                             (b["ni"], b["nj"])))) * n
        cells += n
        tw += [bc["T"] for bc in b["bc"] if bc["type"] in (D.DIFFUSE, D.ADSORBING)]
    T0 = float(np.mean(tw)) if tw else float(np.mean([np.mean(b["fill"].get("T", 1.0)) for b in case["blocks"]]))
    return rho / cells, T0


def reference_table(const, rho0, T0):
    """The UGKS_REF_* array of include/ugks_b200.h for a reference Maxwellian
    at rest with density rho0 and temperature T0 on this velocity grid."""
    vg = const.vgrid
    lam0 = 1.0 / T0
    P0 = rho0 * lam0 / const.PI
    kb0 = 0.5 * const.K / lam0
    q = vg.quad
    mh = vg.weight * P0 * np.exp(-lam0 * (q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]))
    x, y = q[:, 0], q[:, 1]
    mom = [np.sum(mh), np.sum(x * mh), np.sum(y * mh), np.sum(x * x * mh), np.sum(x * y * mh),
           np.sum(y * y * mh), np.sum(x * x * x * mh), np.sum(x * x * y * mh), np.sum(x * y * y * mh),
           np.sum(y * y * y * mh), np.sum(kb0 * mh), np.sum(x * kb0 * mh), np.sum(y * kb0 * mh)]
    u = q[::vg.v_num, 0]
    v = q[:vg.v_num, 1]
    Au = vg.wu * np.sqrt(P0) * np.exp(-lam0 * u * u)
    Av = vg.wv * np.sqrt(P0) * np.exp(-lam0 * v * v)
    out = np.zeros(_lib.REF_TAB + vg.Nv + vg.u_num + vg.v_num)
    out[_lib.REF_LAMBDA], out[_lib.REF_P0], out[_lib.REF_KB0] = lam0, P0, kb0
    out[_lib.REF_MOM:_lib.REF_MOM + len(mom)] = mom
    out[_lib.REF_TAB:_lib.REF_TAB + vg.Nv] = mh
    out[_lib.REF_TAB + vg.Nv:_lib.REF_TAB + vg.Nv + vg.u_num] = Au
    out[_lib.REF_TAB + vg.Nv + vg.u_num:] = Av
    return out


def pair_count(vg) -> int:
    """Velocity pairs per cell of the mixed storage: ceil(u_num / 2) v_num."""
    return (vg.u_num + 1) // 2 * vg.v_num


def to_pairs(f, ref, vg):
    """(..., Nv, 2) FP64 distributions -> (..., pair_count, 4) FP32 deviations
    from the reference Maxwellian: pair a v_num + jv holds velocities
    (2a, jv) and (2a + 1, jv) as (h, h', b, b'); an odd u_num pads the last
    pair row's second lane with zeros."""
    nv, un, vn = vg.Nv, vg.u_num, vg.v_num
    lead = f.shape[:-2]
    mh = ref[_lib.REF_TAB:_lib.REF_TAB + nv]
    d = np.zeros(lead + (un + (un & 1), vn, 2))
    d[..., :un, :, 0] = (f[..., 0] - mh).reshape(lead + (un, vn))
    d[..., :un, :, 1] = (f[..., 1] - ref[_lib.REF_KB0] * mh).reshape(lead + (un, vn))
    d = d.reshape(lead + ((un + 1) // 2, 2, vn, 2))             # (a, lane, jv, component)
    d = np.moveaxis(d, -3, -1)                                   # (a, jv, component, lane)
    return np.ascontiguousarray(d.reshape(lead + (pair_count(vg), 4))).astype(np.float32)


def from_pairs(p, ref, vg):
    """Inverse of to_pairs: FP64 (..., Nv, 2) distributions."""
    nv, un, vn = vg.Nv, vg.u_num, vg.v_num
    lead = p.shape[:-2]
    d = np.asarray(p, dtype=np.float64).reshape(lead + ((un + 1) // 2, vn, 2, 2))  # (a, jv, comp, lane)
    d = np.moveaxis(d, -1, -3).reshape(lead + (un + (un & 1), vn, 2))[..., :un, :, :].reshape(lead + (nv, 2))
    mh = ref[_lib.REF_TAB:_lib.REF_TAB + nv]
    out = np.empty(d.shape)
    out[..., 0] = d[..., 0] + mh
    out[..., 1] = d[..., 1] + ref[_lib.REF_KB0] * mh
    return out


class _Block:
    pass


class FusedSolver:
    def __init__(self, cases, precision: str = "fp64", device="cuda", stream=None, restart=None, tune=False):
        """restart: {caller's solve index: checkpoint path or the dict of
        checkpoint.read}; those solves resume from the saved state (the
        reference's restart, ugks_sim.py:824-840, ugks_block.py:274-300)
        instead of starting from their fill condition.
        tune: pick the launch shapes with tuner.tune (cached per kind of
        segment; timed on a scratch copy when not cached)."""
        torch = _torch()
        if precision not in ("fp64", "mixed"):
            raise ValueError(precision)
        self.lib = _lib.lib()
        if not torch.cuda.is_available():
            raise RuntimeError("FusedSolver needs a CUDA device (no CPU fallback)")
        self.precision = precision
        self.device = torch.device(device)
        self.sdtype = torch.float64 if precision == "fp64" else torch.float32
        if isinstance(cases, dict):
            cases = [cases]
        cases = list(cases)
        # solves are stored grouped by flux method, then by velocity-grid size
        # (a face-pass launch covers a contiguous run of one method and one Nv,
        # with shared memory sized for it); order[k] is the internal index of
        # the caller's solve k
        nvs = [VelocityGrid(c["quad"]).Nv for c in cases]
        perm = sorted(range(len(cases)), key=lambda k: (D.FLUX_METHODS[cases[k]["flux_method"]], nvs[k], k))
        self.order = [0] * len(cases)
        for internal, k in enumerate(perm):
            self.order[k] = internal
        self.cases = [cases[k] for k in perm]
        self.blocks = []
        self.solve_blocks = []
        self._keep = []
        structs = []
        for s, case in enumerate(self.cases):
            const = Constants(case)
            geoms = geometry(case, const.ghost)
            vg = const.vgrid
            tabs = dict(quad=self._dev(vg.quad), weight=self._dev(vg.weight),
                        mNS=self._dev(vg.mirror_NS, torch.int32), mEW=self._dev(vg.mirror_EW, torch.int32),
                        mD=self._dev(vg.mirror_D, torch.int32))
            if precision == "mixed":
                if vg.u_num * vg.v_num != vg.Nv:
                    raise ValueError("mixed precision needs a tensor velocity grid")
                tabs["ref_host"] = reference_table(const, *reference_state(case))
                tabs["ref"] = self._dev(tabs["ref_host"])
            self._keep.append(tabs)
            first = len(self.blocks)
            ids = []
            for k, (b, g) in enumerate(zip(case["blocks"], geoms)):
                blk = self._make_block(s, k, first, case, b, g, const, tabs)
                ids.append(len(self.blocks))
                self.blocks.append(blk)
                structs.append(blk.struct)
            self.solve_blocks.append(ids)
        arr = (_lib.FusedBlock * len(structs))(*structs)
        self.sizes = _lib.FusedSizes()
        rc = self.lib.ugks_fused_layout(arr, len(structs), C.byref(self.sizes))
        if rc != 0:
            raise RuntimeError("ugks_fused_layout rejected the block table (%d)" % rc)
        self.n_faces, self.n_cells, self.n_ghost = self.sizes.n_faces, self.sizes.n_cells, self.sizes.n_ghost
        self.max_nv = self.sizes.max_nv
        raw = np.frombuffer(bytes(arr), dtype=np.uint8).copy()
        self.table = torch.from_numpy(raw).to(self.device)
        self.nblocks = len(structs)
        st = (_lib.SolveState * len(self.cases))()
        for s, case in enumerate(self.cases):
            st[s].CFL = float(case["CFL"])
            st[s].delta_dt = float(case.get("delta_dt", 1.0))
            st[s].active = 1
            st[s].nblocks = len(self.solve_blocks[s])
            st[s].first_block = self.solve_blocks[s][0]
        # restarts: load the saved state into the block arrays
        with_f = set()
        for k, ck in (restart or {}).items():
            s = self.order[k]
            data = ck if isinstance(ck, dict) else checkpoint.read(ck)
            if len(data["blocks"]) != len(self.solve_blocks[s]):
                raise ValueError("checkpoint has %d blocks, solve %d has %d"
                                 % (len(data["blocks"]), k, len(self.solve_blocks[s])))
            for bi, bd in zip(self.solve_blocks[s], data["blocks"]):
                blk = self.blocks[bi]
                if bd["macro"].shape != tuple(blk.macro.shape):
                    raise ValueError("checkpoint block shape %s != %s" % (bd["macro"].shape, tuple(blk.macro.shape)))
                blk.macro.copy_(self._dev(bd["macro"]))
                blk.Q.copy_(self._dev(bd["Q"]))
                if bd["f"] is not None:
                    blk.f.copy_(self._dev(self._stored_f(blk, np.asarray(bd["f"], dtype=np.float64))))
                    with_f.add(s)
            st[s].time = data["blocks"][0]["time"]
            st[s].steps = int(data["final_step"])
        self.solves = torch.from_numpy(np.frombuffer(bytes(st), dtype=np.uint8).copy()).to(self.device)
        self.nsolves = len(self.cases)
        self._stream = stream
        init = self.lib.ugks_init_fp64 if precision == "fp64" else self.lib.ugks_init_mixed
        rst = self.lib.ugks_restart_fp64 if precision == "fp64" else self.lib.ugks_restart_mixed
        args = lambda: (self.table.data_ptr(), self.nblocks, C.byref(self.sizes), self.solves.data_ptr(),
                        self.nsolves, self._sptr())
        if not with_f:
            _lib.check(init(*args()), "ugks_init")
        else:
            # solves restarted with saved f skip the equilibrium start-up
            self._set_active_internal([s not in with_f for s in range(self.nsolves)])
            if len(with_f) < self.nsolves:
                _lib.check(init(*args()), "ugks_init")
            self._set_active_internal([s in with_f for s in range(self.nsolves)])
            _lib.check(rst(*args()), "ugks_restart")
            self._set_active_internal([True] * self.nsolves)
        self._step_fn = self.lib.ugks_step_fp64 if precision == "fp64" else self.lib.ugks_step_mixed
        self.graph = None
        self.shapes = None
        if tune:
            from . import tuner
            self.shapes = tuner.tune(self)

    # ---------------------------------------------------------------- set-up
    def _dev(self, a, dtype=None):
        torch = _torch()
        t = torch.from_numpy(np.ascontiguousarray(a))
        if dtype is not None:
            t = t.to(dtype)
        return t.to(self.device)

    def _make_block(self, s, k, first, case, b, g, const, tabs):
        torch = _torch()
        blk = _Block()
        G = const.ghost
        ni, nj = b["ni"], b["nj"]
        Ni, Nj, Nv = ni + 2 * G, nj + 2 * G, const.Nv
        blk.solve, blk.index, blk.ni, blk.nj, blk.Ni, blk.Nj, blk.Nv, blk.G = s, k, ni, nj, Ni, Nj, Nv, G
        blk.bc = b["bc"]
        dev = self.device
        z = lambda *shape, dt=torch.float64: torch.zeros(shape, dtype=dt, device=dev)
        # FP64: (h, b) per velocity; mixed: FP32 deviations in velocity pairs
        shape = (Ni, Nj, Nv, 2) if self.precision == "fp64" else (Ni, Nj, pair_count(const.vgrid), 4)
        blk.ref = tabs.get("ref_host")
        blk.vgrid = const.vgrid
        blk.f = z(*shape, dt=self.sdtype)
        blk.flux_S = z(*shape, dt=self.sdtype)
        blk.flux_W = z(*shape, dt=self.sdtype)
        blk.flux_macro_S = z(Ni, Nj, 4)
        blk.flux_macro_W = z(Ni, Nj, 4)
        macro, Q = fill_arrays(b)
        blk.macro = self._dev(macro)
        blk.Q = self._dev(Q)
        blk.prim_old = z(ni, nj, 4)
        for name in ("area", "centre", "mid_side", "normal", "side_length", "xy"):
            setattr(blk, name, self._dev(np.nan_to_num(g[name], nan=0.0) if name != "xy" else g[name]))
        wl = max(ni, nj)
        blk.wall_prop = z(wl, 4, 4)
        cover = np.zeros((wl, 4, 4))
        for f, bc in enumerate(b["bc"]):
            cover[:, f, 0] = bc.get("cover_initial", 0.0)
        blk.wall_cover = self._dev(cover)
        blk.wall_fluxes = z(wl, 4, 8)
        blk.wall_dist = z(wl, Nv, 2)
        blk.cell_mom = z(Ni, Nj, 4)
        blk.Q_next = z(ni, nj, 2)
        blk.face_geo = z(Ni, Nj, 2, 6)
        if self.precision != "fp64":
            # the mixed face pass's scratch: slopes beside the stored face
            # deviations, and a record per face between its three launches
            blk.aux_S = z(*shape, dt=self.sdtype)
            blk.aux_W = z(*shape, dt=self.sdtype)
            blk.face_rec = z(Ni, Nj, 2, _lib.FACE_REC)
        x = _lib.FusedBlock()
        d = x.d
        d.ni, d.nj, d.Ni, d.Nj, d.ghost, d.Nv = ni, nj, Ni, Nj, G, Nv
        d.flux_method, d.relax_type = const.flux_code, const.relax_type
        d.u_num, d.v_num = const.vgrid.u_num, const.vgrid.v_num
        d.PI, d.Pr, d.umax, d.vmax = const.PI, const.Pr, const.umax, const.vmax
        d.Kn_eff, d.gam, d.K, d.omega = const.Kn_eff, const.gam, const.K, const.omega
        d.B = const.B
        d.quad, d.weight = tabs["quad"].data_ptr(), tabs["weight"].data_ptr()
        d.mirror_NS, d.mirror_EW, d.mirror_D = (tabs["mNS"].data_ptr(), tabs["mEW"].data_ptr(),
                                                tabs["mD"].data_ptr())
        fill_walls(d, b, self._keep, self.device)
        for f, bc in enumerate(b["bc"]):
            x.bc_type[f] = bc["type"]
            if bc["type"] in (D.ADJACENT, D.PERIODIC):  # both copy through edgeExchange
                x.bc_block[f] = first + bc["other_block"]
                x.bc_face[f] = bc["other_face"]
                x.bc_ori[f] = bc.get("orientation", 1)
                x.bc_flip[f] = bc.get("flip", D.NO_FLIP)
        x.solve = s
        for name in ("f", "flux_S", "flux_W", "flux_macro_S", "flux_macro_W", "macro", "Q", "prim_old",
                     "area", "centre", "mid_side", "normal", "side_length", "xy", "wall_prop",
                     "wall_cover", "wall_fluxes", "wall_dist", "cell_mom", "Q_next", "face_geo"):
            setattr(x, name, getattr(blk, name).data_ptr())
        if "ref" in tabs:
            x.ref = tabs["ref"].data_ptr()
        if self.precision != "fp64":
            x.aux_S, x.aux_W, x.face_rec = blk.aux_S.data_ptr(), blk.aux_W.data_ptr(), blk.face_rec.data_ptr()
        blk.struct = x
        return blk

    def _sptr(self):
        torch = _torch()
        s = self._stream if self._stream is not None else torch.cuda.current_stream(self.device)
        return s.cuda_stream

    # ---------------------------------------------------------------- stepping
    def launches_per_step(self) -> int:
        """Kernel launches of one ugks_step_* call (ugks_step_launches): one
        face pass per (limiter, Nv) segment, one retry pass per limiter
        present, two dt checks, the cell pass, the dt update and the ghost
        pass; mixed precision adds the face pass's coefficient and flux
        launches."""
        return self.lib.ugks_step_launches(C.byref(self.sizes), 0 if self.precision == "fp64" else 1)

    def step(self, n: int = 1):
        """Advance every active solve by n steps (asynchronous)."""
        for _ in range(n):
            _lib.check(self._step_fn(self.table.data_ptr(), self.nblocks, C.byref(self.sizes),
                                     self.solves.data_ptr(), self.nsolves, self._sptr()), "ugks_step")

    def capture(self, steps: int):
        """Capture `steps` steps as one CUDA graph; ``replay()`` runs it."""
        torch = _torch()
        # kernel attributes are set before capture (not a stream operation)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.ugks_prepare(0 if self.precision == "fp64" else 1), "ugks_prepare")
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        old = self._stream
        with torch.cuda.stream(s):
            self._stream = s
            with torch.cuda.graph(g, stream=s):
                self.step(steps)
        self._stream = old
        torch.cuda.current_stream(self.device).wait_stream(s)
        self.graph = g
        self.graph_steps = steps
        return g

    def replay(self):
        self.graph.replay()

    def compute_residual(self):
        _lib.check(self.lib.ugks_residual(self.table.data_ptr(), self.nblocks, self.solves.data_ptr(),
                                          self.nsolves, self._sptr()), "ugks_residual")

    # ---------------------------------------------------------------- readback
    def solve_state(self):
        """Host copy of every ugks_solve_state (synchronises)."""
        raw = self.solves.cpu().numpy().tobytes()
        arr = (_lib.SolveState * self.nsolves).from_buffer_copy(raw)
        out = [dict(dt=x.dt, time=x.time, max_dt=x.max_dt, status=x.status, steps=x.steps,
                    retries=x.retries, active=x.active, stopped=x.stopped, residual=list(x.residual))
               for x in arr]
        return [out[self.order[k]] for k in range(self.nsolves)]

    def set_stop_rule(self, solve: int, tol: float = 0.0, max_steps: int = 0, start: int = 10):
        """The device-side stop rule of the caller's solve (ugks_stop_check):
        stop when the density residual falls below tol once at least `start`
        steps are done (the reference's residual_start: a solve that starts
        from rest changes its density by round-off in its first steps), or
        after max_steps steps (0 disables either)."""
        torch = _torch()
        torch.cuda.synchronize(self.device)
        st = (_lib.SolveState * self.nsolves).from_buffer_copy(self.solves.cpu().numpy().tobytes())
        s = self.order[solve]
        st[s].stop_residual = float(tol)
        st[s].stop_steps = int(max_steps)
        st[s].stop_after = int(start)
        self.solves.copy_(torch.from_numpy(np.frombuffer(bytes(st), dtype=np.uint8).copy()))

    def set_active(self, flags):
        """Switch solves on/off for the next steps (device-side flag)."""
        self._set_active_internal([flags[k] for k in sorted(range(self.nsolves), key=lambda k: self.order[k])])

    def _set_active_internal(self, flags):
        torch = _torch()
        torch.cuda.synchronize(self.device)  # the solve records may be written on another stream
        st = (_lib.SolveState * self.nsolves).from_buffer_copy(self.solves.cpu().numpy().tobytes())
        for s, a in enumerate(flags):
            st[s].active = 1 if a else 0
        self.solves.copy_(torch.from_numpy(np.frombuffer(bytes(st), dtype=np.uint8).copy()))

    def _stored_f(self, b, f):
        """FP64 (Ni, Nj, Nv, 2) distributions in this solver's storage form."""
        return f if self.precision == "fp64" else to_pairs(f, b.ref, b.vgrid)

    def full_f(self, b):
        """Block b's distributions with ghosts as FP64 (Ni, Nj, Nv, 2) numpy."""
        f = b.f.cpu().numpy()
        return f if self.precision == "fp64" else from_pairs(f, b.ref, b.vgrid)

    def _full_f_device(self, b):
        """The same as a CUDA FP64 tensor in the reference layout (for the
        drop-in diagnostic kernels)."""
        return b.f if self.precision == "fp64" else self._dev(self.full_f(b))

    def save_checkpoint(self, path: str, solve: int = 0, save_f: bool = True):
        """Write one solve's state as a checkpoint (checkpoint.py; the
        reference's saveHDF5 + close_HDF5, ugks_sim.py:1022-1096)."""
        s = self.order[solve]
        state = self.solve_state()[solve]
        const = Constants(self.cases[s])
        blocks = []
        for k, bi in enumerate(self.solve_blocks[s]):
            b = self.blocks[bi]
            m = b.macro.cpu().numpy()
            f_full = self.full_f(b)
            q = self._heat_flux(b, f_full[b.G:-b.G, b.G:-b.G], m)
            blocks.append(checkpoint.block_datasets(
                k, state["dt"], state["time"], m, checkpoint.external_heat_flux(q, const.K),
                b.wall_prop.cpu().numpy(), b.wall_cover.cpu().numpy(), b.wall_fluxes.cpu().numpy(),
                f_full if save_f else None))
        meta = dict(Nv=const.Nv, K=const.K, CFL=float(self.cases[s]["CFL"]), quad=const.vgrid.quad,
                    weight=const.vgrid.weight)
        checkpoint.write(path, state["steps"], blocks, meta)

    def fields(self, solve: int = 0):
        """Per block interior fields of one solve (caller's index) as numpy:
        rho, U, V, T, qx, qy (Q re-taken from the current f, as the
        reference's updateHost does)."""
        out = []
        for bi in self.solve_blocks[self.order[solve]]:
            b = self.blocks[bi]
            m = b.macro.cpu().numpy()
            f = self.full_f(b)[b.G:-b.G, b.G:-b.G]
            q = self._heat_flux(b, f, m)
            out.append(dict(rho=m[:, :, 0], U=m[:, :, 1], V=m[:, :, 2], T=1.0 / m[:, :, 3],
                            qx=q[:, :, 0], qy=q[:, :, 1]))
        return out

    def _heat_flux(self, b, f, m):
        vg = Constants(self.cases[b.solve]).vgrid
        K = Constants(self.cases[b.solve]).K
        cx = vg.quad[None, None, :, 0] - m[:, :, None, 1]
        cy = vg.quad[None, None, :, 1] - m[:, :, None, 2]
        t = (cx * cx + cy * cy) * f[..., 0] + f[..., 1] / K
        return np.stack([0.5 * np.sum(cx * t, axis=-1), 0.5 * np.sum(cy * t, axis=-1)], -1)

    def interior_f(self, solve: int = 0):
        out = []
        for bi in self.solve_blocks[self.order[solve]]:
            b = self.blocks[bi]
            out.append(self.full_f(b)[b.G:-b.G, b.G:-b.G])
        return out

    def _program(self, bi):
        from .kernel_program import KernelProgram
        b = self.blocks[bi]
        if not hasattr(b, "prg"):
            b.prg = KernelProgram(b.struct.d)
        return b.prg

    def internal_data(self, solve: int = 0):
        """Per block of the caller's solve (Txyz [ni, nj, 4], stress
        [ni, nj, 3]) from getInternal (clKernel.c:314-375)."""
        from .diagnostics import internal_data
        out = []
        for bi in self.solve_blocks[self.order[solve]]:
            b = self.blocks[bi]
            out.append(internal_data(self._program(bi), self._full_f_device(b), b.ni, b.nj))
        return out

    def interface_distribution(self, solve: int = 0):
        """Per block of the caller's solve the reconstructed distribution
        at its walls (get_interface_distribution, ugks_block.py:985-1047)."""
        from .diagnostics import interface_distribution
        out = []
        for bi in self.solve_blocks[self.order[solve]]:
            b = self.blocks[bi]
            out.append(interface_distribution(self._program(bi), self._full_f_device(b), b.centre, b.mid_side,
                                              b.normal, b.ni, b.nj, b.G))
        return out

    def solve_block_ids(self, solve: int):
        """Indices in self.blocks of the blocks of the caller's solve."""
        return self.solve_blocks[self.order[solve]]
