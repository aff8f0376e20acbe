"""Drop-in kernels (ugks_<kernel> C ABI via KernelProgram) against the C oracle.

``TeeProgram`` sits under the oracle's restatement of the reference host
sequence: every kernel call is executed by the oracle (oracle/ugks_port.c) and
by the CUDA entry point on identical inputs, and every buffer argument is
compared afterwards.  Index-only ghost kernels must be bit-exact; arithmetic
kernels agree to 1e-12 relative (exp/erfc/pow ulps and reduction order).
"""
import numpy as np
import pytest
import torch

import host
import programs
from conftest import fields_err, rel_err
from pyugks_b200 import configs
from pyugks_b200.desc import VelocityTables, block_desc
from pyugks_b200.kernel_program import KernelProgram
from pyugks_b200.problem import Constants
from pyugks_b200.ugks_sim import UGKSim

pytestmark = pytest.mark.gpu

BIT_EXACT = {"edgeExchange", "edgeExtrapolate", "edgeMirror", "edgeBounceBack", "edgeConstGrad",
             "paraBC"}
KERNEL_TOL = 1e-12
# heat fluxes are compared against their physical scale rho*c^3 ~ 1: near
# equilibrium they are round-off sized and a pure relative error is noise
SCALE_FLOOR = {"calcQ": 1.0, "calcFaceQ": 1.0}


class TeeProgram:
    """Runs each kernel on the oracle and on the GPU and records the worst
    relative difference of every buffer argument."""

    def __init__(self, port, gpu, errors, where=None):
        self.port, self.gpu, self.errors = port, gpu, errors
        self.where = where if where is not None else {}
        self.cache = {}

    def _dev(self, a):
        t = self.cache.get(id(a))
        if t is None or t[0] is not a:
            t = (a, torch.empty(a.shape, dtype=torch.float64, device="cuda"))
            self.cache[id(a)] = t
        t[1].copy_(torch.from_numpy(a))
        return t[1]

    def __getattr__(self, name):
        def call(gsize, *args):
            dev = [self._dev(a) if isinstance(a, np.ndarray) else a for a in args]
            getattr(self.gpu, name)(None, gsize, None, *dev)
            getattr(self.port, name)(gsize, *args)
            torch.cuda.synchronize()
            worst = 0.0
            for ai, (a, d) in enumerate(zip(args, dev)):
                if isinstance(a, np.ndarray):
                    g = d.cpu().numpy()
                    if name in BIT_EXACT:
                        e = 0.0 if np.array_equal(g, a, equal_nan=True) else 1.0
                    else:
                        fin = np.isfinite(a)
                        ga, aa = np.where(fin, g, 0), np.where(fin, a, 0)
                        floor = SCALE_FLOOR.get(name, 0.0)
                        if name == "iFace":  # slopes: scale of f (round-off sized at equilibrium)
                            floor = float(np.max(np.abs(args[0])))
                        den = max(float(np.max(np.abs(aa))), floor)
                        diff = np.abs(ga - aa)
                        num = float(np.max(diff))
                        e = num / den if den > 0 else num
                        if not np.all(np.isfinite(ga[fin])):
                            e = np.inf
                    if e > worst:
                        worst = e
                        if e > KERNEL_TOL:
                            loc = np.unravel_index(np.argmax(np.where(np.isfinite(g - a), np.abs(g - a), np.inf)), a.shape)
                            self.where[name] = (ai, tuple(int(x) for x in loc), float(a[loc]), float(g[loc]), gsize)
            self.errors[name] = max(self.errors.get(name, 0.0), worst)
        return call


def tee_sim(case):
    errors = {}
    where = {}
    sim = host.OracleSim.__new__(host.OracleSim)
    # build the oracle simulation with tee programs in place of the port
    import ugks_setup as us
    sim.case = case
    sim.const = us.Constants(case)
    sim.time = sim.dt = 0.0
    sim.step = 0
    sim.force_time = False
    pconst = Constants(case)
    tabs = VelocityTables(pconst, torch.device("cuda"))
    geoms = us.block_geometry(case, sim.const.ghost)
    sim.blocks = []
    sim._keep = [tabs]
    for bid, (b, g) in enumerate(zip(case["blocks"], geoms)):
        port = programs.PortProgram(sim.const, b, bid)
        desc = block_desc(pconst, b, tabs)
        sim._keep.append(desc)
        tee = TeeProgram(port, KernelProgram(desc), errors, where)
        sim.blocks.append(host.OracleBlock(sim, bid, b, g, tee))
    sim.is_open = any(bc["type"] in (us.EXTRAPOLATE_OUT, us.INFLOW, us.OUTFLOW, us.CONSTANT)
                      for b in case["blocks"] for bc in b["bc"])
    for blk in sim.blocks:
        blk.init_functions()
    sim.update_all_bc()
    sim.calc_time_step()
    sim.update_time_step(limit=False)
    sim.initial_mass_total = sum(sim.total_mass())
    sim.global_residual = None
    sim.flux_passes = 0
    sim.where = where
    return sim, errors


CASES = {
    "cavity_vanleer": lambda: configs.cavity(n=8, m=8, vlim=4.0),
    "cavity_minmod": lambda: configs.cavity(n=8, m=8, vlim=4.0, flux_method="minmod", CFL=0.5),
    "multiblock_weno5": lambda: configs.cavity_multiblock(nb=2, n=8, m=8),
    "channel_langmuir": lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.0),
    "channel_first_order": lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.01),
    "channel_specular": lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.0, reflect_type="S"),
    "channel_cl": lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.01, reflect_type="CL", alpha_n=0.5,
                                          alpha_t=0.7),
    "channel_isotherm": lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.0, adsorb=configs.langmuir_table()),
    # block connections beyond opposite aligned faces, and the open faces
    "rotated_north_east": lambda: configs.rotated_pair(n=8, m=8),
    "flipped_north_north": lambda: configs.flipped_pair(n=8, m=8),
    "self_connected_flips": lambda: configs.mirror_cavity(n=8, m=8),
    "periodic_couette": lambda: configs.periodic_couette(n=8, m=8),
    "constant_outflow": lambda: configs.open_channel(n=8, m=8),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_every_kernel_matches_oracle(cuda, name):
    sim, errors = tee_sim(CASES[name]())
    for k in range(3):
        sim.one_step(get_res=(k == 2))
    assert errors, "no kernel ran"
    bad = {k: v for k, v in errors.items()
           if (v != 0.0 if k in BIT_EXACT else v > KERNEL_TOL)}
    assert not bad, (bad, sim.where)


@pytest.mark.parametrize("name", ["cavity_vanleer", "multiblock_weno5", "channel_first_order",
                                  "channel_specular", "channel_cl", "channel_isotherm"])
def test_dropin_driver_matches_oracle(cuda, name):
    case = CASES[name]()
    ora = host.OracleSim(case, "port")
    gpu = UGKSim(case)
    for k in range(15):
        ora.one_step(get_res=(k % 5 == 4))
        gpu.one_step(get_res=(k % 5 == 4))
    assert abs(gpu.dt - ora.dt) <= 1e-12 * ora.dt
    assert fields_err(gpu.fields(), ora.fields()) < 1e-11
    for a, b in zip(gpu.interior_f(), ora.interior_f()):
        assert rel_err(a, b) < 1e-11
    np.testing.assert_allclose(gpu.global_residual, ora.global_residual, rtol=1e-9)


def test_reflect_and_bounce_back_ghosts_bit_exact(cuda):
    """Specular and double-mirror ghost faces (edgeMirror / edgeBounceBack)."""
    case = configs.cavity(n=8, m=8, vlim=4.0)
    b = case["blocks"][0]
    b["bc"][0] = {"type": 3}
    b["bc"][1] = {"type": 9}
    b["bc"][2] = {"type": 3}
    b["bc"][3] = {"type": 1}
    sim, errors = tee_sim(case)
    for _ in range(2):
        sim.one_step()
    for k in ("edgeMirror", "edgeBounceBack", "edgeExtrapolate"):
        assert errors.get(k, None) == 0.0, (k, errors)
