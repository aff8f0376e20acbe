"""Restart of the fused path from checkpoint files (ugks_restart_*), against
the oracle's restatement of the reference restart (ugks_sim.py:824-840,
ugks_block.py:274-300) on the same file: with saved f (including the inflow
ghosts that read the saved, converted Q), without f (fEQ start-up), a
restart that shares the block table with a fresh solve, and the GPU's own
save -> restart round trip against an uninterrupted run."""
import numpy as np
import pytest

import host
from conftest import fields_err, rel_err
from pyugks_b200 import checkpoint, configs
from pyugks_b200.fused import FusedSolver

pytestmark = pytest.mark.gpu
FP64_TOL = 1e-11


def save_oracle(sim, path, with_f=True):
    blocks = []
    for k, b in enumerate(sim.blocks):
        d = b.save_data(with_f)
        blocks.append(checkpoint.block_datasets(k, sim.dt, sim.time, d["macro"], d["Q_ext"], d["wall_prop"],
                                                d["wall_cover"], d["wall_fluxes"], d["f"]))
    checkpoint.write(path, sim.step, blocks, dict(Nv=sim.const.Nv, K=sim.const.K))


@pytest.mark.parametrize("make,with_f", [
    (lambda: configs.channel(nblocks=2, n=8, m=8), True),
    (lambda: configs.cavity_multiblock(nb=2, n=8, m=8), True),
    (lambda: configs.cavity(n=8, m=8, vlim=4.0), False),
])
def test_restart_matches_oracle(cuda, tmp_path, make, with_f):
    sim = host.OracleSim(make(), "port")
    sim.run(5)
    path = str(tmp_path / "ck.npz")
    save_oracle(sim, path, with_f)
    data = checkpoint.read(path)
    ora = host.OracleSim(make(), "port", restart=data)
    gpu = FusedSolver(make(), precision="fp64", restart={0: path})
    st = gpu.solve_state()[0]
    assert st["steps"] == 5 and st["time"] == ora.time
    assert abs(st["dt"] - ora.dt) <= 1e-12 * ora.dt
    ora.run(8)
    gpu.step(8)
    st = gpu.solve_state()[0]
    assert st["status"] == 0 and st["steps"] == 13
    assert abs(st["time"] - ora.time) <= 1e-12 * ora.time
    assert fields_err(gpu.fields(), ora.fields()) < FP64_TOL
    for g, o in zip(gpu.interior_f(), ora.interior_f()):
        assert rel_err(g, o) < FP64_TOL


def test_restart_beside_a_fresh_solve(cuda, tmp_path):
    """Solve 1 restarts while solve 0 of the same table starts fresh: each
    matches its own single-solve run."""
    a_case = lambda: configs.cavity(n=8, m=8, vlim=4.0)
    b_case = lambda: configs.channel(nblocks=2, n=8, m=8)
    sim = host.OracleSim(b_case(), "port")
    sim.run(4)
    path = str(tmp_path / "ck.npz")
    save_oracle(sim, path)
    both = FusedSolver([a_case(), b_case()], precision="fp64", restart={1: path})
    alone_a = FusedSolver(a_case(), precision="fp64")
    alone_b = FusedSolver(b_case(), precision="fp64", restart={0: path})
    both.step(6)
    alone_a.step(6)
    alone_b.step(6)
    assert fields_err(both.fields(0), alone_a.fields(0)) == 0.0
    assert fields_err(both.fields(1), alone_b.fields(0)) == 0.0
    s = both.solve_state()
    assert s[0]["steps"] == 6 and s[1]["steps"] == 10


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_gpu_save_restart_round_trip(cuda, tmp_path, precision, tol):
    case = lambda: configs.cavity(n=16, m=16, vlim=4.0)
    whole = FusedSolver(case(), precision=precision)
    whole.step(20)
    first = FusedSolver(case(), precision=precision)
    first.step(10)
    path = str(tmp_path / "ck.npz")
    first.save_checkpoint(path)
    with np.load(path) as z:
        assert int(z["final_step"]) == 10
        # the file holds the distributions themselves (the mixed path's
        # reference Maxwellian plus its stored deviation, in FP64)
        assert z["block_0/f"].dtype == np.float64
    second = FusedSolver(case(), precision=precision, restart={0: path})
    second.step(10)
    a, b = whole.solve_state()[0], second.solve_state()[0]
    assert b["steps"] == 20 and abs(a["time"] - b["time"]) <= 1e-13 * a["time"]
    assert fields_err(second.fields(), whole.fields()) < tol


def test_dropin_driver_restart_matches_oracle(cuda, tmp_path):
    """The per-kernel drop-in driver (UGKSim over KernelProgram) restarts the
    same way as the oracle, from the oracle's file and from its own."""
    from pyugks_b200.ugks_sim import UGKSim
    make = lambda: configs.channel(nblocks=2, n=8, m=8)
    sim = host.OracleSim(make(), "port")
    sim.run(4)
    path = str(tmp_path / "ck.npz")
    save_oracle(sim, path)
    ora = host.OracleSim(make(), "port", restart=checkpoint.read(path))
    drv = UGKSim(make(), restart=path)
    assert drv.step == 4 and drv.time == ora.time
    for _ in range(5):
        ora.one_step()
        drv.one_step()
    assert fields_err(drv.fields(), ora.fields()) < FP64_TOL
    # its own checkpoint: restarted by the driver and by the oracle alike
    # (with inflow boundaries a restart is not the uninterrupted run: the
    # start-up ghosts read the saved Q^n where the running solve used Q^(n-1))
    p2 = str(tmp_path / "ck2.npz")
    drv.save_checkpoint(p2)
    again = UGKSim(make(), restart=p2)
    ora2 = host.OracleSim(make(), "port", restart=checkpoint.read(p2))
    for _ in range(3):
        ora2.one_step()
        again.one_step()
    assert again.step == ora2.step == 12
    assert fields_err(again.fields(), ora2.fields()) < FP64_TOL
