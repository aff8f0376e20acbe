"""Diagnostics on the GPU: the getInternal drop-in against the oracle, the
drivers' internal_data / interface_distribution against the oracle's, and
the run loop's max_time exit landing on max_time (ugks_sim.py:592-597,
700-702)."""
import numpy as np
import pytest

import host
from pyugks_b200 import configs
from pyugks_b200.fused import FusedSolver
from pyugks_b200.ugks_sim import UGKSim
from test_dropin_gpu import KERNEL_TOL, tee_sim

pytestmark = pytest.mark.gpu

CASES = {
    "cavity_vanleer": lambda: configs.cavity(n=8, m=8, vlim=4.0),
    "channel_weno5": lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.01),
}


def close(a, b, tol):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b))) <= tol * max(float(np.max(np.abs(b))), 1e-300)


@pytest.mark.parametrize("name", sorted(CASES))
def test_getInternal_kernel_matches_oracle(cuda, name):
    sim, errors = tee_sim(CASES[name]())
    for _ in range(3):
        sim.one_step()
    errors.clear()
    for blk in sim.blocks:
        blk.internal_data()
        blk.interface_distribution()
    assert errors["getInternal"] <= KERNEL_TOL, (errors, sim.where)
    assert errors["iFace"] <= KERNEL_TOL, (errors, sim.where)


@pytest.mark.parametrize("driver", ["dropin", "fused"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_driver_diagnostics_match_oracle(cuda, name, driver):
    case = CASES[name]()
    ora = host.OracleSim(case, "port")
    ora.run(8)
    if driver == "dropin":
        gpu = UGKSim(case)
        for _ in range(8):
            gpu.one_step()
        internal, faces = gpu.internal_data(), gpu.interface_distribution()
    else:
        gpu = FusedSolver(case, precision="fp64")
        gpu.step(8)
        internal, faces = gpu.internal_data(), gpu.interface_distribution()
    for blk, (txyz, stress), fd in zip(ora.blocks, internal, faces):
        o_txyz, o_stress = blk.internal_data()
        assert close(txyz, o_txyz, 1e-11)
        assert close(stress, o_stress, 1e-9)
        o_faces = blk.interface_distribution()
        for k in "NESW":
            assert close(fd[k], o_faces[k], 1e-10), k


def test_run_stops_on_max_time(cuda):
    case = configs.cavity(n=8, m=8, vlim=4.0)
    gpu = UGKSim(case)
    gpu.one_step()
    max_time = gpu.time + 3.5 * gpu.dt
    why = gpu.run(100, max_time=max_time)
    assert why == "time limit reached"
    assert abs(gpu.time - max_time) <= 1e-12 * max_time
