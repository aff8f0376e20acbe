"""Parity at the benchmarked sizes.

The bench workload (config 2: the 128 x 128 cavity as 2 x 2 blocks of 64 x 64
cells, 33 x 33 velocities, WENO5, Kn 0.01, built by bench.workload exactly as
the bench builds it) and the config-4 channel (256 x 64 cells in 4 blocks,
33 x 33 velocities, WENO5, Kn 0.05, adsorbing lower wall) are stepped by the
fused path, by the drop-in driver and by the reference's own kernels compiled
for the CPU (oracle/_ref, OpenMP over every host core), three steps each.
The reference has no first-order desorption, so the channel runs with the
reference's Langmuir desorption against the compiled reference, and with
k_des = 0.01 against the oracle's restatement (bit-exact with the reference
where both apply).

Bar: rho, U, V, T, q and f within 1e-11 relative, dt and time within 1e-12.
"""
import os

import numpy as np
import pytest

import bench
import host
import programs
import ugks_setup
from conftest import field_errors, rel_err
from pyugks_b200 import configs
from pyugks_b200.fused import FusedSolver
from pyugks_b200.ugks_sim import UGKSim

pytestmark = pytest.mark.gpu
TOL = 1e-11
STEPS = 3


def _oracle(case, backend):
    if backend == "ref":
        c = ugks_setup.Constants(case)
        # the reference's kernels for these cases are built by
        # __graft_entry__.build() into oracle/_ref, which ships with the tree:
        # a missing build is a packaging error, not a reason to skip
        assert all(programs.reference_available(c, b, k) for k, b in enumerate(case["blocks"])), \
            "compiled reference for this case not built (run __graft_entry__.build())"
        return host.OracleSim(case, "ref", threads=os.cpu_count())
    return host.OracleSim(case, "port")


# Three steps from rest leave the heat flux round-off sized in places (a sum
# of O(rho c^3) terms that cancel): it is compared against
# max(max |q|, Q_FLOOR) with Q_FLOOR a thousandth of its physical scale
# rho c^3 ~ 1, so that 1e-11 still bounds any real difference.
Q_FLOOR = 1e-3


def _compare(name, fields, fs, dt, time, ora):
    assert abs(dt - ora.dt) <= 1e-12 * ora.dt, (name, dt, ora.dt)
    assert abs(time - ora.time) <= 1e-12 * ora.time, (name, time, ora.time)
    for k, (a, b) in enumerate(zip(fields, ora.fields())):
        errs = field_errors(a, b)
        scale = max(float(np.max(np.hypot(b["qx"], b["qy"]))), Q_FLOOR)
        errs["q"] = float(np.max(np.hypot(a["qx"] - b["qx"], a["qy"] - b["qy"]))) / scale
        assert max(errs.values()) < TOL, (name, k, errs)
    for k, (a, b) in enumerate(zip(fs, ora.interior_f())):
        assert rel_err(a, b) < TOL, (name, k, rel_err(a, b))


CASES = {
    "config2_bench": (lambda: bench.workload("multiblock")[0][0], "ref"),
    "config4_langmuir": (lambda: configs.channel(nblocks=4, n=64, m=32, Kn=0.05, k_des=0.0,
                                                 CFL=configs.WORKLOAD_CFL), "ref"),
    "config4_first_order": (lambda: bench.workload("channel")[0][0], "port"),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_fused_fullsize_matches_reference(cuda, name):
    make, backend = CASES[name]
    case = make()
    ora = _oracle(case, backend)
    gpu = FusedSolver(case, precision="fp64")
    for _ in range(STEPS):
        ora.one_step()
    gpu.step(STEPS)
    st = gpu.solve_state()[0]
    assert st["status"] == 0 and st["steps"] == STEPS
    _compare(name, gpu.fields(), gpu.interior_f(), st["dt"], st["time"], ora)


@pytest.mark.parametrize("name", ["config2_bench", "config4_first_order"])
def test_dropin_fullsize_matches_reference(cuda, name):
    make, backend = CASES[name]
    case = make()
    ora = _oracle(case, backend)
    gpu = UGKSim(case)
    for _ in range(STEPS):
        ora.one_step()
        gpu.one_step()
    _compare(name, gpu.fields(), gpu.interior_f(), gpu.dt, gpu.time, ora)
