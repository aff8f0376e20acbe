"""Fused step path (ugks_step_fp64 / ugks_step_mixed) against the C oracle.

The oracle (oracle/ugks_port.c, bit-exact with the reference kernels compiled
for the CPU) runs the same case step by step; the fused GPU path must match
density, velocity, temperature, heat flux and f to 1e-11 relative in FP64
(differences come only from exp/erfc/pow ulps and reduction order), and to
1e-5 relative in mixed precision (FP32 storage of f and the face fluxes).
"""
import numpy as np
import pytest

import host
from conftest import fields_err, rel_err
from pyugks_b200 import configs
from pyugks_b200.fused import FusedSolver

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-11
MIXED_TOL = 1e-5


def run_both(case, steps, precision="fp64"):
    ora = host.OracleSim(case, "port")
    gpu = FusedSolver(case, precision=precision)
    for _ in range(steps):
        ora.one_step()
    gpu.step(steps)
    return ora, gpu


def test_cavity_vanleer_fp64(cuda):
    ora, gpu = run_both(configs.cavity(n=8, m=8, vlim=4.0), 30)
    st = gpu.solve_state()[0]
    assert st["status"] == 0 and st["steps"] == 30
    assert abs(st["dt"] - ora.dt) <= 1e-12 * ora.dt
    assert abs(st["time"] - ora.time) <= 1e-12 * ora.time
    assert fields_err(gpu.fields(), ora.fields()) < FP64_TOL
    assert rel_err(gpu.interior_f()[0], ora.interior_f()[0]) < FP64_TOL


def test_cavity_multiblock_weno5_fp64(cuda):
    ora, gpu = run_both(configs.cavity_multiblock(nb=2, n=8, m=8), 20)
    assert fields_err(gpu.fields(), ora.fields()) < FP64_TOL
    for a, b in zip(gpu.interior_f(), ora.interior_f()):
        assert rel_err(a, b) < FP64_TOL


@pytest.mark.parametrize("reflect,k_des", [("D", 0.01), ("S", 0.0), ("S", 0.01), ("CL", 0.01)])
def test_channel_adsorbing_fp64(cuda, reflect, k_des):
    """Adsorbing lower wall with each re-emission model (adsorbingWall{D,S,CL}_P2)."""
    case = configs.channel(nblocks=2, n=8, m=8, k_des=k_des, reflect_type=reflect, alpha_n=0.5, alpha_t=0.7)
    ora, gpu = run_both(case, 20)
    assert fields_err(gpu.fields(), ora.fields()) < FP64_TOL
    for bi, ob in zip(gpu.solve_block_ids(0), ora.blocks):
        cov = gpu.blocks[bi].wall_cover.cpu().numpy()
        assert rel_err(cov[:8, 2, :], ob.wall_cover[:8, 2, :]) < FP64_TOL


def test_channel_tabulated_isotherm_fp64(cuda):
    """Langmuir desorption with the equilibrium coverage interpolated from a
    tabulated isotherm (vartheta_langmuir, clAdsorb.c:171-247)."""
    case = configs.channel(nblocks=2, n=8, m=8, k_des=0.0, adsorb=configs.langmuir_table())
    ora, gpu = run_both(case, 20)
    assert gpu.solve_state()[0]["status"] == 0
    assert fields_err(gpu.fields(), ora.fields()) < FP64_TOL
    for bi, ob in zip(gpu.solve_block_ids(0), ora.blocks):
        cov = gpu.blocks[bi].wall_cover.cpu().numpy()
        assert rel_err(cov[:8, 2, :], ob.wall_cover[:8, 2, :]) < FP64_TOL


def test_isotherm_outside_the_table_flags_status_4(cuda):
    """A wall state outside the tabulated isotherm sets the reference's
    ERR_CLAMPING_ADSORB_ISOTHERM (4) in the solve record; nothing faults."""
    table = configs.langmuir_table(p_range=(2.0, 3.0))   # pressures far above the channel's
    case = configs.channel(nblocks=2, n=8, m=8, k_des=0.0, adsorb=table)
    ora, gpu = run_both(case, 2)
    assert gpu.solve_state()[0]["status"] == 4
    # the reference skips the rest of that wall face and ignores the error
    # return (ugks_block.py:949-950, 1084); so does the oracle
    assert fields_err(gpu.fields(), ora.fields()) < FP64_TOL


def test_cavity_mixed_precision(cuda):
    ora, gpu = run_both(configs.cavity(n=8, m=8, vlim=4.0), 30, precision="mixed")
    assert fields_err(gpu.fields(), ora.fields()) < MIXED_TOL


@pytest.mark.parametrize("flux_method", ["vanLeer", "WENO5"])
def test_wide_velocity_grid(cuda, flux_method):
    """49 x 49 = 2401 velocities: above the narrow kernels' shared-memory limit,
    so the face pass runs its wide shape (more threads per face)."""
    case = lambda: configs.cavity(n=6, m=48, vlim=5.0, flux_method=flux_method, Kn=0.05, CFL=0.3)
    ora, gpu = run_both(case(), 12)
    assert gpu.blocks[0].Nv == 2401
    assert fields_err(gpu.fields(), ora.fields()) < FP64_TOL
    assert rel_err(gpu.interior_f()[0], ora.interior_f()[0]) < FP64_TOL
    ora, mixed = run_both(case(), 12, precision="mixed")
    assert fields_err(mixed.fields(), ora.fields()) < MIXED_TOL
