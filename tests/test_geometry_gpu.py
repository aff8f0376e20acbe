"""Curvilinear blocks on the GPU: the geometry set-up kernels (ugks_xyExchange,
ugks_xyExtrapolate, ugks_cellGeom) against the host restatement, which the
CPU suite pins to the reference's own kernels; and the fused and drop-in time
steps on warped grids (face normals off the axes, curved block interfaces)
against the oracle."""
import numpy as np
import pytest

import host
from conftest import fields_err, rel_err
from pyugks_b200 import configs
from pyugks_b200.fused import FusedSolver
from pyugks_b200.geometry import device_geometry
from pyugks_b200.problem import Constants, geometry
from pyugks_b200.ugks_sim import UGKSim

pytestmark = pytest.mark.gpu
FP64_TOL = 1e-11

CASES = {
    "warped_1x1": lambda: configs.warped_cavity(nb=1, n=8, m=8),
    "warped_2x2_weno": lambda: configs.warped_cavity(nb=2, n=8, m=8, flux_method="WENO5", vlim=5.0),
    "cartesian_2x2": lambda: configs.cavity_multiblock(nb=2, n=8, m=8),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_geometry_matches_host(cuda, name):
    case = CASES[name]()
    dev = device_geometry(case)
    ref = geometry(case, Constants(case).ghost)
    for d, h in zip(dev, ref):
        for key in ("xy", "area", "centre", "mid_side", "normal", "side_length"):
            a, b = np.asarray(d[key]), np.asarray(h[key])
            assert np.array_equal(np.isnan(a), np.isnan(b)), (name, key)
            assert np.array_equal(np.nan_to_num(a), np.nan_to_num(b)), (name, key)


@pytest.mark.parametrize("name", ["warped_1x1", "warped_2x2_weno"])
def test_fused_step_on_warped_grid(cuda, name):
    case = CASES[name]()
    ora = host.OracleSim(case, "port")
    gpu = FusedSolver(case, precision="fp64")
    for _ in range(15):
        ora.one_step()
    gpu.step(15)
    assert gpu.solve_state()[0]["status"] == 0
    assert fields_err(gpu.fields(), ora.fields()) < FP64_TOL
    for a, b in zip(gpu.interior_f(), ora.interior_f()):
        assert rel_err(a, b) < FP64_TOL


def test_dropin_driver_with_device_geometry_on_warped_grid(cuda):
    case = CASES["warped_2x2_weno"]()
    ora = host.OracleSim(case, "port")
    gpu = UGKSim(case, device_geometry=True)
    for _ in range(10):
        ora.one_step()
        gpu.one_step()
    assert fields_err(gpu.fields(), ora.fields()) < FP64_TOL
