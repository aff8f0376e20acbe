"""Many independent solves in one block table (uneven grids, velocity grids
and limiters).  Every solve must come out bit-identical to the same solve run
alone -- the batch shares launches, not arithmetic -- and match the oracle."""
import numpy as np
import pytest

import host
from conftest import fields_err
from pyugks_b200 import configs
from pyugks_b200.fused import FusedSolver

pytestmark = pytest.mark.gpu


def mix():
    return [configs.cavity(n=8, m=8, vlim=4.0, flux_method="WENO5", Kn=0.05, lid=0.1),
            configs.cavity(n=12, m=12, vlim=5.0, flux_method="vanLeer", Kn=0.3, lid=0.2, T_wall=1.1),
            configs.cavity_multiblock(nb=2, n=6, m=8, flux_method="vanLeer"),
            configs.cavity(n=10, nj=6, m=16, vlim=5.0, flux_method="WENO5", Kn=0.01, lid=0.25)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_each_solve_same_alone_and_in_the_mix(cuda, precision):
    cases = mix()
    batch = FusedSolver(cases, precision=precision)
    batch.step(12)
    for k, case in enumerate(cases):
        alone = FusedSolver(case, precision=precision)
        alone.step(12)
        assert batch.solve_state()[k]["dt"] == alone.solve_state()[0]["dt"]
        for a, b in zip(batch.interior_f(k), alone.interior_f(0)):
            np.testing.assert_array_equal(a, b)


def test_batch_matches_oracle(cuda):
    cases = mix()
    batch = FusedSolver(cases, precision="fp64")
    batch.step(8)
    for k, case in enumerate(cases):
        ora = host.OracleSim(case, "port")
        for _ in range(8):
            ora.one_step()
        assert fields_err(batch.fields(k), ora.fields()) < 1e-11


def test_inactive_solve_is_frozen(cuda):
    cases = mix()[:2]
    batch = FusedSolver(cases, precision="fp64")
    batch.step(2)
    before = batch.interior_f(1)[0].copy()
    batch.set_active([True, False])
    batch.step(3)
    st = batch.solve_state()
    assert st[0]["steps"] == 5 and st[1]["steps"] == 2
    np.testing.assert_array_equal(batch.interior_f(1)[0], before)
