"""Diagnostics on the CPU: the oracle's getInternal and wall interface
distributions against the reference's own kernels compiled for the CPU, and
the run loop's residual exit rules (UGKSim.run, ugks_sim.py:604-645, with
analyse_residual, ugks_sim.py:722-811) on synthetic residual histories."""
import numpy as np
import pytest

import host
import programs
from pyugks_b200 import configs
from pyugks_b200.diagnostics import ResidualMonitor

CASES = {
    "cavity_vanleer": lambda: configs.cavity(n=8, m=8, vlim=4.0),
    "channel_weno5": lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.01, flux_method="WENO5"),
}


def reference_programs(sim):
    out = []
    for k, b in enumerate(sim.case["blocks"]):
        if not programs.reference_available(sim.const, b, k):
            pytest.skip("compiled reference not available")
        out.append(programs.RefProgram(sim.const, b, k))
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_internal_data_and_wall_distributions_match_the_reference(name):
    sim = host.OracleSim(CASES[name](), "port")
    sim.run(4)
    refs = reference_programs(sim)
    for blk, ref in zip(sim.blocks, refs):
        txyz, stress = blk.internal_data()
        port_prg = blk.prg
        blk.prg = ref
        try:
            r_txyz, r_stress = blk.internal_data()
            r_faces = blk.interface_distribution()
        finally:
            blk.prg = port_prg
        np.testing.assert_allclose(txyz, r_txyz, rtol=1e-13, atol=0)
        np.testing.assert_allclose(stress, r_stress, rtol=1e-12, atol=1e-15)
        faces = blk.interface_distribution()
        for k in "NESW":
            np.testing.assert_allclose(faces[k], r_faces[k], rtol=1e-12, atol=1e-15)
        # T is the mean of the directional temperatures weighted by degrees of freedom
        K = sim.const.K
        T = (txyz[..., 0] + txyz[..., 1] + K * txyz[..., 2]) / (2.0 + K)
        np.testing.assert_allclose(txyz[..., 3], T, rtol=1e-12)
        # the flow is not at rest: the stress is not round-off
        assert np.max(np.abs(stress)) > 1e-6


def test_residual_reduction_limit():
    m = ResidualMonitor(min_residual=0.0, res_drop=100.0, residual_start=10)
    for step in range(1, 100):
        why = m.record(step, np.full(4, 10.0 ** (-step / 10.0)))
        if why:
            break
    # first record at step 10 holds 1e-1; a drop of 100 is 1e-3 at step 30
    assert why == "residual reduction limit reached" and step == 30


def test_minimum_residual_needs_every_component():
    m = ResidualMonitor(min_residual=1e-6)
    assert m.record(1, [1e-7, 1e-7, 1e-7, 1e-5]) is None
    # a NaN component (no mass flow through an open system) never passes
    assert m.record(2, [1e-7, 1e-7, 1e-7, np.nan]) is None
    assert m.record(3, [1e-7, 1e-7, 1e-7, 1e-7]) == "minimum residual reached"


def test_slope_is_linear_in_the_power_law_exponent_and_stabilised_exit():
    # interpolation, filtfilt and the difference are linear in log10 R, so
    # R = N^-a gives a slope proportional to a (the reference's resampling
    # clamps the last sample, which biases the end slope low for every a)
    last = {}
    for a in (1.0, 2.0, 4.0):
        m = ResidualMonitor(slope_start=10, min_slope=1e-3)
        for step in range(1, 200):
            assert m.record(step, np.full(3, float(step) ** -a)) is None
        last[a] = np.asarray(m.last_slope)
        assert np.all(last[a] > 1e-3)
    np.testing.assert_allclose(last[2.0], 2.0 * last[1.0], rtol=1e-9)
    np.testing.assert_allclose(last[4.0], 4.0 * last[1.0], rtol=1e-9)
    # before slope_start no slope is taken
    m = ResidualMonitor(slope_start=10, min_slope=1e-3)
    m.record(5, np.ones(2))
    assert m.last_slope == np.inf
    # a flat residual stabilises: two consecutive records under min_slope
    m = ResidualMonitor(slope_start=10, min_slope=1e-3)
    whys = [m.record(step, np.full(2, 1e-4)) for step in range(1, 20)]
    assert whys[:10] == [None] * 10 and whys[10] == "residual stabilised"
