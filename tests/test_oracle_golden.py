"""The oracle (plain-C restatement, oracle/ugks_port.c) pinned against golden
vectors produced by the reference's own kernels compiled for the CPU
(tests/golden/make_golden.py).  The restatement reproduces the reference
operation for operation, so the fields agree to the last bit; the bound below
only leaves room for a different libm."""
import os

import numpy as np
import pytest

import host
from conftest import field_errors, rel_err
from pyugks_b200 import configs

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-14

CASES = {
    "cavity8": (lambda: configs.cavity(n=8, m=8, vlim=4.0), (1, 10, 50)),
    "multiblock8": (lambda: configs.cavity_multiblock(nb=2, n=8, m=8), (1, 10, 30)),
    "channel8": (lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.0), (1, 10, 30)),
    "cavity32": (lambda: configs.cavity(n=32, m=24, vlim=4.0), (1, 10)),
    "channel8_specular": (lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.0, reflect_type="S"), (1, 10, 30)),
    "channel8_cl": (lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.0, reflect_type="CL", alpha_n=0.5,
                                            alpha_t=0.7), (1, 10, 30)),
    "channel8_isotherm": (lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.0,
                                                  adsorb=configs.langmuir_table()), (1, 10, 30)),
    "cavity8_minmod": (lambda: configs.cavity(n=8, m=8, vlim=4.0, flux_method="minmod", CFL=0.5), (1, 10, 50)),
    "rotated8": (lambda: configs.rotated_pair(n=8, m=8), (1, 10, 30)),
    "flipped8": (lambda: configs.flipped_pair(n=8, m=8), (1, 10, 30)),
    "mirror8": (lambda: configs.mirror_cavity(n=8, m=8), (1, 10, 30)),
    "periodic8": (lambda: configs.periodic_couette(n=8, m=8), (1, 10, 30)),
    "open8": (lambda: configs.open_channel(n=8, m=8), (1, 10, 30)),
}
# the Cercignani-Lampis kernel's Bessel I0: a power series in the port, a
# rational approximation in the reference
CASE_TOL = {"channel8_cl": 1e-12}


@pytest.mark.parametrize("name", sorted(CASES))
def test_port_matches_reference_golden(name):
    make, steps = CASES[name]
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    sim = host.OracleSim(make(), "port")
    done = 0
    for s in steps:
        while done < s:
            sim.one_step()
            done += 1
        assert abs(sim.dt - float(g["s%d_dt" % s])) == 0.0
        assert abs(sim.time - float(g["s%d_time" % s])) <= 1e-15 * sim.time
        for k, fl in enumerate(sim.fields()):
            gold = {key: g["s%d_b%d_%s" % (s, k, key)] for key in fl}
            errs = field_errors(fl, gold)
            assert max(errs.values()) <= CASE_TOL.get(name, TOL), (name, s, k, errs)
        key = "s%d_b0_f" % s
        if key in g:
            for k, f in enumerate(sim.interior_f()):
                assert rel_err(f, g["s%d_b%d_f" % (s, k)]) <= CASE_TOL.get(name, TOL)
                assert rel_err(sim.blocks[k].wall_cover, g["s%d_b%d_cover" % (s, k)]) <= CASE_TOL.get(name, TOL)


def test_reference_build_matches_port_when_sources_present():
    """Direct A/B of the compiled reference and the port (needs the sources
    or prebuilt libraries in oracle/_ref)."""
    import programs
    import ugks_setup
    case = configs.cavity(n=8, m=8, vlim=4.0)
    c = ugks_setup.Constants(case)
    if not programs.reference_available(c, case["blocks"][0], 0):
        pytest.skip("compiled reference not available")
    a = host.OracleSim(case, "port")
    b = host.OracleSim(case, "ref", threads=2)
    for _ in range(5):
        a.one_step()
        b.one_step()
    np.testing.assert_array_equal(a.interior_f()[0], b.interior_f()[0])
