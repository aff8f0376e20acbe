"""Host set-up of the product against the oracle's restatement of the
reference preparation (quadrature, header constants, geometry), the case
builders, and known answers that the reference fixes."""
import numpy as np
import pytest

import ugks_setup as us
from pyugks_b200 import configs
from pyugks_b200 import defs as D
from pyugks_b200.problem import Constants, geometry, newton_weight


def test_newton_weights_known_answers():
    # ugks_data.py:404-417: end points 14/15 (not Boole's 14/45), then 64/45,
    # 24/45, 64/45, 28/45 repeating
    n = 9
    w = [newton_weight(i, n) for i in range(1, n + 1)]
    assert w[0] == w[-1] == 14.0 / 15.0
    assert w[1:8] == [64 / 45, 24 / 45, 64 / 45, 28 / 45, 64 / 45, 24 / 45, 64 / 45]


@pytest.mark.parametrize("m,expect", [(24, 25), (32, 33), (16, 17), (48, 49), (8, 9), (25, 25)])
def test_newton_rounding_to_4k_plus_1(m, expect):
    c = Constants(configs.cavity(n=4, m=m))
    assert c.vgrid.u_num == expect and c.Nv == expect * expect


@pytest.mark.parametrize("make", [lambda: configs.cavity(n=8, m=24, vlim=4.0),
                                  lambda: configs.cavity_multiblock(nb=2, n=6, m=16),
                                  lambda: configs.channel(nblocks=3, n=6, m=16, nj=5)])
def test_product_setup_matches_oracle_setup(make):
    case = make()
    a, b = Constants(case), us.Constants(case)
    np.testing.assert_array_equal(a.vgrid.quad, b.quad)
    np.testing.assert_array_equal(a.vgrid.weight, b.weight)
    np.testing.assert_array_equal(a.vgrid.mirror_NS, b.mirror_NS)
    np.testing.assert_array_equal(a.vgrid.mirror_EW, b.mirror_EW)
    np.testing.assert_array_equal(a.vgrid.mirror_D, b.mirror_D)
    for k in ("PI", "Pr", "umax", "vmax", "Kn_eff", "gam", "K", "omega"):
        assert getattr(a, k) == getattr(b, k), k
    ga, gb = geometry(case, a.ghost), us.block_geometry(case, b.ghost)
    for x, y in zip(ga, gb):
        for k in ("xy", "area", "centre", "mid_side", "normal", "side_length"):
            np.testing.assert_array_equal(x[k], y[k], err_msg=k)


def test_header_rounding_of_constants():
    # the generated header prints Pr and gamma with Python-2 str() (12 digits)
    c = Constants(configs.cavity(n=4, m=8))
    assert c.Pr == 0.666666666667 and c.gam == 1.66666666667 and c.K == 1.0


def test_case_builders_are_deterministic():
    a = configs.batched_cavities(8, seed=1)
    b = configs.batched_cavities(8, seed=1)
    assert [(c["blocks"][0]["ni"], c["quad"]["u_num"], c["Kn_eff"]) for c in a] == \
           [(c["blocks"][0]["ni"], c["quad"]["u_num"], c["Kn_eff"]) for c in b]
    r1 = configs.smoothed_density(16, seed=0)
    assert abs(r1.mean() - 1.0) < 0.01 and r1.std() < 0.01


def test_multiblock_connections_are_symmetric():
    case = configs.cavity_multiblock(nb=3, n=4)
    for k, b in enumerate(case["blocks"]):
        for f, bc in enumerate(b["bc"]):
            if bc["type"] == D.ADJACENT:
                o = case["blocks"][bc["other_block"]]["bc"][bc["other_face"]]
                assert o["type"] == D.ADJACENT and o["other_block"] == k and o["other_face"] == f


def test_workload_sizes():
    assert configs.workload_size(configs.cavity(n=32, m=24)) == 32 * 32 * 625
    assert configs.workload_size(configs.cavity_multiblock()) == 128 * 128 * 1089
