"""Host side of the mixed-precision storage (no GPU): the reference
Maxwellian table (UGKS_REF_* of include/ugks_b200.h) and the velocity-pair
deviation layout the *_mixed entry points read and write."""
import numpy as np

from pyugks_b200 import _lib, configs
from pyugks_b200.fused import from_pairs, pair_count, reference_state, reference_table, to_pairs
from pyugks_b200.problem import Constants


def _table(case):
    const = Constants(case)
    return const, reference_table(const, *reference_state(case))


def test_reference_state_follows_fill_and_walls():
    assert reference_state(configs.cavity(n=8, m=8, T_wall=1.1)) == (1.0, 1.1)
    rho0, T0 = reference_state(configs.channel(nblocks=2, n=8, m=8))
    assert abs(rho0 - 1.1) < 0.02 and T0 == 1.0


def test_reference_table_moments_and_axis_factors():
    for m in (8, 9, 24):  # odd and even velocity counts
        const, ref = _table(configs.cavity(n=8, m=m, vlim=4.0, T_wall=0.9))
        vg = const.vgrid
        mh = ref[_lib.REF_TAB:_lib.REF_TAB + vg.Nv]
        lam0 = ref[_lib.REF_LAMBDA]
        assert abs(lam0 - 1.0 / 0.9) < 1e-15
        q = vg.quad
        expect = vg.weight * ref[_lib.REF_P0] * np.exp(-lam0 * (q[:, 0] ** 2 + q[:, 1] ** 2))
        assert np.array_equal(mh, expect)
        mom = ref[_lib.REF_MOM:_lib.REF_MOM + 13]
        assert abs(mom[0] - np.sum(mh)) <= 1e-15 * mom[0]
        # symmetric grid: odd moments vanish to round-off
        for k in (1, 2, 4, 6, 7, 8, 9, 11, 12):
            assert abs(mom[k]) < 1e-14 * mom[0]
        Au = ref[_lib.REF_TAB + vg.Nv:_lib.REF_TAB + vg.Nv + vg.u_num]
        Av = ref[_lib.REF_TAB + vg.Nv + vg.u_num:]
        assert np.allclose(np.outer(Au, Av).ravel(), mh, rtol=1e-13, atol=0)


def test_pair_layout_round_trip():
    rng = np.random.default_rng(5)
    for m in (8, 9, 12):  # u_num 9 (odd: padded pair row) and 13
        const, ref = _table(configs.cavity(n=8, m=m, vlim=4.0))
        vg = const.vgrid
        nv, vn = vg.Nv, vg.v_num
        mh = ref[_lib.REF_TAB:_lib.REF_TAB + nv]
        f = np.stack([mh, ref[_lib.REF_KB0] * mh], -1) * (1.0 + 0.1 * rng.standard_normal((3, 4, nv, 2)))
        p = to_pairs(f, ref, vg)
        assert p.dtype == np.float32 and p.shape == (3, 4, pair_count(vg), 4)
        # pair a v_num + jv = (h(2a, jv), h(2a + 1, jv), b(2a, jv), b(2a + 1, jv))
        a, jv = 1, 3
        v0, v1 = 2 * a * vn + jv, (2 * a + 1) * vn + jv
        assert p[1, 2, a * vn + jv, 1] == np.float32(f[1, 2, v1, 0] - mh[v1])
        assert p[1, 2, a * vn + jv, 2] == np.float32(f[1, 2, v0, 1] - ref[_lib.REF_KB0] * mh[v0])
        if vg.u_num & 1:
            assert np.all(p[..., -vn:, 1] == 0) and np.all(p[..., -vn:, 3] == 0)
        g = from_pairs(p, ref, vg)
        # only the deviation is rounded: error relative to the deviation's size
        dev = np.abs(f - np.stack([mh, ref[_lib.REF_KB0] * mh], -1))
        assert np.all(np.abs(g - f) <= 1.2e-7 * dev + 1e-300)
