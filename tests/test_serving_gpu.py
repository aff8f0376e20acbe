"""Continuous batching: solves join and leave the shared block table between
launches.  A solve's result must be bit-identical alone and in the mix, and a
small request stream must be served to completion with latency statistics."""
import numpy as np
import pytest

from pyugks_b200 import configs
from pyugks_b200.fused import FusedSolver
from pyugks_b200.serving import Request, Server, SolvePool, footprint_bytes

pytestmark = pytest.mark.gpu


def solo(case, steps, precision="fp64"):
    s = FusedSolver(case, precision=precision)
    s.step(steps)
    return s.interior_f(0)


def test_membership_changes_do_not_perturb_solves(cuda):
    a = configs.cavity(n=8, m=8, vlim=4.0, flux_method="WENO5")
    b = configs.channel(nblocks=2, n=8, m=8)
    c = configs.cavity(n=10, m=12, vlim=5.0, flux_method="vanLeer", Kn=0.2)
    pool = SolvePool("fp64")
    ia = pool.admit(a)
    pool.step(4)
    ib = pool.admit(b)
    pool.step(3)
    ic = pool.admit(c)
    pool.step(3)            # a: 10 steps, b: 6, c: 3
    pool.retire(ia)
    pool.step(2)            # b: 8, c: 5
    st = pool.states()
    assert st[ib]["steps"] == 8 and st[ic]["steps"] == 5
    for sid, case, n in ((ib, b, 8), (ic, c, 5)):
        for x, y in zip(pool.interior_f(sid), solo(case, n)):
            np.testing.assert_array_equal(x, y)


def test_server_completes_a_small_stream(cuda):
    reqs = [Request(k, 0.05 * k, configs.cavity(n=8 + 2 * (k % 3), m=8, vlim=4.0,
                                                  flux_method="vanLeer" if k % 2 else "WENO5"),
                    max_steps=60, tol=1e-4) for k in range(6)]
    server = Server(budget_bytes=3 * footprint_bytes(reqs[0].case, "mixed"), precision="mixed",
                    steps_per_tick=20)
    done = server.run(reqs, time_limit=120)
    assert len(done) == 6
    assert all(r.reason in ("converged", "max_steps") for r in done)
    lat = sorted(r.finished - r.arrival for r in done)
    assert lat[0] > 0 and np.percentile(lat, 99) >= np.percentile(lat, 50)
