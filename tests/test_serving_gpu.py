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


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_ticks_match_eager_ticks(cuda, precision):
    """A tick replayed from a CUDA graph gives the same bits as the same
    launches made one by one."""
    cases = [configs.cavity(n=8, m=8, vlim=4.0, flux_method="WENO5"), configs.channel(nblocks=2, n=8, m=8)]
    pools = [SolvePool(precision, graphs=g) for g in (True, False)]
    ids = [[p.admit(c) for c in cases] for p in pools]
    for p in pools:
        p.tick(5)
        p.tick(5)
    for k in range(len(cases)):
        for x, y in zip(pools[0].interior_f(ids[0][k]), pools[1].interior_f(ids[1][k])):
            np.testing.assert_array_equal(x, y)


def test_fused_solver_capture_matches_step(cuda):
    case = configs.cavity_multiblock(nb=2, n=8, m=8)
    a, b = FusedSolver(case), FusedSolver(case)
    a.capture(6)
    a.replay()
    a.replay()
    b.step(12)
    assert a.solve_state()[0]["steps"] == 12
    for x, y in zip(a.interior_f(), b.interior_f()):
        np.testing.assert_array_equal(x, y)


def test_device_stop_rule(cuda):
    """A solve stops on the device at the step it meets its rule; the others
    in the table go on, unperturbed."""
    pool = SolvePool("fp64")
    capped = pool.admit(configs.cavity(n=8, m=8, vlim=4.0), max_steps=7)
    loose = pool.admit(configs.cavity(n=10, m=8, vlim=4.0), tol=1e-1, start=3)
    early = pool.admit(configs.cavity(n=10, m=8, vlim=4.0), tol=1e3, start=6)
    free = pool.admit(configs.cavity(n=8, m=12, vlim=5.0, flux_method="WENO5"))
    pool.tick(5)
    pool.tick(5)
    st = pool.states()
    assert st[capped]["steps"] == 7 and st[capped]["stopped"] == 2 and not st[capped]["active"]
    assert st[loose]["stopped"] == 1 and st[loose]["residual"][0] < 1e-1 and 3 <= st[loose]["steps"] < 10
    # below its tolerance from the first step, but the rule starts at step 6
    assert st[early]["stopped"] == 1 and st[early]["steps"] == 6
    assert st[free]["steps"] == 10 and st[free]["stopped"] == 0
    for x, y in zip(pool.interior_f(free), solo(configs.cavity(n=8, m=12, vlim=5.0, flux_method="WENO5"), 10)):
        np.testing.assert_array_equal(x, y)


def test_one_at_a_time_arm_same_stop_rule(cuda):
    """The comparison arm serves the same requests to the same stop rule: in
    the same precision each request ends at the same step as in the batch."""
    from pyugks_b200.serving import serve_one_at_a_time
    make = lambda: [Request(k, 0.0, configs.cavity(n=8 + 2 * k, m=8, vlim=4.0, lid=0.1 + 0.05 * k),
                            max_steps=40, tol=2e-3) for k in range(3)]
    server = Server(precision="mixed", steps_per_tick=10)
    done = {r.id: r for r in server.run(make())}
    arm = serve_one_at_a_time(make(), precision="mixed", steps_per_tick=10)
    assert [done[k].steps for k in range(3)] == arm["steps"]
    assert [done[k].reason for k in range(3)] == arm["reasons"]
    assert all(x > 0 for x in arm["latency"]) and arm["value"] > 0
