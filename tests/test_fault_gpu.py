"""Failure detection without a GPU fault: a NaN is planted on the host.

The reference's only runtime guard is the NaN flag of UGKS_update
(clUGKS.c:1242-1243) read back by get_flag (ugks_block.py:840-876), on which
the run loop stops (ugks_sim.py:597-601).  Here a CPU copy of f gets one NaN,
is uploaded, and the solve is stepped:

* the fused table reports status 1 (ERR_NAN) for that solve, and a second
  solve in the same table is untouched: bit-identical to it running alone;
* the drop-in driver's run loop stops with "nan" at the step the NaN reached
  the update, as the reference's does;
* the serving loop retires the request with reason "error" and serves the
  others to the end.
"""
import numpy as np
import pytest
import torch

from pyugks_b200 import configs
from pyugks_b200.fused import FusedSolver
from pyugks_b200.serving import Request, Server
from pyugks_b200.ugks_sim import UGKSim

pytestmark = pytest.mark.gpu


def _plant_nan(f, G):
    """One NaN in the interior of a distribution tensor, through a host copy."""
    h = f.cpu().numpy()
    h[G + 2, G + 3, 5, 0] = np.nan
    f.copy_(torch.from_numpy(h))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_nan_sets_status_and_spares_other_solves(cuda, precision):
    sick, healthy = configs.cavity(n=8, m=8, vlim=4.0), configs.cavity(n=10, m=8, vlim=4.0, lid=0.2)
    both = FusedSolver([sick, healthy], precision=precision)
    alone = FusedSolver(healthy, precision=precision)
    both.step(3)
    alone.step(3)
    b = both.blocks[both.solve_block_ids(0)[0]]
    _plant_nan(b.f, b.G)
    both.step(4)
    alone.step(4)
    st = both.solve_state()
    assert st[0]["status"] == 1
    assert st[1]["status"] == 0 and alone.solve_state()[0]["status"] == 0
    for x, y in zip(both.interior_f(1), alone.interior_f(0)):
        assert np.array_equal(x, y)
    assert st[1]["dt"] == alone.solve_state()[0]["dt"]


def test_dropin_run_loop_stops_on_nan(cuda):
    sim = UGKSim(configs.cavity(n=8, m=8, vlim=4.0))
    assert sim.run(3) == "max_step"
    b = sim.blocks[0]
    _plant_nan(b.f_D, b.ghost)
    assert sim.run(20) == "nan"
    # the flagged step is not completed: the counter stays where the NaN hit
    assert sim.step == 3


def test_serving_retires_a_failed_request(cuda):
    reqs = [Request(k, 0.0, configs.cavity(n=8, m=8, vlim=4.0, lid=0.1 + 0.05 * k), 60, 0.0) for k in range(3)]
    server = Server(precision="mixed", steps_per_tick=5)
    pool = server.pool
    orig_tick = pool.tick
    planted = []

    def tick_and_fault(n):
        orig_tick(n)
        if not planted and len(pool.solves) == 3:
            # request 1's solve: its one block, through a host copy
            sid = sorted(pool.solves)[1]
            blk = pool.solves[sid].solver.blocks[0]
            _plant_nan(blk.f, blk.G)
            planted.append(sid)

    pool.tick = tick_and_fault
    done = server.run(reqs)
    reasons = {r.id: r.reason for r in done}
    assert reasons == {0: "max_steps", 1: "error", 2: "max_steps"}, reasons


def test_bulk_copy_wait_is_bounded(cuda):
    """The mixed face pass waits on its bulk copies (cp.async.bulk completing
    on an mbarrier) with a bound: a copy that never comes leaves status 8 and
    a usable context, a copy that comes is waited for and lands intact.  The
    wait is made to run out by arming the barrier for bytes nothing sends."""
    from pyugks_b200 import _lib
    L = _lib.lib()
    dev = torch.device("cuda")
    src = torch.arange(128, dtype=torch.float32, device=dev)  # 512 bytes
    status = torch.full((1,), 99, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(L.ugks_check_copy_wait(None, 1000, status.data_ptr(), stream), "ugks_check_copy_wait")
    torch.cuda.synchronize()
    assert int(status.item()) == 8
    _lib.check(L.ugks_check_copy_wait(src.data_ptr(), 1 << 20, status.data_ptr(), stream), "ugks_check_copy_wait")
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    # the context is still usable
    s = FusedSolver(configs.cavity(n=8, m=8, vlim=4.0), precision="mixed")
    s.step(2)
    assert s.solve_state()[0]["status"] == 0


def test_checked_build_matches_and_passes(cuda):
    """The UGKS_CHECKED library (every fused work item checked against its
    block; a failed check would set status 9 and skip the item) runs the same
    steps to bit-identical results with status 0, in both precisions."""
    import os
    import subprocess
    import sys
    from pyugks_b200 import build as B
    if not os.path.exists(B.LIB_CHECKED):
        pytest.fail("libugks_b200_checked.so not built (python -m pyugks_b200.build --checked)")
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "from pyugks_b200 import configs\n"
        "from pyugks_b200.fused import FusedSolver\n"
        "out = {}\n"
        "for prec in ('fp64', 'mixed'):\n"
        "    s = FusedSolver([configs.cavity_multiblock(nb=2, n=8, m=8), configs.channel(nblocks=2, n=8, m=8)],"
        " precision=prec)\n"
        "    s.step(6)\n"
        "    st = s.solve_state()\n"
        "    out[prec] = [int(x['status']) for x in st] + [float(np.sum([f['rho'].sum() + f['T'].sum() for f in"
        " s.fields(k)])) for k in range(2)]\n"
        "print(repr(out))\n") % os.path.dirname(B.HERE)
    runs = []
    for lib in (B.LIB, B.LIB_CHECKED):
        env = dict(os.environ, UGKS_LIB_PATH=lib)
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        runs.append(eval(r.stdout.strip().splitlines()[-1]))
    plain, checked = runs
    for prec in ("fp64", "mixed"):
        assert checked[prec][:2] == [0, 0]
        assert checked[prec] == plain[prec]
