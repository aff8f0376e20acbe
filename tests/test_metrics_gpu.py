"""Metrics of a running solve and of the serving loop as JSON lines."""
import pytest
import torch

from pyugks_b200 import configs
from pyugks_b200.fused import FusedSolver
from pyugks_b200.metrics import MetricsLog, read
from pyugks_b200.serving import Request, Server

pytestmark = pytest.mark.gpu


def test_solver_step_records(cuda, tmp_path):
    path = str(tmp_path / "m.jsonl")
    s = FusedSolver([configs.cavity(n=12, m=8, vlim=4.0), configs.cavity(n=8, m=8, vlim=4.0, lid=0.2)],
                    precision="mixed")
    log = MetricsLog(path, workload="two cavities")
    log.solver_step(s)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    s.step(20)
    b.record()
    torch.cuda.synchronize()
    log.solver_step(s, device_ms=a.elapsed_time(b))
    log.close()
    recs = read(path)
    assert len(recs) == 4 and {r["solve"] for r in recs} == {0, 1}
    last = [r for r in recs if r["step"] == 20]
    assert len(last) == 2
    for r in last:
        # closed cavities: the bulk mass stays put to round-off
        assert abs(r["mass_drift"]) < 1e-12 and r["status"] == 0
        assert r["cell_vel_per_s"] > 0 and len(r["residual"]) == 4


def test_serving_records(cuda, tmp_path):
    path = str(tmp_path / "s.jsonl")
    reqs = [Request(k, 0.0, configs.cavity(n=8 + 2 * k, m=8, vlim=4.0), max_steps=30, tol=0.0) for k in range(3)]
    with MetricsLog(path, workload="serving") as log:
        done = Server(precision="mixed", steps_per_tick=10).run(reqs, metrics=log)
    recs = read(path)
    got = [r for r in recs if r["kind"] == "request"]
    assert sorted(r["id"] for r in got) == [0, 1, 2] and len(done) == 3
    assert all(r["steps"] == 30 and r["reason"] == "max_steps" for r in got)
    assert any(r["kind"] == "tick" for r in recs)
