"""The JSON-lines metrics log: records carry their kind, wall-clock time and
the log's context, one parseable object per line."""
import json

from pyugks_b200.metrics import MetricsLog, read


class _Req:
    id, arrival, admitted, finished, steps, reason, units = 3, 0.5, 0.6, 2.5, 40, "converged", 1000


def test_records_round_trip(tmp_path):
    path = tmp_path / "m.jsonl"
    with MetricsLog(str(path), workload="cavity", precision="mixed") as log:
        log.write("note", a=1, b=[1.0, 2.0])
        log.request(_Req())
        log.tick(1.25, running=4, backlog=2, used_bytes=1e9, budget_bytes=150e9, units=123)
    recs = read(str(path))
    assert [r["kind"] for r in recs] == ["note", "request", "tick"]
    assert all(r["workload"] == "cavity" and r["precision"] == "mixed" and r["t"] > 0 for r in recs)
    assert recs[1]["latency"] == 2.0 and recs[1]["work"] == 40000 and recs[1]["reason"] == "converged"
    assert recs[2]["running"] == 4 and recs[2]["backlog"] == 2
    # one object per line
    for line in path.read_text().splitlines():
        json.loads(line)


def test_appends_to_an_existing_log(tmp_path):
    path = tmp_path / "m.jsonl"
    for k in range(2):
        with MetricsLog(str(path), run=k) as log:
            log.write("bench", value=float(k))
    assert [r["run"] for r in read(str(path))] == [0, 1]
