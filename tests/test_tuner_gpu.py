"""The launch-shape autotuner: every compiled face and cell shape gives the
oracle's result (the shape only reorders per-face sums), a tuned choice is
cached and reused without timing."""
import pytest

import host
from conftest import fields_err
from pyugks_b200 import configs, tuner
from pyugks_b200.fused import FusedSolver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("face", [1, 2, 3, 4])
def test_every_shape_matches_the_oracle(cuda, face):
    case = configs.cavity_multiblock(nb=2, n=8, m=8)
    ora = host.OracleSim(case, "port")
    for _ in range(10):
        ora.one_step()
    gpu = FusedSolver(case, precision="fp64")
    for k in range(gpu.sizes.n_segments):
        gpu.sizes.seg_variant[k] = face
    gpu.sizes.cell_variant = 2 if face % 2 else 3
    gpu.step(10)
    assert fields_err(gpu.fields(), ora.fields()) < 1e-11
    mixed = FusedSolver(case, precision="mixed")
    for k in range(mixed.sizes.n_segments):
        mixed.sizes.seg_variant[k] = face
    mixed.step(10)
    assert fields_err(mixed.fields(), ora.fields()) < 1e-5


def test_tune_caches_and_reuses(cuda, tmp_path, monkeypatch):
    monkeypatch.setenv("UGKS_TUNE_CACHE", str(tmp_path / "shapes.json"))
    cases = [configs.cavity(n=8, m=8, vlim=4.0), configs.cavity(n=8, m=16, vlim=5.0, flux_method="WENO5")]
    a = FusedSolver(cases, precision="mixed", tune=True)
    assert a.shapes["timed"]
    assert set(a.shapes["face"].values()) <= set(tuner.FACE_SHAPES) and a.shapes["cell"] in tuner.CELL_SHAPES
    assert len(a.shapes["face"]) == len(tuner.segments(a.sizes)) == 2
    b = FusedSolver(cases, precision="mixed", tune=True)
    assert not b.shapes["timed"] and b.shapes["face"] == a.shapes["face"]
    assert [b.sizes.seg_variant[k] for k in range(2)] == [a.shapes["face"][k] for k in range(2)]
    b.step(5)
    assert b.solve_state()[0]["status"] == 0
