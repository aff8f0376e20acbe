"""Checkpoint files and the reference's restart semantics, on the oracle
(CPU): the dataset names of save_hdf / close_HDF5, the Q conversion of
updateHost, and a restart with saved f continuing where the saved run was,
to round-off (the file holds T, so lambda comes back as 1/T;
ugks_sim.py:824-840, ugks_block.py:274-300)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import host  # noqa: E402

from pyugks_b200 import checkpoint, configs  # noqa: E402


def save_oracle(sim, path, with_f=True):
    blocks = []
    for k, b in enumerate(sim.blocks):
        d = b.save_data(with_f)
        blocks.append(checkpoint.block_datasets(k, sim.dt, sim.time, d["macro"], d["Q_ext"], d["wall_prop"],
                                                d["wall_cover"], d["wall_fluxes"], d["f"]))
    checkpoint.write(path, sim.step, blocks, dict(Nv=sim.const.Nv, K=sim.const.K))


def test_dataset_names_and_values(tmp_path):
    sim = host.OracleSim(configs.channel(nblocks=2, n=8, m=8), "port")
    sim.run(3)
    path = str(tmp_path / "ck.npz")
    save_oracle(sim, path)
    with np.load(path) as z:
        keys = set(z.files)
        assert {"final_step", "Nb", "Nv", "K"} <= keys
        for bid in range(2):
            p = "block_%d/" % bid
            assert {p + n for n in ("dt", "time", "rho", "UV", "Q", "T", "f")} <= keys
            for face in checkpoint.FACES:
                for n in ("rho", "U", "V", "T", "cover", "reflected", "adsorbed", "desorbed") + checkpoint.WALL_FLUX_NAMES:
                    assert p + "wall/%s/%s" % (face, n) in keys
        assert int(z["final_step"]) == 3
        b = sim.blocks[1]
        assert np.array_equal(z["block_1/rho"], b.macro[:, :, 0])
        assert np.array_equal(z["block_1/T"], 1.0 / b.macro[:, :, 3])
        assert np.array_equal(z["block_1/f"], b.f)
        # adsorbing south wall: coverage saved
        assert np.array_equal(z["block_1/wall/S/cover"], b.wall_cover[:8, 2, 0])
    data = checkpoint.read(path)
    assert data["final_step"] == 3 and len(data["blocks"]) == 2
    # the file holds T, and 1/(1/lambda) is lambda to an ulp
    assert np.array_equal(data["blocks"][0]["macro"][:, :, :3], sim.blocks[0].macro[:, :, :3])
    assert np.allclose(data["blocks"][0]["macro"][:, :, 3], sim.blocks[0].macro[:, :, 3], rtol=4e-16, atol=0)


def test_restart_with_f_continues_the_run(tmp_path):
    case = lambda: configs.cavity(n=8, m=8, vlim=4.0)
    a = host.OracleSim(case(), "port")
    a.run(12)
    b = host.OracleSim(case(), "port")
    b.run(6)
    path = str(tmp_path / "ck.npz")
    save_oracle(b, path)
    c = host.OracleSim(case(), "port", restart=checkpoint.read(path))
    assert c.step == 6 and c.time == b.time
    c.run(6)
    assert c.step == a.step
    assert abs(c.time - a.time) <= 1e-14 * a.time and abs(c.dt - a.dt) <= 1e-14 * a.dt
    # the restored lambda = 1/T differs from the running one by an ulp
    for x, y in zip(a.fields(), c.fields()):
        for k in x:
            scale = max(np.max(np.abs(x[k])), 1e-300)
            assert np.max(np.abs(x[k] - y[k])) <= 1e-12 * scale, k


def test_restart_without_f_starts_from_equilibrium(tmp_path):
    sim = host.OracleSim(configs.cavity(n=8, m=8, vlim=4.0), "port")
    sim.run(4)
    path = str(tmp_path / "ck.npz")
    save_oracle(sim, path, with_f=False)
    data = checkpoint.read(path)
    assert data["blocks"][0]["f"] is None
    r = host.OracleSim(configs.cavity(n=8, m=8, vlim=4.0), "port", restart=data)
    # f := fEQ(saved macro, saved Q); the macro is then re-taken from the
    # discrete f, which on this coarse 9x9 velocity grid moves rho by a few %
    assert r.step == 4
    saved = data["blocks"][0]["macro"][:, :, 0]
    assert np.max(np.abs(r.blocks[0].macro[:, :, 0] - saved) / saved) < 0.1
    r.run(2)
    assert r.step == 6
