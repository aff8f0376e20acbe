"""Block connections and open faces on the GPU against the oracle.

* The drop-in ugks_edgeExchange for every pairing of faces, orientation flag,
  velocity flip and corner alignment (clGhostRoutines.c:47-138, 407-538):
  bit-exact.
* The fused step's ghost pass (ugks_fused.cu ghost_pass) for all sixteen
  face pairings with both orientation flags and every flip: the block table
  is started from random distributions through the restart path, which
  leaves f as given and fills the ghost layers, and the whole of f must equal
  the oracle's after UGKSBlock.updateBC (bit-exact: index copies).
* The fused ghost pass for the open and copy faces (CONSTANT, INFLOW,
  OUTFLOW, EXTRAPOLATE_OUT, REFLECT, BOUNCE_BACK and the constant-gradient
  ghosts of walls): copies bit-exact, equilibrium ghosts to 1e-14 (exp from
  CUDA against glibc).
"""
import numpy as np
import pytest
import torch

import host
import programs
import ugks_setup
from conftest import FLIPS, exchange_args, pairings, square_pair_case
from pyugks_b200 import configs
from pyugks_b200 import defs as D
from pyugks_b200.desc import VelocityTables, block_desc
from pyugks_b200.fused import FusedSolver
from pyugks_b200.kernel_program import KernelProgram
from pyugks_b200.problem import Constants

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("flux_method", ["vanLeer", "WENO5"])
def test_dropin_edge_exchange_every_pairing(cuda, flux_method):
    case = square_pair_case(flux_method)
    c = ugks_setup.Constants(case)
    blk = case["blocks"][0]
    port = programs.PortProgram(c, blk, 0)
    tabs = VelocityTables(Constants(case), cuda)
    desc = block_desc(Constants(case), blk, tabs)
    gpu = KernelProgram(desc)
    G, n = c.ghost, blk["ni"]
    N = n + 2 * G
    rng = np.random.default_rng(12)
    fB = rng.random((N, N, c.Nv, 2))
    dB = torch.from_numpy(fB).to(cuda)
    for (this, that, ori, flip, aligned) in pairings():
        xyA, xyB = exchange_args(case, G, this, that, aligned)
        g = (n, G) if this in (0, 2) else (G, n)
        fa = rng.random((N, N, c.Nv, 2))
        dA = torch.from_numpy(fa).to(cuda)
        port.edgeExchange(g, fa, xyA, this, fB, xyB, N, N, that, ori, flip)
        gpu.edgeExchange(None, g, None, dA, torch.from_numpy(xyA).to(cuda), this, dB,
                         torch.from_numpy(xyB).to(cuda), N, N, that, ori, flip)
        assert np.array_equal(dA.cpu().numpy(), fa), (this, that, ori, flip, aligned)


def _restart_data(case, G, rng):
    """Random positive distributions (ghost layers included) and a macro
    state near rest for every block, in checkpoint.read's layout."""
    const = Constants(case)
    blocks = []
    for b in case["blocks"]:
        ni, nj = b["ni"], b["nj"]
        macro = np.stack([1.0 + 0.1 * rng.random((ni, nj)), 0.05 * rng.standard_normal((ni, nj)),
                          0.05 * rng.standard_normal((ni, nj)), 1.0 + 0.1 * rng.random((ni, nj))], -1)
        blocks.append(dict(macro=macro, Q=1e-3 * rng.standard_normal((ni, nj, 2)),
                           f=rng.random((ni + 2 * G, nj + 2 * G, const.Nv, 2)), time=0.0, dt=0.0))
    return dict(final_step=0, blocks=blocks)


def _ghost_fill(case, data):
    ora = host.OracleSim(case, "port", restart=data)
    gpu = FusedSolver(case, precision="fp64", restart={0: data})
    torch.cuda.synchronize()
    assert gpu.solve_state()[0]["status"] == 0
    return ora, gpu


@pytest.mark.parametrize("shift", [0, 1, 2, 3])
def test_fused_ghost_pass_every_face_pairing(cuda, shift):
    """Block 0's face f joins block 1's face (f + shift) % 4 and back, with
    the orientation flag and the flip code varying over the faces."""
    links = {}
    for f in range(4):
        o = (f + shift) % 4
        ori, flip = (f + shift) % 2, FLIPS[(f + 2 * shift) % 4]
        links[(0, f)] = (1, o, ori, flip)
        links[(1, o)] = (0, f, 1 - ori, FLIPS[(f + 2 * shift + 1) % 4])
    for flux_method in ("vanLeer", "WENO5"):
        case = square_pair_case(flux_method, links=links)
        G = ugks_setup.Constants(case).ghost
        ora, gpu = _ghost_fill(case, _restart_data(case, G, np.random.default_rng(20 + shift)))
        for k, ob in enumerate(ora.blocks):
            got = gpu.blocks[gpu.solve_block_ids(0)[k]].f.cpu().numpy()
            assert np.array_equal(got, ob.f), (flux_method, shift, k)


@pytest.mark.parametrize("name", ["rotated", "flipped", "mirror", "periodic", "multiblock"])
def test_fused_ghost_pass_physical_connections(cuda, name):
    """The connection cases with aligned corners (rotated, multiblock),
    orientation-flipped ones, self connections through the velocity
    permutations and a PERIODIC face, from random distributions."""
    make = {"rotated": configs.rotated_pair, "flipped": configs.flipped_pair, "mirror": configs.mirror_cavity,
            "periodic": configs.periodic_couette,
            "multiblock": lambda n, m: configs.cavity_multiblock(nb=2, n=n, m=m)}[name]
    case = make(n=8, m=8)
    G = ugks_setup.Constants(case).ghost
    ora, gpu = _ghost_fill(case, _restart_data(case, G, np.random.default_rng(31)))
    for k, ob in enumerate(ora.blocks):
        assert np.array_equal(gpu.blocks[gpu.solve_block_ids(0)[k]].f.cpu().numpy(), ob.f), (name, k)


def test_fused_ghost_pass_open_and_copy_faces(cuda):
    """Block 0: CONSTANT (N), OUTFLOW (E), INFLOW (S), EXTRAPOLATE_OUT (W);
    block 1: REFLECT (N), BOUNCE_BACK (E), a diffuse wall's
    constant-gradient ghosts (S), an adsorbing wall's (W)."""
    case = square_pair_case("WENO5", n=6)
    b0, b1 = case["blocks"]
    b0["bc"] = [configs.constant(1.1, 1.2, U=0.05, V=-0.02), configs.outflow(0.9, 1.0),
                configs.inflow(1.2, 1.0), {"type": D.EXTRAPOLATE_OUT}]
    b1["bc"] = [configs.reflect(), {"type": D.BOUNCE_BACK}, configs.diffuse(1.0),
                configs.adsorbing(1.0, k_des=0.01)]
    G = ugks_setup.Constants(case).ghost
    ora, gpu = _ghost_fill(case, _restart_data(case, G, np.random.default_rng(41)))
    for k, ob in enumerate(ora.blocks):
        got = gpu.blocks[gpu.solve_block_ids(0)[k]].f.cpu().numpy()
        Ni, Nj = ob.Ni, ob.Nj
        strips = {0: (slice(G, Ni - G), slice(Nj - G, Nj)), 1: (slice(Ni - G, Ni), slice(G, Nj - G)),
                  2: (slice(G, Ni - G), slice(0, G)), 3: (slice(0, G), slice(G, Nj - G))}
        for face, bc in enumerate(case["blocks"][k]["bc"]):
            a, b = got[strips[face]], ob.f[strips[face]]
            if bc["type"] in (D.CONSTANT, D.INFLOW, D.OUTFLOW):
                assert np.max(np.abs(a - b)) <= 1e-14 * np.max(np.abs(b)), (k, face)
            else:
                assert np.array_equal(a, b), (k, face, bc["type"])
