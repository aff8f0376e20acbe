"""Mixed precision (FP32 f and face fluxes, FP64 moments / conserved update /
relaxation / dt) against the plain FP64 step: relative L2 error of density,
velocity, temperature and heat flux <= 1e-5 on small versions of every
workload (cavity with each limiter, multi-block WENO5 cavity, adsorbing
channel, a mixed batch)."""
import pytest

from pyugks_b200 import configs
from pyugks_b200.mixed_error import compare

pytestmark = pytest.mark.gpu
L2_TOL = 1e-5


@pytest.mark.parametrize("make", [
    lambda: [configs.cavity(n=16, m=24, vlim=4.0)],
    lambda: [configs.cavity(n=12, m=16, vlim=4.0, flux_method="minmod", CFL=0.5)],
    lambda: [configs.cavity_multiblock(nb=2, n=8, m=16)],
    lambda: [configs.channel(nblocks=2, n=8, m=16)],
    lambda: [configs.cavity(n=12, m=16, vlim=5.0, flux_method="WENO5", Kn=0.01),
             configs.cavity(n=8, nj=10, m=8, vlim=5.0, flux_method="vanLeer", Kn=0.5)],
])
def test_mixed_precision_error_bound(cuda, make):
    for res in compare(make(), steps=50):
        for name, e in res.items():
            assert e["L2"] <= L2_TOL, (name, e)


def test_mixed_precision_batched_sample_1000_steps(cuda):
    """Four solves of the 64-cavity batch (seed 1) in one table for 1000
    steps: the high-Kn solves, whose relaxation is slowest and whose heat
    flux is smallest against the moments it is taken from (0: 48x48 cells,
    Nv 1089, Kn 0.77; 32: 64x64, Nv 625, vanLeer, Kn 0.87; 44: 64x64, Nv 289,
    Kn 0.78; 55: 64x64, Nv 289, Kn 0.68, walls at T 0.85 against the fill's
    1.0).  Every field of every solve within 1e-5 relative L2 of the FP64
    run.  (Earlier, while solve 55 cools from its fill temperature, its
    velocity error passes 1e-5 for a few hundred steps; FP64 itself moves the
    heat flux of solve 44 by 2.3e-5 after 500 steps when f starts perturbed
    by 1e-7.)"""
    batch = configs.batched_cavities(64, seed=1)
    sample = [batch[k] for k in (0, 32, 44, 55)]
    for k, res in enumerate(compare(sample, steps=1000)):
        for name, e in res.items():
            assert e["L2"] <= L2_TOL, (k, name, e)


def _perturbed(solver, rel, seed):
    """f of every interior cell times (1 + rel N(0,1)), on the device."""
    import torch
    gen = torch.Generator(device=solver.device).manual_seed(seed)
    for blk in solver.blocks:
        G = blk.G
        x = blk.f[G:-G, G:-G]
        x.mul_(1.0 + rel * torch.randn(x.shape, generator=gen, device=x.device, dtype=x.dtype))


def test_channel_mixed_error_within_fp64_envelope(cuda):
    """Config 4 (the 256x64 adsorbing channel, Nv 1089) after 2000 steps: the
    mixed run's density, temperature and velocity within 1e-5 of FP64, and its
    heat flux within the FP64 run's own envelope -- the difference between
    FP64 and FP64 started from f perturbed by 1e-7 relative (the size of FP32
    rounding), which the scheme carries to about 2e-4 in q by this step."""
    import bench
    from pyugks_b200.fused import FusedSolver
    from pyugks_b200.mixed_error import errors
    cases = bench.workload("channel")[0]
    hi = FusedSolver(cases, precision="fp64")
    hp = FusedSolver(cases, precision="fp64")
    lo = FusedSolver(cases, precision="mixed")
    _perturbed(hp, 1e-7, 5)
    for s in (hi, hp, lo):
        s.step(2000)
    env = errors(hp.fields(0), hi.fields(0))
    mix = errors(lo.fields(0), hi.fields(0))
    for name in ("rho", "T", "UV"):
        assert mix[name]["L2"] <= L2_TOL, (name, mix[name])
    assert env["q"]["L2"] > 1e-5, env  # the envelope itself is above the tolerance
    assert mix["q"]["L2"] <= env["q"]["L2"], (mix["q"], env["q"])
