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
