"""ugks_getDT_noalloc: the time-step frequency for callers that cannot
allocate device memory.

Some hosts of this solver may not call cudaMalloc while they drive it (a
runtime that forbids allocation inside its time loop, or one that works from a
fixed memory plan).  For them the library offers the block's maximum CFL
frequency with the per-cell frequencies kept in a static array of the library
(at most NOALLOC_MAX_CELLS cells) instead of a caller buffer.  These tests call
it through the C ABI and check it against the two-call form the drop-in driver
uses (ugks_clFindDT into a caller buffer, then ugks_array_max), on two calls in
a row and after a call on a differently sized block, since every call shares
the array.  This file is collected last so that a failure here stops a run
only after every other test has run.
"""
import ctypes as C

import pytest
import torch

from pyugks_b200 import _lib, configs
from pyugks_b200.ugks_sim import UGKSim

pytestmark = pytest.mark.gpu
TOL = 1e-12


def two_call_frequency(L, blk, Kn):
    ts = torch.zeros((blk.ni, blk.nj), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(L.ugks_clFindDT(C.byref(blk.desc), blk.ni, blk.nj, blk.xy_D.data_ptr(),
                               blk.area_D.data_ptr(), blk.macro_D.data_ptr(), ts.data_ptr(), Kn, s),
               "ugks_clFindDT")
    _lib.check(L.ugks_array_max(ts.data_ptr(), ts.numel(), out.data_ptr(), s), "ugks_array_max")
    return float(out.cpu())


def noalloc_frequency(L, blk, Kn):
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    rc = L.ugks_getDT_noalloc(C.byref(blk.desc), blk.xy_D.data_ptr(), blk.area_D.data_ptr(),
                              blk.macro_D.data_ptr(), Kn, out.data_ptr(),
                              torch.cuda.current_stream().cuda_stream)
    assert rc == 0, rc
    return float(out.cpu())


def test_noalloc_frequency_matches_two_call_form(cuda):
    L = _lib.lib()
    big = UGKSim(configs.cavity(n=32, m=24, vlim=4.0))
    small = UGKSim(configs.cavity_multiblock(nb=2, n=8, m=8))
    for sim in (big, small):
        for _ in range(3):
            sim.one_step()
    for sim in (big, small, big):  # a smaller block between two calls on the larger one
        for blk in sim.blocks:
            ref = two_call_frequency(L, blk, sim.Kn_eff)
            for _ in range(2):  # two calls in a row share the array
                got = noalloc_frequency(L, blk, sim.Kn_eff)
                assert abs(got - ref) <= TOL * ref, (got, ref)
                assert sim.CFL / got == pytest.approx(blk.max_dt, rel=1e-3)


def test_noalloc_rejects_blocks_beyond_the_limit(cuda):
    L = _lib.lib()
    d = _lib.BlockDesc()
    d.ni, d.nj = 2048, _lib.NOALLOC_MAX_CELLS // 2048 + 1
    d.ghost, d.Ni, d.Nj = 2, d.ni + 4, d.nj + 4
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = L.ugks_getDT_noalloc(C.byref(d), None, None, None, 0.1, out.data_ptr(), None)
    assert rc == _lib.ERR_TOO_LARGE
    d.ni = 0
    assert L.ugks_getDT_noalloc(C.byref(d), None, None, None, 0.1, out.data_ptr(), None) == _lib.ERR_BAD_SIZE
