"""Block connections on the CPU: the oracle's edgeExchange
(oracle/ugks_port.c) against the reference's own kernel compiled for the CPU,
for every pairing of faces, orientation flag, velocity flip and corner
alignment (clGhostRoutines.c:47-138, 407-538).  An index copy, so the two
must agree to the bit."""
import numpy as np
import pytest

import programs
import ugks_setup
from conftest import exchange_args, pairings, square_pair_case


@pytest.mark.parametrize("flux_method", ["vanLeer", "WENO5"])
def test_port_edge_exchange_matches_reference_every_pairing(flux_method):
    case = square_pair_case(flux_method)
    c = ugks_setup.Constants(case)
    blk = case["blocks"][0]
    if not programs.reference_available(c, blk, 0):
        pytest.skip("compiled reference not available")
    port = programs.PortProgram(c, blk, 0)
    ref = programs.RefProgram(c, blk, 0, threads=1)
    G, n = c.ghost, blk["ni"]
    N = n + 2 * G
    rng = np.random.default_rng(11)
    fB = rng.random((N, N, c.Nv, 2))
    for (this, that, ori, flip, aligned) in pairings():
        xyA, xyB = exchange_args(case, G, this, that, aligned)
        g = (n, G) if this in (0, 2) else (G, n)
        fa = rng.random((N, N, c.Nv, 2))
        before, fr = fa.copy(), fa.copy()
        port.edgeExchange(g, fa, xyA, this, fB, xyB, N, N, that, ori, flip)
        ref.edgeExchange(g, fr, xyA, this, fB, xyB, N, N, that, ori, flip)
        assert not np.array_equal(fa, before)  # the ghost strip was written
        assert np.array_equal(fa, fr), (this, that, ori, flip, aligned)
