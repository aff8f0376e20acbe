"""Host-side validation of a fused block table (ugks_fused_layout), with no
GPU: a corrupted entry -- sizes that disagree with the ghost layers or the
limiter's stencil, a missing array, a connection outside the table or to a
face of another extent -- is rejected (-3) before any kernel could index
outside its arrays; the ordering rules give -2.  Pointers are placeholders:
the layout only checks and counts, it never dereferences them."""
import ctypes as C

import pytest

from pyugks_b200 import _lib
from pyugks_b200 import defs as D

FAKE = 0x10000


def block(solve=0, ni=8, nj=8, method=1, ghost=3, m=9):
    x = _lib.FusedBlock()
    d = x.d
    d.ni, d.nj, d.ghost = ni, nj, ghost
    d.Ni, d.Nj = ni + 2 * ghost, nj + 2 * ghost
    d.u_num, d.v_num, d.Nv = m, m, m * m
    d.flux_method = method
    d.quad = d.weight = d.mirror_NS = d.mirror_EW = d.mirror_D = FAKE
    for name in ("f", "flux_S", "flux_W", "flux_macro_S", "flux_macro_W", "macro", "Q", "prim_old", "area",
                 "centre", "mid_side", "normal", "side_length", "xy", "wall_prop", "wall_cover", "wall_fluxes",
                 "wall_dist", "cell_mom", "Q_next", "face_geo"):
        setattr(x, name, FAKE)
    x.solve = solve
    for f in range(4):
        x.bc_type[f] = D.DIFFUSE
    return x


def pair():
    """Two blocks of one solve joined east-west."""
    a, b = block(), block()
    a.bc_type[D.EAST], a.bc_block[D.EAST], a.bc_face[D.EAST] = D.ADJACENT, 1, D.WEST
    b.bc_type[D.WEST], b.bc_block[D.WEST], b.bc_face[D.WEST] = D.ADJACENT, 0, D.EAST
    return [a, b]


def layout(blocks):
    arr = (_lib.FusedBlock * len(blocks))(*blocks)
    z = _lib.FusedSizes()
    rc = _lib.lib().ugks_fused_layout(arr, len(blocks), C.byref(z))
    return rc, z


def test_valid_table():
    rc, z = layout(pair())
    assert rc == 0
    assert z.n_cells == 128 and z.n_faces == 2 * 2 * 9 * 9 and z.n_wall == 2 * 2 * 16


@pytest.mark.parametrize("corrupt", [
    lambda t: setattr(t[0].d, "ghost", 2),                          # WENO5 needs 3 ghost layers
    lambda t: setattr(t[1].d, "Ni", t[1].d.Ni + 1),                 # Ni != ni + 2 ghost
    lambda t: setattr(t[0].d, "ni", 0),
    lambda t: setattr(t[0].d, "Nv", 80),                             # u_num * v_num != Nv
    lambda t: setattr(t[1], "f", None),                              # a missing array
    lambda t: setattr(t[0].d, "quad", None),                         # a missing table
    lambda t: t[0].bc_block.__setitem__(D.EAST, 7),                  # neighbour outside the table
    lambda t: t[0].bc_face.__setitem__(D.EAST, 9),                   # no such face
    lambda t: (setattr(t[1].d, "nj", 10), setattr(t[1].d, "Nj", 16)),  # joined faces of other extents
    lambda t: t[0].bc_type.__setitem__(D.NORTH, 42),                 # unknown boundary code
])
def test_corrupted_entry_is_rejected(corrupt):
    t = pair()
    corrupt(t)
    assert layout(t)[0] == -3


def test_ordering_rules():
    a, b = block(solve=0), block(solve=2)
    assert layout([a, b])[0] == -2                                   # solves not contiguous
    c, e, g = block(solve=0, method=1), block(solve=1, method=0, ghost=2), block(solve=2, method=1)
    assert layout([c, e, g])[0] == -2                                # limiter runs not contiguous
