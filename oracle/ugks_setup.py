"""Oracle set-up: CPU restatement of pyUGKS's problem preparation.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``pyugks_b200``) imports
this module; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU arms of
``bench.py`` use it, as the checker.

It turns a *case description* (the plain dict built by
``pyugks_b200.configs``: sizes, boundary conditions, fill, physics constants)
into what the reference's kernels see:

* the Newton-Cotes velocity quadrature (``ugks_data.py:273-299``,
  ``newton_coeff`` ``ugks_data.py:404-417``, ``umax`` ``ugks_data.py:311-312``);
* the constants of the generated OpenCL header, rounded the way
  ``ugks_CL.py:20-400`` prints them (Python-2 ``str()`` keeps 12 significant
  digits, ``%0.15e`` keeps 16);
* the block geometry with ghost cells: ghost vertices by ``xyExtrapolate`` /
  ``xyExchange`` (``source/clGhostRoutines.c:155-398``) and the cell metrics by
  ``cellGeom`` (``source/clKernel.c:31-135``), restated in numpy with the same
  arithmetic order.
"""
from __future__ import annotations

import math

import numpy as np

# face numbering of the block boundary list (geom/geom_defs.py)
NORTH, EAST, SOUTH, WEST = 0, 1, 2, 3
# boundary condition codes (geom/geom_bc_defs.py:27-37)
ADJACENT, EXTRAPOLATE_OUT, CONSTANT, REFLECT, DIFFUSE = 0, 1, 2, 3, 4
PERIODIC, INFLOW, OUTFLOW, ADSORBING, BOUNCE_BACK = 5, 6, 7, 8, 9
# velocity permutations (geom/geom_bc_defs.py:40-43)
NO_FLIP, FLIP_NS, FLIP_D, FLIP_EW = 0, 1, 2, 3
# xy transforms (geom/geom_bc_defs.py:46-48)
NO_TRANSFORM, TRANSFORM, MIRROR = 0, 1, 2

FLUX_METHODS = {"vanLeer": 0, "WENO5": 1, "minmod": 3}


def py2_str(x) -> str:
    """Python-2 ``str()`` of a number, as ``'{}'.format`` prints it in
    ``ugks_CL.py:86-95`` (floats keep 12 significant digits)."""
    if isinstance(x, (bool, np.bool_)):
        return str(int(x))
    if isinstance(x, (int, np.integer)):
        return str(int(x))
    s = "%.12g" % float(x)
    if not any(c in s for c in ".enN"):
        s += ".0"
    return s


def e15(x) -> float:
    """Value after ``'%0.15e' % x`` printing (``ugks_CL.py:84,89,96,318-346``)."""
    return float("%0.15e" % float(x))


def newton_coeff(i: int, n: int) -> float:
    """Newton-Cotes weight, 1-based index (``ugks_data.py:404-417``).
    The end weight is 14/15 exactly as the reference has it."""
    if i == 1 or i == n:
        return 14.0 / 15.0
    if (i - 5) % 4 == 0:
        return 28.0 / 45.0
    if (i - 3) % 4 == 0:
        return 24.0 / 45.0
    return 64.0 / 45.0


def newton_quadrature(q: dict):
    """Tensor Newton grid (``ugks_data.py:273-299``): returns quad (Nv,2),
    weight (Nv,), mirror_NS/EW/D (Nv,) and the rounded point counts."""
    u_num = int(q["u_num"] / 4) * 4 + 1
    v_num = int(q["v_num"] / 4) * 4 + 1
    nv = u_num * v_num
    du = (q["u_max"] - q["u_min"]) / float(u_num - 1)
    dv = (q["v_max"] - q["v_min"]) / float(v_num - 1)
    quad = np.zeros((nv, 2))
    weight = np.zeros(nv)
    index = np.zeros((u_num, v_num), dtype=np.int64)
    count = 0
    for i in range(u_num):
        for j in range(v_num):
            index[i, j] = count
            quad[count, 0] = q["u_min"] + i * du
            quad[count, 1] = q["v_min"] + j * dv
            weight[count] = (newton_coeff(i + 1, u_num) * du) * (newton_coeff(j + 1, v_num) * dv)
            count += 1
    mirror_ns = np.ravel(np.fliplr(index))
    mirror_ew = np.ravel(np.flipud(index))
    mirror_d = np.ravel(np.flipud(np.fliplr(index)))
    return quad, weight, mirror_ns, mirror_ew, mirror_d, u_num, v_num


class Constants:
    """The per-simulation constants the reference bakes into its header."""

    def __init__(self, case: dict):
        q = case["quad"]
        assert q.get("type", "Newton") == "Newton", "only the Newton quadrature is restated"
        quad, weight, mns, mew, md, u_num, v_num = newton_quadrature(q)
        self.u_num, self.v_num = u_num, v_num
        self.Nv = u_num * v_num
        # tables as the header prints them ('%0.15e')
        self.quad = np.vectorize(e15)(quad)
        self.weight = np.vectorize(e15)(weight)
        self.mirror_NS, self.mirror_EW, self.mirror_D = mns, mew, md
        self.flux_method = case["flux_method"]
        self.flux_code = FLUX_METHODS[self.flux_method]
        self.ghost = 3 if self.flux_method == "WENO5" else 2  # ugks_block.py:88-91
        gamma = case["gamma"]
        b = 2.0 / (gamma - 1.0)  # ugks_data.py:367-368
        K = b - 2
        # header text values (ugks_CL.py:84-96)
        self.text = {
            "PI": "%0.15e" % math.pi,
            "Pr": py2_str(case["Pr"]),
            "umax": py2_str(abs(np.max(quad[:, 0]))),
            "vmax": py2_str(abs(np.max(quad[:, 1]))),
            "Kn_eff": "%0.15e" % case["Kn_eff"],
            "gam": py2_str(gamma),
            "B": py2_str(b),
            "K": py2_str(K),
            "OMEGA": py2_str(case["omega"]),
            "RELAX_TYPE": str(int(case["relax_type"])),
            "CFL": "%0.15e" % case["CFL"],
        }
        # the numeric values the kernels compute with
        self.PI = float(self.text["PI"])
        self.Pr = float(self.text["Pr"])
        self.umax = float(self.text["umax"])
        self.vmax = float(self.text["vmax"])
        self.Kn_eff = float(self.text["Kn_eff"])
        self.gam = float(self.text["gam"])
        self.B = float(self.text["B"])
        self.K = float(self.text["K"])
        self.omega = float(self.text["OMEGA"])
        self.relax_type = int(case["relax_type"])
        self.CFL_header = float(self.text["CFL"])
        # host-side values (unrounded) used by the Python driver
        self.CFL = float(case["CFL"])
        self.Kn_eff_host = float(case["Kn_eff"])
        self.delta_dt = float(case.get("delta_dt", 1.0))


def isotherm_tables(adsorb):
    """Tabulated isotherm of an adsorbing face (ugks_CL.py:158-252): points
    (P, T, theta) as printed with %0.15e, padded to (n, 4); the Delaunay
    triangles of (P, T) (scipy.spatial.Delaunay, as the reference) and
    their neighbours, padded to (n_tri, 4) with 0."""
    from scipy.spatial import Delaunay
    a = np.asarray(adsorb, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] != 3:
        raise RuntimeError("Passed in array for isotherm values is not an n*3 array")
    pts = np.zeros((a.shape[0], 4))
    pts[:, :3] = [[e15(x) for x in row] for row in a]
    dl = Delaunay(a[:, 0:2])
    tri = np.zeros((dl.simplices.shape[0], 4), dtype=np.int32)
    nbr = np.zeros((dl.neighbors.shape[0], 4), dtype=np.int32)
    tri[:, :3] = dl.simplices
    nbr[:, :3] = dl.neighbors
    return pts, tri, nbr


def wall_text(bc: dict):
    """WALL_<f>_{D,U,V,T,P} macro bodies for one face (``ugks_CL.py:277-310``)."""
    t = bc["type"]
    if t in (ADSORBING, DIFFUSE, CONSTANT, INFLOW, OUTFLOW):
        d = {
            "D": py2_str(bc.get("D", 0.0)),
            "U": py2_str(bc.get("U", 0.0)),
            "V": py2_str(bc.get("V", 0.0)),
            "T": "1.0/(%s)" % py2_str(bc.get("T", 0.0)),
            "P": py2_str(bc.get("P", 0.0)) if t == OUTFLOW else "-1",
        }
    else:
        d = {k: "-1" for k in "DUVTP"}
    return d


def wall_values(bc: dict):
    """Numeric (D, U, V, lambda-or-T macro, P) as the kernels evaluate them."""
    t = wall_text(bc)
    D = float(t["D"])
    U = float(t["U"])
    V = float(t["V"])
    if t["T"] == "-1":
        T = -1.0
    else:
        T = 1.0 / float(t["T"][5:-1])
    P = float(t["P"])
    return D, U, V, T, P


# ----------------------------------------------------------------------------
# geometry: ghost vertices and cell metrics
# ----------------------------------------------------------------------------

def _rot90(i, j, n, Ni, Nj):
    for _ in range(n):
        i, j = Nj - j - 1, i
        Ni, Nj = Nj, Ni
    return i, j


def swap_index(this_face, i, j, that_face, NI, NJ, NIB, NJB, G, vertex):
    """``getSwapIndex`` (``source/clGhostRoutines.c:47-138``)."""
    adjust_flip, adjust_rot = (0, 1) if vertex else (-1, 0)
    if this_face == EAST:
        if that_face == EAST:
            i = (NI + adjust_flip) - i
            i += NIB - 2 * G
        elif that_face == WEST:
            i -= NI - 2 * G
        elif that_face == NORTH:
            i, j = _rot90(i, j, 3, NI + adjust_rot, NJ + adjust_rot)
            j += NJB - 2 * G
        elif that_face == SOUTH:
            i, j = _rot90(i, j, 1, NI + adjust_rot, NJ + adjust_rot)
            j -= NI - 2 * G
    elif this_face == WEST:
        if that_face == WEST:
            i = (NI + adjust_flip) - i
            i -= NI - 2 * G
        elif that_face == EAST:
            i += NIB - 2 * G
        elif that_face == NORTH:
            i, j = _rot90(i, j, 1, NI + adjust_rot, NJ + adjust_rot)
            j += NJB - 2 * G
        elif that_face == SOUTH:
            i, j = _rot90(i, j, 3, NI + adjust_rot, NJ + adjust_rot)
            j -= NI - 2 * G
    elif this_face == NORTH:
        if that_face == NORTH:
            j = (NJ + adjust_flip) - j
            j += NJB - 2 * G
        elif that_face == SOUTH:
            j -= NJ - 2 * G
        elif that_face == EAST:
            i, j = _rot90(i, j, 1, NI + adjust_rot, NJ + adjust_rot)
            i += NIB - 2 * G
        elif that_face == WEST:
            i, j = _rot90(i, j, 3, NI + adjust_rot, NJ + adjust_rot)
            i -= NJ - 2 * G
    elif this_face == SOUTH:
        if that_face == SOUTH:
            j = (NJ + adjust_flip) - j
            j -= NJ - 2 * G
        elif that_face == NORTH:
            j += NJB - 2 * G
        elif that_face == EAST:
            i, j = _rot90(i, j, 3, NI + adjust_rot, NJ + adjust_rot)
            i += NIB - 2 * G
        elif that_face == WEST:
            i, j = _rot90(i, j, 1, NI + adjust_rot, NJ + adjust_rot)
            i -= NJ - 2 * G
    return i, j


def face_corner_indices(face, NI, NJ, G):
    """Vertex indices of the two corners of a block face (A1, A2)."""
    if face == NORTH:
        return (G, NJ - G), (NI - G, NJ - G)
    if face == EAST:
        return (NI - G, G), (NI - G, NJ - G)
    if face == SOUTH:
        return (G, G), (NI - G, G)
    return (G, G), (G, NJ - G)


def _equal(a, b, tol):
    return abs(a - b) <= tol


def _transform(a0, a1, b0, b1, n):
    """Affine corner map of ``transform`` (``source/clFunctions.c:381-402``)."""
    d1 = abs(a0[0] - a1[0]) * abs(a0[0] - a1[0]) + abs(a0[1] - a1[1]) * abs(a0[1] - a1[1])
    d2 = ((a0[0] - a1[0]) * (a0[0] - a1[0]) + (a0[1] - a1[1]) * (a0[1] - a1[1])) * \
         (abs(b0[0] - b1[0]) * abs(b0[0] - b1[0]) + abs(b0[1] - b1[1]) * abs(b0[1] - b1[1]))
    mx = a0[0] - ((-(a1[0] * ((b0[0] - b1[0]) * (b0[0] - n[0]) + (b0[1] - b1[1]) * (b0[1] - n[1])))
                   + a0[0] * (b0[0] * b0[0] + b1[0] * n[0] - b0[0] * (b1[0] + n[0]) + (b0[1] - b1[1]) * (b0[1] - n[1]))
                   + (a0[1] - a1[1]) * (b0[1] * b1[0] - b0[0] * b1[1] - b0[1] * n[0] + b1[1] * n[0] + b0[0] * n[1] - b1[0] * n[1])) * d1) / d2
    my = a0[1] - ((a0[1] * (b0[0] * b0[0] + b1[0] * n[0] - b0[0] * (b1[0] + n[0]) + (b0[1] - b1[1]) * (b0[1] - n[1]))
                   - a1[1] * (b0[0] * b0[0] + b1[0] * n[0] - b0[0] * (b1[0] + n[0]) + (b0[1] - b1[1]) * (b0[1] - n[1]))
                   + (a0[0] - a1[0]) * (b0[0] * b1[1] - b1[1] * n[0] + b0[1] * (-b1[0] + n[0]) - b0[0] * n[1] + b1[0] * n[1])) * d1) / d2
    return mx, my


def _mirror2d(a, b, p):
    l2 = (b[0] - a[0]) * (b[0] - a[0]) + (b[1] - a[1]) * (b[1] - a[1])
    if l2 == 0.0:
        return p
    t = ((p[0] - a[0]) * (b[0] - a[0]) + (p[1] - a[1]) * (b[1] - a[1])) / l2
    r = (a[0] + t * (b[0] - a[0]), a[1] + t * (b[1] - a[1]))
    return (r[0] + (r[0] - p[0]), r[1] + (r[1] - p[1]))


def xy_extrapolate(xy, face, ni, nj, G):
    """``xyExtrapolate`` (``source/clGhostRoutines.c:291-398``)."""
    NI, NJ = ni + 2 * G, nj + 2 * G
    if face in (NORTH, SOUTH):
        rng = [(a, b) for a in range(ni) for b in range(G)]
    else:
        rng = [(a, b) for a in range(G) for b in range(nj)]
    for (a, b) in rng:
        if face == NORTH:
            gi, gj = a + G, b + NJ - G
            ei, ej = gi, NJ - G - 1
            m = float(gj - ej)
            d1 = m * (xy[ei, ej + 1] - xy[ei, ej])
            d2 = m * (xy[ei + 1, ej + 1] - xy[ei + 1, ej])
            xy[gi, gj] = xy[ei, ej] + d1
            xy[gi + 1, gj] = xy[ei + 1, ej] + d2
            xy[gi + 1, gj + 1] = xy[ei + 1, ej + 1] + d2
            xy[gi, gj + 1] = xy[ei, ej + 1] + d1
        elif face == EAST:
            gi, gj = a + NI - G, b + G
            ei, ej = NI - G - 1, gj
            m = float(gi - ei)
            d1 = m * (xy[ei + 1, ej] - xy[ei, ej])
            d2 = m * (xy[ei + 1, ej + 1] - xy[ei, ej + 1])
            xy[gi, gj] = xy[ei, ej] + d1
            xy[gi + 1, gj] = xy[ei + 1, ej] + d1
            xy[gi + 1, gj + 1] = xy[ei + 1, ej + 1] + d2
            xy[gi, gj + 1] = xy[ei, ej + 1] + d2
        elif face == SOUTH:
            gi, gj = a + G, b
            ei, ej = gi, G
            m = float(ej - gj)
            d1 = m * (xy[ei, ej] - xy[ei, ej + 1])
            d2 = m * (xy[ei + 1, ej] - xy[ei + 1, ej + 1])
            xy[gi, gj] = xy[ei, ej] + d1
            xy[gi + 1, gj] = xy[ei + 1, ej] + d2
            xy[gi + 1, gj + 1] = xy[ei + 1, ej + 1] + d2
            xy[gi, gj + 1] = xy[ei, ej + 1] + d1
        else:
            gi, gj = a, b + G
            ei, ej = G, gj
            m = float(ei - gi)
            d1 = m * (xy[ei, ej] - xy[ei + 1, ej])
            d2 = m * (xy[ei, ej + 1] - xy[ei + 1, ej + 1])
            xy[gi, gj] = xy[ei, ej] + d1
            xy[gi + 1, gj] = xy[ei + 1, ej] + d1
            xy[gi + 1, gj + 1] = xy[ei + 1, ej + 1] + d2
            xy[gi, gj + 1] = xy[ei, ej + 1] + d2


def xy_exchange(xyA, face, xyB, NIB, NJB, that_face, ori, affine, flip_normal, ni, nj, G):
    """``xyExchange`` (``source/clGhostRoutines.c:155-284``)."""
    NI, NJ = ni + 2 * G, nj + 2 * G
    if face in (NORTH, SOUTH):
        rng = [(a, b) for a in range(ni) for b in range(G - 1)]
    else:
        rng = [(a, b) for a in range(G - 1) for b in range(nj)]
    (a1i, a1j), (a2i, a2j) = face_corner_indices(face, NI, NJ, G)
    if flip_normal == 1:
        (a1i, a1j), (a2i, a2j) = (a2i, a2j), (a1i, a1j)
    (b1i, b1j), (b2i, b2j) = face_corner_indices(that_face, NIB, NJB, G)
    A1, A2 = tuple(xyA[a1i, a1j]), tuple(xyA[a2i, a2j])
    B1, B2 = tuple(xyB[b1i, b1j]), tuple(xyB[b2i, b2j])
    misalign = (not _equal(A1[0], B1[0], 1e-12)) or (not _equal(A1[1], B1[1], 1e-12)) or \
               (not _equal(A2[0], B2[0], 1e-12)) or (not _equal(A2[1], B2[1], 1e-12))
    for (a, b) in rng:
        if face == NORTH:
            gi, gj = a + G, b + NJ - G + 1
        elif face == EAST:
            gi, gj = a + NI - G + 1, b + G
        elif face == SOUTH:
            gi, gj = a + G, b
        else:
            gi, gj = a, b + G
        for ii in range(2):
            for jj in range(2):
                iB, jB = gi + ii, gj + jj
                if misalign and ori == 1:
                    if face in (EAST, WEST):
                        jB = NJ - jB
                    else:
                        iB = NI - iB
                iB, jB = swap_index(face, iB, jB, that_face, NI, NJ, NIB, NJB, G, True)
                p = tuple(xyB[iB, jB])
                if affine == NO_TRANSFORM:
                    xyA[gi + ii, gj + jj] = p
                elif affine == MIRROR:
                    xyA[gi + ii, gj + jj] = _mirror2d(A1, A2, p)
                else:
                    xyA[gi + ii, gj + jj] = _transform(A1, A2, B1, B2, p)


def cell_geom(xy):
    """``cellGeom`` (``source/clKernel.c:31-135``) over every cell of the
    ghosted block.  Returns area (Ni,Nj), centre (Ni,Nj,2),
    mid_side (Ni,Nj,2,2), normal (Ni,Nj,2,2), side_length (Ni,Nj,2)."""
    with np.errstate(invalid="ignore", divide="ignore"):
        xA, yA = xy[1:, :-1, 0], xy[1:, :-1, 1]
        xB, yB = xy[1:, 1:, 0], xy[1:, 1:, 1]
        xC, yC = xy[:-1, 1:, 0], xy[:-1, 1:, 1]
        xD, yD = xy[:-1, :-1, 0], xy[:-1, :-1, 1]
        tSx, tSy = xA - xD, yA - yD
        tWx, tWy = xD - xC, yD - yC
        nSx, nSy = -tSy, tSx
        nWx, nWy = -tWy, tWx
        lS_n = np.sqrt(nSx * nSx + nSy * nSy)
        lW_n = np.sqrt(nWx * nWx + nWy * nWy)
        Ni, Nj = xA.shape
        normal = np.empty((Ni, Nj, 2, 2))
        normal[:, :, 0, 0] = nSx / lS_n
        normal[:, :, 0, 1] = nSy / lS_n
        normal[:, :, 1, 0] = nWx / lW_n
        normal[:, :, 1, 1] = nWy / lW_n
        area = 0.5 * ((xB + xA) * (yB - yA) + (xC + xB) * (yC - yB) +
                      (xD + xC) * (yD - yC) + (xA + xD) * (yA - yD))
        cx = 1.0 / (area * 6.0) * ((yB - yA) * (xA * xA + xA * xB + xB * xB) +
                                   (yC - yB) * (xB * xB + xB * xC + xC * xC) +
                                   (yD - yC) * (xC * xC + xC * xD + xD * xD) +
                                   (yA - yD) * (xD * xD + xD * xA + xA * xA))
        cx = np.where(np.abs(cx) > 1.0e6, np.nan, cx)
        cy = -1.0 / (area * 6.0) * ((xB - xA) * (yA * yA + yA * yB + yB * yB) +
                                    (xC - xB) * (yB * yB + yB * yC + yC * yC) +
                                    (xD - xC) * (yC * yC + yC * yD + yD * yD) +
                                    (xA - xD) * (yD * yD + yD * yA + yA * yA))
        cy = np.where(np.abs(cy) > 1.0e6, np.nan, cy)
        centre = np.stack([cx, cy], axis=-1)
        mid = np.empty((Ni, Nj, 2, 2))
        mid[:, :, 0, 0] = 0.5 * (xD + xA)
        mid[:, :, 0, 1] = 0.5 * (yD + yA)
        mid[:, :, 1, 0] = 0.5 * (xD + xC)
        mid[:, :, 1, 1] = 0.5 * (yD + yC)
        length = np.empty((Ni, Nj, 2))
        length[:, :, 0] = np.sqrt((xD - xA) * (xD - xA) + (yD - yA) * (yD - yA))
        length[:, :, 1] = np.sqrt((xC - xD) * (xC - xD) + (yC - yD) * (yC - yD))
    return area, centre, mid, normal, length


def block_geometry(case: dict, G: int):
    """Ghosted vertex arrays and cell metrics of every block, in the order the
    reference builds them (``ugks_sim.py:256-262`` -> ``ugks_block.py:718-838``):
    block by block, faces N, E, S, W, then cellGeom."""
    blocks = case["blocks"]
    xys = []
    for b in blocks:
        ni, nj = b["ni"], b["nj"]
        xy = np.full((ni + 2 * G + 1, nj + 2 * G + 1, 2), np.nan)
        xy[G:G + ni + 1, G:G + nj + 1, 0] = b["x"]
        xy[G:G + ni + 1, G:G + nj + 1, 1] = b["y"]
        xys.append(xy)
    geoms = []
    for bi, b in enumerate(blocks):
        ni, nj = b["ni"], b["nj"]
        for face, bc in enumerate(b["bc"]):
            if bc["type"] == ADJACENT:
                ob = bc["other_block"]
                xy_exchange(xys[bi], face, xys[ob], blocks[ob]["ni"] + 2 * G,
                            blocks[ob]["nj"] + 2 * G, bc["other_face"],
                            bc.get("orientation", 1), bc.get("transform", TRANSFORM),
                            bc.get("flip_normal", 0), ni, nj, G)
            else:
                xy_extrapolate(xys[bi], face, ni, nj, G)
        area, centre, mid, normal, length = cell_geom(xys[bi])
        geoms.append(dict(xy=xys[bi], area=area, centre=centre, mid_side=mid,
                          normal=normal, side_length=length))
    return geoms


def initial_macro(block: dict):
    """Fill arrays (``ugks_block.py:270-331``): macro (ni,nj,4) holding
    (rho, U, V, 1/T) and Q (ni,nj,2)."""
    ni, nj = block["ni"], block["nj"]
    fill = block["fill"]
    macro = np.ones((ni, nj, 4))
    macro[:, :, 0] *= np.asarray(fill.get("D", 1.0), dtype=np.float64)
    macro[:, :, 1] *= np.asarray(fill.get("U", 0.0), dtype=np.float64)
    macro[:, :, 2] *= np.asarray(fill.get("V", 0.0), dtype=np.float64)
    macro[:, :, 3] *= 1.0 / np.asarray(fill.get("T", 1.0), dtype=np.float64)
    Q = np.ones((ni, nj, 2))
    Q[:, :, 0] *= fill.get("qx", 0.0)
    Q[:, :, 1] *= fill.get("qy", 0.0)
    return macro, Q
