"""Problem set-up on the host: velocity quadrature, kernel constants, geometry.

Turns a case description (``configs``) into the per-block constants the
kernels use and the ghosted geometry arrays.  Set-up only; none of this runs
per step.

* Newton-Cotes quadrature: ``init_quad`` / ``newton_coeff``
  (``ugks_data.py:273-299, 311-312, 404-417``), including the reference's
  end weight 14/15 and the 4k+1 rounding of the point count.
* Kernel constants are the values the reference's generated OpenCL header
  held (``ugks_CL.py:84-96, 318-346``): it printed Pr, gamma, K, omega, umax
  with Python-2 ``str()`` (12 significant digits) and the velocity tables,
  Kn and CFL with ``%0.15e``; the same rounding is applied here so that both
  codes compute with identical numbers.
* Geometry: ghost vertices by extrapolation or from the neighbour block
  (``xyExtrapolate`` / ``xyExchange``, ``source/clGhostRoutines.c:155-398``),
  then the cell metrics of ``cellGeom`` (``source/clKernel.c:31-135``).
"""
from __future__ import annotations

import math

import numpy as np

from . import defs as D


def _round_py2(x: float) -> float:
    return float("%.12g" % float(x))


def _round_e15(x):
    return np.array([float("%0.15e" % v) for v in np.ravel(x)]).reshape(np.shape(x))


def newton_weight(i: int, n: int) -> float:
    """1-based Newton-Cotes weight of point i of n (``ugks_data.py:404-417``)."""
    if i == 1 or i == n:
        return 14.0 / 15.0
    if (i - 5) % 4 == 0:
        return 28.0 / 45.0
    if (i - 3) % 4 == 0:
        return 24.0 / 45.0
    return 64.0 / 45.0


class VelocityGrid:
    """Tensor Newton grid; velocity index v = iu * v_num + jv (v innermost)."""

    def __init__(self, q: dict):
        if q.get("type", "Newton") != "Newton":
            raise NotImplementedError("only the Newton quadrature is supported")
        self.u_num = int(q["u_num"] / 4) * 4 + 1
        self.v_num = int(q["v_num"] / 4) * 4 + 1
        self.Nv = self.u_num * self.v_num
        du = (q["u_max"] - q["u_min"]) / float(self.u_num - 1)
        dv = (q["v_max"] - q["v_min"]) / float(self.v_num - 1)
        iu = np.arange(self.u_num)
        jv = np.arange(self.v_num)
        u = np.array([q["u_min"] + i * du for i in iu])
        v = np.array([q["v_min"] + j * dv for j in jv])
        wu = np.array([newton_weight(i + 1, self.u_num) * du for i in iu])
        wv = np.array([newton_weight(j + 1, self.v_num) * dv for j in jv])
        self.wu, self.wv = wu, wv      # 1-D weights: weight = wu x wv (before rounding)
        quad = np.empty((self.Nv, 2))
        quad[:, 0] = np.repeat(u, self.v_num)
        quad[:, 1] = np.tile(v, self.u_num)
        weight = (wu[:, None] * wv[None, :]).ravel()
        self.umax_exact = abs(np.max(quad[:, 0]))
        self.vmax_exact = abs(np.max(quad[:, 1]))
        self.quad = _round_e15(quad)
        self.weight = _round_e15(weight)
        idx = np.arange(self.Nv).reshape(self.u_num, self.v_num)
        self.mirror_NS = idx[:, ::-1].ravel().astype(np.int32)   # reflects v
        self.mirror_EW = idx[::-1, :].ravel().astype(np.int32)   # reflects u
        self.mirror_D = idx[::-1, ::-1].ravel().astype(np.int32)


class Constants:
    """Physics constants as the kernels see them."""

    def __init__(self, case: dict):
        self.vgrid = VelocityGrid(case["quad"])
        self.Nv = self.vgrid.Nv
        self.flux_method = case["flux_method"]
        self.flux_code = D.FLUX_METHODS[self.flux_method]
        self.ghost = 3 if self.flux_method == "WENO5" else 2
        gamma = float(case["gamma"])
        b = 2.0 / (gamma - 1.0)
        self.PI = float("%0.15e" % math.pi)
        self.Pr = _round_py2(case["Pr"])
        self.gam = _round_py2(gamma)
        self.K = _round_py2(b - 2)
        self.B = _round_py2(b)
        self.omega = _round_py2(case["omega"])
        self.umax = _round_py2(self.vgrid.umax_exact)
        self.vmax = _round_py2(self.vgrid.vmax_exact)
        self.Kn_eff = float("%0.15e" % case["Kn_eff"])
        self.relax_type = int(case["relax_type"])
        # host-side values of the driver (unrounded)
        self.CFL = float(case["CFL"])
        self.delta_dt = float(case.get("delta_dt", 1.0))


def wall_values(bc: dict):
    """(D, U, V, T-macro, P) of one face as the WALL_* macros evaluate
    (``ugks_CL.py:277-310``): walls, CONSTANT, INFLOW and OUTFLOW carry values,
    other faces -1; the T macro holds 1/T."""
    if bc["type"] in (D.ADSORBING, D.DIFFUSE, D.CONSTANT, D.INFLOW, D.OUTFLOW):
        T = _round_py2(bc.get("T", 0.0))
        return (_round_py2(bc.get("D", 0.0)), _round_py2(bc.get("U", 0.0)),
                _round_py2(bc.get("V", 0.0)), (1.0 / T) if T != 0 else math.inf,
                _round_py2(bc.get("P", 0.0)) if bc["type"] == D.OUTFLOW else -1.0)
    return (-1.0, -1.0, -1.0, -1.0, -1.0)


# ---------------------------------------------------------------------------
# geometry
# ---------------------------------------------------------------------------

def _rot90(i, j, n, Ni, Nj):
    for _ in range(n):
        i, j = Nj - j - 1, i
        Ni, Nj = Nj, Ni
    return i, j


def vertex_swap(this, i, j, that, NI, NJ, NIB, NJB, G):
    """getSwapIndex for vertex indices (``clGhostRoutines.c:47-138``, v=1)."""
    key = (this, that)
    if key == (D.EAST, D.EAST):
        return NI - i + NIB - 2 * G, j
    if key == (D.EAST, D.WEST):
        return i - (NI - 2 * G), j
    if key == (D.EAST, D.NORTH):
        i, j = _rot90(i, j, 3, NI + 1, NJ + 1); return i, j + NJB - 2 * G
    if key == (D.EAST, D.SOUTH):
        i, j = _rot90(i, j, 1, NI + 1, NJ + 1); return i, j - (NI - 2 * G)
    if key == (D.WEST, D.WEST):
        return NI - i - (NI - 2 * G), j
    if key == (D.WEST, D.EAST):
        return i + NIB - 2 * G, j
    if key == (D.WEST, D.NORTH):
        i, j = _rot90(i, j, 1, NI + 1, NJ + 1); return i, j + NJB - 2 * G
    if key == (D.WEST, D.SOUTH):
        i, j = _rot90(i, j, 3, NI + 1, NJ + 1); return i, j - (NI - 2 * G)
    if key == (D.NORTH, D.NORTH):
        return i, NJ - j + NJB - 2 * G
    if key == (D.NORTH, D.SOUTH):
        return i, j - (NJ - 2 * G)
    if key == (D.NORTH, D.EAST):
        i, j = _rot90(i, j, 1, NI + 1, NJ + 1); return i + NIB - 2 * G, j
    if key == (D.NORTH, D.WEST):
        i, j = _rot90(i, j, 3, NI + 1, NJ + 1); return i - (NJ - 2 * G), j
    if key == (D.SOUTH, D.SOUTH):
        return i, NJ - j - (NJ - 2 * G)
    if key == (D.SOUTH, D.NORTH):
        return i, j + NJB - 2 * G
    if key == (D.SOUTH, D.EAST):
        i, j = _rot90(i, j, 3, NI + 1, NJ + 1); return i + NIB - 2 * G, j
    i, j = _rot90(i, j, 1, NI + 1, NJ + 1)
    return i - (NJ - 2 * G), j


def _corners(face, NI, NJ, G):
    return {D.NORTH: ((G, NJ - G), (NI - G, NJ - G)), D.EAST: ((NI - G, G), (NI - G, NJ - G)),
            D.SOUTH: ((G, G), (NI - G, G)), D.WEST: ((G, G), (G, NJ - G))}[face]


def _affine(a0, a1, b0, b1, p):
    """``transform`` (``clFunctions.c:381-402``): the map taking b0->a0, b1->a1."""
    ax, ay = a0
    cx, cy = a1
    bx, by = b0
    ex, ey = b1
    nx, ny = p
    d1 = abs(ax - cx) * abs(ax - cx) + abs(ay - cy) * abs(ay - cy)
    d2 = ((ax - cx) * (ax - cx) + (ay - cy) * (ay - cy)) * \
         (abs(bx - ex) * abs(bx - ex) + abs(by - ey) * abs(by - ey))
    t = bx * bx + ex * nx - bx * (ex + nx) + (by - ey) * (by - ny)
    mx = ax - ((-(cx * ((bx - ex) * (bx - nx) + (by - ey) * (by - ny))) + ax * t +
                (ay - cy) * (by * ex - bx * ey - by * nx + ey * nx + bx * ny - ex * ny)) * d1) / d2
    my = ay - ((ay * t - cy * t +
                (ax - cx) * (bx * ey - ey * nx + by * (-ex + nx) - bx * ny + ex * ny)) * d1) / d2
    return mx, my


def _extrapolate(xy, face, ni, nj, G):
    NI, NJ = ni + 2 * G, nj + 2 * G
    if face == D.NORTH:
        for a in range(ni):
            for b in range(G):
                gi, gj = a + G, b + NJ - G
                ei, ej = gi, NJ - G - 1
                m = float(gj - ej)
                d1 = m * (xy[ei, ej + 1] - xy[ei, ej])
                d2 = m * (xy[ei + 1, ej + 1] - xy[ei + 1, ej])
                xy[gi, gj] = xy[ei, ej] + d1
                xy[gi + 1, gj] = xy[ei + 1, ej] + d2
                xy[gi + 1, gj + 1] = xy[ei + 1, ej + 1] + d2
                xy[gi, gj + 1] = xy[ei, ej + 1] + d1
    elif face == D.SOUTH:
        for a in range(ni):
            for b in range(G):
                gi, gj = a + G, b
                ei, ej = gi, G
                m = float(ej - gj)
                d1 = m * (xy[ei, ej] - xy[ei, ej + 1])
                d2 = m * (xy[ei + 1, ej] - xy[ei + 1, ej + 1])
                xy[gi, gj] = xy[ei, ej] + d1
                xy[gi + 1, gj] = xy[ei + 1, ej] + d2
                xy[gi + 1, gj + 1] = xy[ei + 1, ej + 1] + d2
                xy[gi, gj + 1] = xy[ei, ej + 1] + d1
    elif face == D.EAST:
        for a in range(G):
            for b in range(nj):
                gi, gj = a + NI - G, b + G
                ei, ej = NI - G - 1, gj
                m = float(gi - ei)
                d1 = m * (xy[ei + 1, ej] - xy[ei, ej])
                d2 = m * (xy[ei + 1, ej + 1] - xy[ei, ej + 1])
                xy[gi, gj] = xy[ei, ej] + d1
                xy[gi + 1, gj] = xy[ei + 1, ej] + d1
                xy[gi + 1, gj + 1] = xy[ei + 1, ej + 1] + d2
                xy[gi, gj + 1] = xy[ei, ej + 1] + d2
    else:
        for a in range(G):
            for b in range(nj):
                gi, gj = a, b + G
                ei, ej = G, gj
                m = float(ei - gi)
                d1 = m * (xy[ei, ej] - xy[ei + 1, ej])
                d2 = m * (xy[ei, ej + 1] - xy[ei + 1, ej + 1])
                xy[gi, gj] = xy[ei, ej] + d1
                xy[gi + 1, gj] = xy[ei + 1, ej] + d1
                xy[gi + 1, gj + 1] = xy[ei + 1, ej + 1] + d2
                xy[gi, gj + 1] = xy[ei, ej + 1] + d2


def _exchange(xyA, face, xyB, NIB, NJB, that, bc, ni, nj, G):
    NI, NJ = ni + 2 * G, nj + 2 * G
    (a1, a2) = _corners(face, NI, NJ, G)
    if bc.get("flip_normal", 0) == 1:
        a1, a2 = a2, a1
    (b1, b2) = _corners(that, NIB, NJB, G)
    A1, A2 = tuple(xyA[a1]), tuple(xyA[a2])
    B1, B2 = tuple(xyB[b1]), tuple(xyB[b2])
    mis = not (abs(A1[0] - B1[0]) <= 1e-12 and abs(A1[1] - B1[1]) <= 1e-12 and
               abs(A2[0] - B2[0]) <= 1e-12 and abs(A2[1] - B2[1]) <= 1e-12)
    ori = bc.get("orientation", 1)
    affine = bc.get("transform", D.TRANSFORM)
    if face in (D.NORTH, D.SOUTH):
        items = [(a, b) for a in range(ni) for b in range(G - 1)]
    else:
        items = [(a, b) for a in range(G - 1) for b in range(nj)]
    off = {D.NORTH: (G, NJ - G + 1), D.EAST: (NI - G + 1, G), D.SOUTH: (G, 0), D.WEST: (0, G)}[face]
    for a, b in items:
        gi, gj = a + off[0], b + off[1]
        for ii in (0, 1):
            for jj in (0, 1):
                iB, jB = gi + ii, gj + jj
                if mis and ori == 1:
                    if face in (D.EAST, D.WEST):
                        jB = NJ - jB
                    else:
                        iB = NI - iB
                iB, jB = vertex_swap(face, iB, jB, that, NI, NJ, NIB, NJB, G)
                p = tuple(xyB[iB, jB])
                if affine == D.NO_TRANSFORM:
                    xyA[gi + ii, gj + jj] = p
                elif affine == D.MIRROR:
                    l2 = (A2[0] - A1[0]) ** 2 + (A2[1] - A1[1]) ** 2
                    t = ((p[0] - A1[0]) * (A2[0] - A1[0]) + (p[1] - A1[1]) * (A2[1] - A1[1])) / l2
                    r = (A1[0] + t * (A2[0] - A1[0]), A1[1] + t * (A2[1] - A1[1]))
                    xyA[gi + ii, gj + jj] = (r[0] + (r[0] - p[0]), r[1] + (r[1] - p[1]))
                else:
                    xyA[gi + ii, gj + jj] = _affine(A1, A2, B1, B2, p)


def cell_metrics(xy):
    """cellGeom over the ghosted block: area, centre, mid_side, normal, length."""
    with np.errstate(invalid="ignore", divide="ignore"):
        xA, yA = xy[1:, :-1, 0], xy[1:, :-1, 1]
        xB, yB = xy[1:, 1:, 0], xy[1:, 1:, 1]
        xC, yC = xy[:-1, 1:, 0], xy[:-1, 1:, 1]
        xD, yD = xy[:-1, :-1, 0], xy[:-1, :-1, 1]
        Ni, Nj = xA.shape
        nS = np.stack([-(yA - yD), xA - xD], -1)
        nW = np.stack([-(yD - yC), xD - xC], -1)
        normal = np.empty((Ni, Nj, 2, 2))
        normal[:, :, 0] = nS / np.sqrt(nS[..., 0] * nS[..., 0] + nS[..., 1] * nS[..., 1])[..., None]
        normal[:, :, 1] = nW / np.sqrt(nW[..., 0] * nW[..., 0] + nW[..., 1] * nW[..., 1])[..., None]
        area = 0.5 * ((xB + xA) * (yB - yA) + (xC + xB) * (yC - yB) + (xD + xC) * (yD - yC) +
                      (xA + xD) * (yA - yD))
        cx = 1.0 / (area * 6.0) * ((yB - yA) * (xA * xA + xA * xB + xB * xB) +
                                   (yC - yB) * (xB * xB + xB * xC + xC * xC) +
                                   (yD - yC) * (xC * xC + xC * xD + xD * xD) +
                                   (yA - yD) * (xD * xD + xD * xA + xA * xA))
        cy = -1.0 / (area * 6.0) * ((xB - xA) * (yA * yA + yA * yB + yB * yB) +
                                    (xC - xB) * (yB * yB + yB * yC + yC * yC) +
                                    (xD - xC) * (yC * yC + yC * yD + yD * yD) +
                                    (xA - xD) * (yD * yD + yD * yA + yA * yA))
        centre = np.stack([np.where(np.abs(cx) > 1e6, np.nan, cx),
                           np.where(np.abs(cy) > 1e6, np.nan, cy)], -1)
        mid = np.empty((Ni, Nj, 2, 2))
        mid[:, :, 0] = np.stack([0.5 * (xD + xA), 0.5 * (yD + yA)], -1)
        mid[:, :, 1] = np.stack([0.5 * (xD + xC), 0.5 * (yD + yC)], -1)
        length = np.stack([np.sqrt((xD - xA) * (xD - xA) + (yD - yA) * (yD - yA)),
                           np.sqrt((xC - xD) * (xC - xD) + (yC - yD) * (yC - yD))], -1)
    return area, centre, mid, normal, length


def geometry(case: dict, G: int):
    """Per block dict of xy (Ni+1, Nj+1, 2), area, centre, mid_side, normal,
    side_length, built block by block with faces in the order N, E, S, W."""
    blocks = case["blocks"]
    xys = []
    for b in blocks:
        xy = np.full((b["ni"] + 2 * G + 1, b["nj"] + 2 * G + 1, 2), np.nan)
        xy[G:G + b["ni"] + 1, G:G + b["nj"] + 1, 0] = b["x"]
        xy[G:G + b["ni"] + 1, G:G + b["nj"] + 1, 1] = b["y"]
        xys.append(xy)
    out = []
    for k, b in enumerate(blocks):
        for face, bc in enumerate(b["bc"]):
            if bc["type"] == D.ADJACENT:
                o = bc["other_block"]
                _exchange(xys[k], face, xys[o], blocks[o]["ni"] + 2 * G, blocks[o]["nj"] + 2 * G,
                          bc["other_face"], bc, b["ni"], b["nj"], G)
            else:
                _extrapolate(xys[k], face, b["ni"], b["nj"], G)
        area, centre, mid, normal, length = cell_metrics(xys[k])
        out.append(dict(xy=xys[k], area=area, centre=centre, mid_side=mid, normal=normal,
                        side_length=length))
    return out


def fill_arrays(block: dict):
    """macro (ni,nj,4) = (rho, U, V, 1/T) and Q (ni,nj,2) of the fill
    (``ugks_block.py:270-331``)."""
    ni, nj = block["ni"], block["nj"]
    f = block["fill"]
    macro = np.ones((ni, nj, 4))
    macro[:, :, 0] *= np.asarray(f.get("D", 1.0), dtype=np.float64)
    macro[:, :, 1] *= np.asarray(f.get("U", 0.0), dtype=np.float64)
    macro[:, :, 2] *= np.asarray(f.get("V", 0.0), dtype=np.float64)
    macro[:, :, 3] *= 1.0 / np.asarray(f.get("T", 1.0), dtype=np.float64)
    Q = np.ones((ni, nj, 2))
    Q[:, :, 0] *= f.get("qx", 0.0)
    Q[:, :, 1] *= f.get("qy", 0.0)
    return macro, Q


def isotherm_tables(adsorb):
    """A tabulated isotherm as the generated header holds it
    (ugks_CL.py:158-252): points (P, T, theta) printed with %0.15e, padded to
    (n, 4); the Delaunay triangles of (P, T) (scipy.spatial.Delaunay) and
    their neighbours, padded to (n_tri, 4)."""
    from scipy.spatial import Delaunay
    a = np.asarray(adsorb, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] != 3:
        raise ValueError("an isotherm table is an (n, 3) array of (P, T, theta)")
    pts = np.zeros((a.shape[0], 4))
    pts[:, :3] = np.vectorize(lambda x: float("%0.15e" % x))(a)
    dl = Delaunay(a[:, 0:2])
    tri = np.zeros((dl.simplices.shape[0], 4), dtype=np.int32)
    nbr = np.zeros((dl.neighbors.shape[0], 4), dtype=np.int32)
    tri[:, :3] = dl.simplices
    nbr[:, :3] = dl.neighbors
    return pts, tri, nbr
