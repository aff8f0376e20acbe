"""Case descriptions: the problems the solver runs, as plain data.

A *case* is a dict holding everything a pyUGKS job file would set for the
time-step path (``ugks_data.py:146-235`` defaults, ``Block2D`` /
``connect_blocks_2D`` / ``*BC`` objects of ``geom/``): physics constants, the
velocity quadrature, and per block its vertex grid, four boundary conditions
and fill.  All values are non-dimensional (reference density, temperature and
length of 1; velocities in units of the most probable speed sqrt(2RT_ref),
``ugks_data.py:362``).

``cavity`` and ``channel`` build the workloads this package is measured on:

CFL: the 32x32 cavity states 0.8; the other workloads state none.  They run at
WORKLOAD_CFL = 0.2, below the reference's default of 0.3 (``ugks_data.py:166``):
with WENO5 the reference scheme diverges at 0.3 on the 2x2-block cavity (its own
kernels, compiled for the CPU, raise the NaN flag at step 1164 of the 2000) and
at 0.8 within ~150 steps, while at 0.2 the 2x2-block cavity (2000 steps), the
channel (5000) and all 64 batched cavities (2000) stay bounded.  The small
builders' defaults (the golden-vector cases) keep 0.3.

* ``cavity(32, 24, ...)``: lid-driven cavity, 32x32 cells, 24x24 velocities on
  [-4,4]^2 (rounded by the Newton rule to 25x25 = 625), vanLeer, Kn 0.075,
  CFL 0.8, diffuse walls at T=1 with the lid at U=0.15;
* ``cavity_multiblock(...)``: the same cavity as 2x2 blocks of 64x64 cells,
  33x33 velocities on [-5,5]^2, WENO5, Kn 0.01, density 1 + 0.01 N(0,1)
  smoothed by three 3x3 box passes (seed 0);
* ``batched_cavities(64, seed=1)``: 64 independent cavities with drawn sizes
  and parameters;
* ``channel(...)``: 256x64 pressure-driven channel in 4 blocks with an
  adsorbing lower wall.
"""
from __future__ import annotations

import numpy as np

from . import defs as D


WORKLOAD_CFL = 0.2


def uniform_grid(ni, nj, x0=0.0, x1=1.0, y0=0.0, y1=1.0):
    """Vertex coordinates (ni+1, nj+1) of a uniform Cartesian block; the
    reference's StructuredGrid layout (``geom/geom_grid.py:61-69``)."""
    i = np.arange(ni + 1, dtype=np.float64)[:, None]
    j = np.arange(nj + 1, dtype=np.float64)[None, :]
    x = x0 + (x1 - x0) * (i / ni) + 0.0 * j
    y = y0 + (y1 - y0) * (j / nj) + 0.0 * i
    return np.ascontiguousarray(x), np.ascontiguousarray(y)


def diffuse(T=1.0, U=0.0, V=0.0, D_=1.0):
    """``DiffuseBC`` (``geom/geom_bc_defs.py:316-353``); U, V are global x/y."""
    return dict(type=D.DIFFUSE, D=D_, T=T, U=U, V=V)


def adjacent(other_block, other_face, orientation=1, flip=D.NO_FLIP):
    """``AdjacentBC`` (``geom/geom_bc_defs.py:198-217``)."""
    return dict(type=D.ADJACENT, other_block=other_block, other_face=other_face,
                orientation=orientation, flip=flip, transform=D.TRANSFORM, flip_normal=0)


def inflow(D_=1.0, T=1.0):
    """``InflowBC`` (``geom/geom_bc_defs.py:416-429``)."""
    return dict(type=D.INFLOW, D=D_, T=T, U=0.0, V=0.0)


def constant(D_=1.0, T=1.0, U=0.0, V=0.0):
    """``ConstantBC`` (``geom/geom_bc_defs.py:262-290``): ghosts hold
    fEQ(D, U, V, T), U and V global x/y."""
    return dict(type=D.CONSTANT, D=D_, T=T, U=U, V=V)


def outflow(P=1.0, D_=1.0, T=1.0):
    """``OutflowBC`` (``geom/geom_bc_defs.py:431-444``) with its D set as
    well: the wall value P/D becomes the ghost's lambda = rho_cell / (D / (P/D))
    (``clGhostRoutines.c:755-839``).  The class itself leaves D at 0, which
    makes that lambda infinite, so a usable outflow face sets D too."""
    return dict(type=D.OUTFLOW, D=D_, T=T, U=0.0, V=0.0, P=P)


def periodic(other_block, other_face, orientation=0, flip=D.NO_FLIP):
    """A PERIODIC face (BC code 5): copied through ``edgeExchange`` like an
    ADJACENT one; its ghost vertices are extrapolated (``ugks_block.py:726-733``).
    orientation 0 (HOLD) keeps the along-face order although the two faces'
    corners lie apart."""
    return dict(type=D.PERIODIC, other_block=other_block, other_face=other_face,
                orientation=orientation, flip=flip, transform=D.TRANSFORM, flip_normal=0)


def reflect():
    return dict(type=D.REFLECT)


def adsorbing(T=1.0, gamma_f=0.5, k_des=0.01, adsorb=0.5, S_T=1.0, reflect_type="D",
              cover_initial=0.0, beta_n=0.0, beta_t=0.0, alpha_n=1.0, alpha_t=1.0):
    """``AdsorbingBC`` (``geom/geom_bc_defs.py:355-414``) with the extra
    first-order desorption rate ``k_des`` (per unit time; 0 restores the
    reference's Langmuir-driven desorption, which needs ``adsorb``).  With
    reference values of 1, ``alpha_p = 1/S_T`` and ``gamma_f = S_T k_f``
    (``ugks_data.py:516-518``).  ``reflect_type`` re-emits the reflected flux
    specularly ('S', the reference's default), diffusely ('D') or through
    the Cercignani-Lampis kernel ('CL', accommodation ``alpha_n``,
    ``alpha_t``)."""
    return dict(type=D.ADSORBING, D=1.0, T=T, U=0.0, V=0.0, gamma_f=gamma_f, alpha_p=1.0 / S_T,
                S_T=S_T, beta_n=beta_n, beta_t=beta_t, adsorb=adsorb, dynamic=1,
                reflect_type=reflect_type, cover_initial=cover_initial, k_des=k_des,
                alpha_n=alpha_n, alpha_t=alpha_t)


def langmuir_table(K0=2.0, E=0.5, n_p=7, n_t=5, p_range=(0.05, 2.5), t_range=(0.5, 2.0), seed=3):
    """A tabulated isotherm for ``adsorbing(adsorb=...)``: points (P, T,
    theta) of the Langmuir form theta = K P / (1 + K P), K = K0 exp(E / T), on
    a slightly jittered P x T grid (jitter keeps the Delaunay triangulation
    of the points unique)."""
    rng = np.random.default_rng(seed)
    P, T = np.meshgrid(np.linspace(*p_range, n_p), np.linspace(*t_range, n_t), indexing="ij")
    dp = (p_range[1] - p_range[0]) / (n_p - 1)
    dt = (t_range[1] - t_range[0]) / (n_t - 1)
    P = P + 0.05 * dp * rng.standard_normal(P.shape)
    T = T + 0.05 * dt * rng.standard_normal(T.shape)
    K = K0 * np.exp(E / T)
    return np.stack([P.ravel(), T.ravel(), (K * P / (1.0 + K * P)).ravel()], axis=1)


def base_case(flux_method, Kn, m, vlim, CFL=0.8):
    return dict(flux_method=flux_method, CFL=CFL, Pr=2.0 / 3.0, gamma=5.0 / 3.0, omega=0.81,
                Kn_eff=Kn, relax_type=2, delta_dt=1.0,
                quad=dict(type="Newton", u_num=m, v_num=m, u_min=-vlim, u_max=vlim,
                          v_min=-vlim, v_max=vlim),
                blocks=[])


def cavity(n=32, m=24, vlim=4.0, flux_method="vanLeer", Kn=0.075, lid=0.15, T_wall=1.0,
           CFL=0.8, rho=1.0, nj=None):
    """Single-block lid-driven cavity on the unit square."""
    nj = n if nj is None else nj
    case = base_case(flux_method, Kn, m, vlim, CFL)
    x, y = uniform_grid(n, nj)
    case["blocks"].append(dict(
        ni=n, nj=nj, x=x, y=y,
        bc=[diffuse(T_wall, U=lid), diffuse(T_wall), diffuse(T_wall), diffuse(T_wall)],
        fill=dict(D=rho, U=0.0, V=0.0, T=1.0, qx=0.0, qy=0.0)))
    return case


def smoothed_density(n, seed=0, amp=0.01, passes=3):
    """1 + amp*N(0,1) per cell, smoothed by box-filter passes with edge
    replication; index [i, j] with i along x."""
    rho = 1.0 + amp * np.random.default_rng(seed).standard_normal((n, n))
    for _ in range(passes):
        p = np.pad(rho, 1, mode="edge")
        rho = sum(p[1 + a:1 + a + n, 1 + b:1 + b + n] for a in (-1, 0, 1) for b in (-1, 0, 1)) / 9.0
    return rho


def cavity_multiblock(nb=2, n=64, m=32, vlim=5.0, flux_method="WENO5", Kn=0.01, lid=0.15,
                      seed=0, CFL=0.3):
    """The cavity split into nb x nb blocks of n x n cells (block id = bi*nb + bj,
    bi along x), connected across every internal face."""
    case = base_case(flux_method, Kn, m, vlim, CFL)
    N = nb * n
    rho = smoothed_density(N, seed)
    for bi in range(nb):
        for bj in range(nb):
            x, y = uniform_grid(n, n, bi / nb, (bi + 1) / nb, bj / nb, (bj + 1) / nb)
            bid = lambda a, b: a * nb + b
            bc = [None] * 4
            bc[D.NORTH] = adjacent(bid(bi, bj + 1), D.SOUTH) if bj + 1 < nb else diffuse(1.0, U=lid)
            bc[D.SOUTH] = adjacent(bid(bi, bj - 1), D.NORTH) if bj > 0 else diffuse(1.0)
            bc[D.EAST] = adjacent(bid(bi + 1, bj), D.WEST) if bi + 1 < nb else diffuse(1.0)
            bc[D.WEST] = adjacent(bid(bi - 1, bj), D.EAST) if bi > 0 else diffuse(1.0)
            case["blocks"].append(dict(
                ni=n, nj=n, x=x, y=y, bc=bc,
                fill=dict(D=np.ascontiguousarray(rho[bi * n:(bi + 1) * n, bj * n:(bj + 1) * n]),
                          U=0.0, V=0.0, T=1.0, qx=0.0, qy=0.0)))
    return case


def warp_grid(x, y, amp=0.04):
    """Curvilinear vertices on the unit square: each vertex moved by
    amp sin(2 pi x) sin(pi y) along x and amp sin(pi x) sin(2 pi y) along y,
    which vanishes on the square's edges (straight walls) and is the same
    function on every block, so shared block edges stay shared."""
    xs = x + amp * np.sin(2 * np.pi * x) * np.sin(np.pi * y)
    ys = y + amp * np.sin(np.pi * x) * np.sin(2 * np.pi * y)
    return np.ascontiguousarray(xs), np.ascontiguousarray(ys)


def warped_cavity(nb=1, n=16, m=8, vlim=4.0, flux_method="vanLeer", Kn=0.05, lid=0.15, amp=0.04, CFL=0.3):
    """The lid-driven cavity on a curvilinear grid (warp_grid), as nb x nb
    connected blocks of n x n cells."""
    case = cavity_multiblock(nb=nb, n=n, m=m, vlim=vlim, flux_method=flux_method, Kn=Kn, lid=lid, CFL=CFL) \
        if nb > 1 else cavity(n=n, m=m, vlim=vlim, flux_method=flux_method, Kn=Kn, lid=lid, CFL=CFL)
    for b in case["blocks"]:
        b["x"], b["y"] = warp_grid(b["x"], b["y"], amp)
    return case


# ---------------------------------------------------------------------------
# block connections and open faces beyond the opposite-face, aligned pairs of
# the cavity and channel: every one is a flow that makes physical sense, so
# that several steps of it are a parity case, not only a copy test
# ---------------------------------------------------------------------------

def _fill(ni, nj, rho=1.0):
    return dict(D=rho if np.ndim(rho) else float(rho), U=0.0, V=0.0, T=1.0, qx=0.0, qy=0.0)


def rotated_pair(n=8, m=8, vlim=4.0, flux_method="vanLeer", Kn=0.05, lid=0.15, CFL=0.3):
    """The unit-square cavity as two blocks whose grids are turned 90 degrees
    against each other, joined NORTH to EAST (getSwapIndex's rotation
    branches, clGhostRoutines.c:47-138).

    A covers [0,1] x [0,1/2] (i along +x, j along +y, n x n/2 cells).  B covers
    [0,1] x [1/2,1] with i along -y and j along +x (n/2 x n cells), so B's EAST
    face lies on y = 1/2 against A's NORTH face, B's WEST face is the lid
    (y = 1), its NORTH face the right wall and its SOUTH face the left wall."""
    h = n // 2
    case = base_case(flux_method, Kn, m, vlim, CFL)
    xa, ya = uniform_grid(n, h, 0.0, 1.0, 0.0, 0.5)
    i = np.arange(h + 1, dtype=np.float64)[:, None]
    j = np.arange(n + 1, dtype=np.float64)[None, :]
    xb = np.ascontiguousarray(j / n + 0.0 * i)
    yb = np.ascontiguousarray(1.0 - 0.5 * (i / h) + 0.0 * j)
    bc_a = [None] * 4
    bc_a[D.NORTH] = adjacent(1, D.EAST)
    bc_a[D.EAST], bc_a[D.SOUTH], bc_a[D.WEST] = diffuse(1.0), diffuse(1.0), diffuse(1.0)
    bc_b = [None] * 4
    bc_b[D.EAST] = adjacent(0, D.NORTH)
    bc_b[D.WEST] = diffuse(1.0, U=lid)
    bc_b[D.NORTH], bc_b[D.SOUTH] = diffuse(1.0), diffuse(1.0)
    rho = smoothed_density(n, seed=4)
    case["blocks"].append(dict(ni=n, nj=h, x=xa, y=ya, bc=bc_a,
                               fill=_fill(n, h, np.ascontiguousarray(rho[:, :h]))))
    # B's cell (i, j) sits at x index j, y index n - 1 - i of the square
    case["blocks"].append(dict(ni=h, nj=n, x=xb, y=yb, bc=bc_b,
                               fill=_fill(h, n, np.ascontiguousarray(rho[:, h:][:, ::-1].T))))
    return case


def flipped_pair(n=8, m=8, vlim=4.0, flux_method="vanLeer", Kn=0.05, lid=0.15, CFL=0.3):
    """The unit-square cavity as two blocks joined NORTH to NORTH, the upper
    block's grid turned 180 degrees: the two faces' corner vertices lie
    apart, so with orientation 1 edgeExchange reverses the along-face index
    (clGhostRoutines.c:506-513) before getSwapIndex.

    A covers [0,1] x [0,1/2] (n x n/2 cells); B covers [0,1] x [1/2,1] with i
    along -x and j along -y, so B's NORTH face lies on y = 1/2, its SOUTH face
    is the lid, its EAST face the left wall and its WEST face the right wall.
    Both sides copy vertices without the affine map (NO_TRANSFORM): the map
    would send B's corner 1 onto A's corner 1, which the turned grid does not
    share."""
    h = n // 2
    case = base_case(flux_method, Kn, m, vlim, CFL)
    xa, ya = uniform_grid(n, h, 0.0, 1.0, 0.0, 0.5)
    i = np.arange(n + 1, dtype=np.float64)[:, None]
    j = np.arange(h + 1, dtype=np.float64)[None, :]
    xb = np.ascontiguousarray(1.0 - i / n + 0.0 * j)
    yb = np.ascontiguousarray(1.0 - 0.5 * (j / h) + 0.0 * i)
    link = lambda other: dict(adjacent(other, D.NORTH, orientation=1), transform=D.NO_TRANSFORM)
    bc_a = [None] * 4
    bc_a[D.NORTH] = link(1)
    bc_a[D.EAST], bc_a[D.SOUTH], bc_a[D.WEST] = diffuse(1.0), diffuse(1.0), diffuse(1.0)
    bc_b = [None] * 4
    bc_b[D.NORTH] = link(0)
    bc_b[D.SOUTH] = diffuse(1.0, U=lid)
    bc_b[D.EAST], bc_b[D.WEST] = diffuse(1.0), diffuse(1.0)
    rho = smoothed_density(n, seed=5)
    case["blocks"].append(dict(ni=n, nj=h, x=xa, y=ya, bc=bc_a,
                               fill=_fill(n, h, np.ascontiguousarray(rho[:, :h]))))
    # B's cell (i, j) sits at x index n - 1 - i, y index n - 1 - j
    case["blocks"].append(dict(ni=n, nj=h, x=xb, y=yb, bc=bc_b,
                               fill=_fill(n, h, np.ascontiguousarray(rho[::-1, ::-1][:, :h]))))
    return case


def mirror_cavity(n=8, m=8, vlim=4.0, flux_method="vanLeer", Kn=0.05, lid=0.15, CFL=0.3):
    """A single-block cavity whose faces other than the lid are connected to
    themselves through the velocity permutations of edgeExchange
    (clGhostRoutines.c:517-535): SOUTH to SOUTH with FLIP_NS (a symmetry
    plane, the same ghosts as REFLECT), WEST to WEST with FLIP_EW and EAST to
    EAST with FLIP_D (a bounce-back wall).  Their ghost vertices are the
    interior ones mirrored about the face (the MIRROR map of xyExchange)."""
    case = base_case(flux_method, Kn, m, vlim, CFL)
    x, y = uniform_grid(n, n)
    bc = [None] * 4
    bc[D.NORTH] = diffuse(1.0, U=lid)
    # the ghost vertices are the interior ones mirrored about the face
    # (xyExchange with the MIRROR map, clGhostRoutines.c:273-275)
    self_link = lambda face, flip: dict(adjacent(0, face, flip=flip), transform=D.MIRROR)
    bc[D.SOUTH] = self_link(D.SOUTH, D.FLIP_NS)
    bc[D.WEST] = self_link(D.WEST, D.FLIP_EW)
    bc[D.EAST] = self_link(D.EAST, D.FLIP_D)
    case["blocks"].append(dict(ni=n, nj=n, x=x, y=y, bc=bc,
                               fill=_fill(n, n, smoothed_density(n, seed=6))))
    return case


def periodic_couette(n=8, m=8, vlim=4.0, flux_method="WENO5", Kn=0.05, lid=0.15, CFL=0.3):
    """Plane Couette flow, periodic in x, as two blocks of n/2 x n cells side
    by side: A.EAST joins B.WEST (ADJACENT), B.EAST joins A.WEST as a
    PERIODIC face (code 5) with orientation 0; the lid (NORTH) moves, the
    floor (SOUTH) is at rest.  The density starts perturbed so that the
    solution varies along x too."""
    h = n // 2
    case = base_case(flux_method, Kn, m, vlim, CFL)
    rho = smoothed_density(n, seed=7)
    for b in range(2):
        x, y = uniform_grid(h, n, 0.5 * b, 0.5 * (b + 1), 0.0, 1.0)
        bc = [None] * 4
        bc[D.NORTH] = diffuse(1.0, U=lid)
        bc[D.SOUTH] = diffuse(1.0)
        if b == 0:
            bc[D.EAST] = adjacent(1, D.WEST)
            bc[D.WEST] = periodic(1, D.EAST)
        else:
            bc[D.WEST] = adjacent(0, D.EAST)
            bc[D.EAST] = periodic(0, D.WEST)
        case["blocks"].append(dict(ni=h, nj=n, x=x, y=y, bc=bc,
                                   fill=_fill(h, n, np.ascontiguousarray(rho[b * h:(b + 1) * h, :]))))
    return case


def open_channel(nblocks=2, n=8, m=8, vlim=5.0, flux_method="WENO5", Kn=0.05, rho_in=1.2, u_in=0.05,
                 P_out=1.0, D_out=1.0, length=2.0, height=1.0, CFL=0.3, nj=None):
    """A channel between diffuse walls, fed through a CONSTANT inlet
    (fEQ(rho_in, u_in, 0, T=1) ghosts, edgeConstant, clGhostRoutines.c:603-658)
    and drained through an OUTFLOW face (edgeOutflow, 755-839, with P_out and
    D_out set)."""
    nj = n if nj is None else nj
    case = base_case(flux_method, Kn, m, vlim, CFL)
    for b in range(nblocks):
        x, y = uniform_grid(n, nj, length * b / nblocks, length * (b + 1) / nblocks, 0.0, height)
        bc = [None] * 4
        bc[D.NORTH], bc[D.SOUTH] = diffuse(1.0), diffuse(1.0)
        bc[D.WEST] = adjacent(b - 1, D.EAST) if b > 0 else constant(rho_in, 1.0, U=u_in)
        bc[D.EAST] = adjacent(b + 1, D.WEST) if b + 1 < nblocks else outflow(P_out, D_out)
        xc = 0.5 * (x[1:, :-1] + x[:-1, :-1])
        rho = rho_in + (1.0 - rho_in) * xc / length
        case["blocks"].append(dict(ni=n, nj=nj, x=x, y=y, bc=bc, fill=_fill(n, nj, np.ascontiguousarray(rho))))
    return case


def channel(nblocks=4, n=64, m=32, vlim=5.0, flux_method="WENO5", Kn=0.05, rho_in=1.2,
            rho_out=1.0, length=4.0, height=1.0, gamma_f=0.5, k_des=0.01, CFL=0.3, nj=None,
            adsorb=0.5, reflect_type="D", alpha_n=1.0, alpha_t=1.0):
    """Pressure-driven channel: nblocks blocks of n x nj cells along x,
    equilibrium inlet/outlet ghosts, diffuse upper wall, adsorbing lower wall."""
    nj = n if nj is None else nj
    case = base_case(flux_method, Kn, m, vlim, CFL)
    for b in range(nblocks):
        x, y = uniform_grid(n, nj, length * b / nblocks, length * (b + 1) / nblocks, 0.0, height)
        bc = [None] * 4
        bc[D.NORTH] = diffuse(1.0)
        bc[D.SOUTH] = adsorbing(1.0, gamma_f=gamma_f, k_des=k_des, adsorb=adsorb, reflect_type=reflect_type,
                                alpha_n=alpha_n, alpha_t=alpha_t)
        bc[D.WEST] = adjacent(b - 1, D.EAST) if b > 0 else inflow(rho_in, 1.0)
        bc[D.EAST] = adjacent(b + 1, D.WEST) if b + 1 < nblocks else inflow(rho_out, 1.0)
        # linear initial density between inlet and outlet
        xc = 0.5 * (x[1:, :-1] + x[:-1, :-1])
        rho = rho_in + (rho_out - rho_in) * xc / length
        case["blocks"].append(dict(ni=n, nj=nj, x=x, y=y, bc=bc,
                                   fill=dict(D=np.ascontiguousarray(rho), U=0.0, V=0.0, T=1.0,
                                             qx=0.0, qy=0.0)))
    return case


CAVITY_SIZES = (24, 32, 48, 64, 96, 128)
CAVITY_VGRIDS = (16, 24, 32, 48)


def batched_cavities(count=64, seed=1):
    """Independent cavity solves with drawn sizes and parameters: n from
    {24..128}, velocity grid m from {16..48} on [-5,5]^2, Kn log-uniform on
    [0.005, 1], lid U(0.05, 0.3), wall T U(0.8, 1.2), vanLeer or WENO5."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice(CAVITY_SIZES))
        m = int(rng.choice(CAVITY_VGRIDS))
        Kn = float(10 ** rng.uniform(np.log10(0.005), 0.0))
        lid = float(rng.uniform(0.05, 0.3))
        Tw = float(rng.uniform(0.8, 1.2))
        scheme = "WENO5" if rng.random() < 0.5 else "vanLeer"
        out.append(cavity(n=n, m=m, vlim=5.0, flux_method=scheme, Kn=Kn, lid=lid, T_wall=Tw,
                          CFL=WORKLOAD_CFL))
    return out


def workload_size(case) -> int:
    """Interior cell-velocity points per step: sum over blocks of ni*nj*Nv."""
    q = case["quad"]
    nv = (int(q["u_num"] / 4) * 4 + 1) * (int(q["v_num"] / 4) * 4 + 1)
    return sum(b["ni"] * b["nj"] for b in case["blocks"]) * nv
