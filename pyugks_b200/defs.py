"""Codes shared by the block driver and the kernels.

Face numbering, boundary-condition codes and velocity permutations keep the
reference's values (``geom/geom_defs.py``, ``geom/geom_bc_defs.py:27-51``,
``source/clError.c:4-20``) so that job descriptions written for pyUGKS map
one to one.
"""

# block faces (geom/geom_defs.py)
NORTH, EAST, SOUTH, WEST = 0, 1, 2, 3
FACE_NAMES = ("north", "east", "south", "west")

# face directions of the flux arrays (clUGKS.c: SOUTH = 0, WEST = 1)
S_DIR, W_DIR = 0, 1

# boundary conditions (geom/geom_bc_defs.py:27-37)
ADJACENT = 0
EXTRAPOLATE_OUT = 1
CONSTANT = 2
REFLECT = 3
DIFFUSE = 4
PERIODIC = 5
INFLOW = 6
OUTFLOW = 7
ADSORBING = 8
BOUNCE_BACK = 9

BC_NAMES = {ADJACENT: "ADJACENT", EXTRAPOLATE_OUT: "EXTRAPOLATE_OUT", CONSTANT: "CONSTANT",
            REFLECT: "REFLECT", DIFFUSE: "DIFFUSE", PERIODIC: "PERIODIC", INFLOW: "INFLOW",
            OUTFLOW: "OUTFLOW", ADSORBING: "ADSORBING", BOUNCE_BACK: "BOUNCE_BACK"}

# velocity permutation applied across a block connection (geom_bc_defs.py:40-43)
NO_FLIP, FLIP_NS, FLIP_D, FLIP_EW = 0, 1, 2, 3

# block-coordinate transform across a connection (geom_bc_defs.py:46-48)
NO_TRANSFORM, TRANSFORM, MIRROR = 0, 1, 2

# status codes written by the kernels (clError.c:4-13, as integers)
ERR_OK = 0
ERR_NAN = 1
ERR_ADSORB_TOO_MUCH = 2
ERR_DESORB_TOO_MUCH = 3
ERR_CLAMPING_ADSORB_ISOTHERM = 4
ERR_TIMEOUT = 5
ERR_BAD_CONNECTION = 6

FLUX_METHODS = {"vanLeer": 0, "WENO5": 1, "minmod": 3}
