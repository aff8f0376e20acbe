"""ctypes binding of libugks_b200.so (include/ugks_b200.h).

The library is the only compute path of this package: there is no CPU
fallback.  ``lib()`` raises if the shared object is missing or was built
against a different struct layout.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# UGKS_LIB_PATH selects another build of the same library (tuning builds)
LIB_PATH = os.environ.get("UGKS_LIB_PATH", os.path.join(HERE, "libugks_b200.so"))

i32, f64, vp = C.c_int32, C.c_double, C.c_void_p


class BlockDesc(C.Structure):
    """ugks_block_desc"""
    _fields_ = [
        ("ni", i32), ("nj", i32), ("Ni", i32), ("Nj", i32), ("ghost", i32), ("Nv", i32),
        ("flux_method", i32), ("relax_type", i32),
        ("PI", f64), ("Pr", f64), ("umax", f64), ("vmax", f64), ("Kn_eff", f64), ("gam", f64),
        ("K", f64), ("omega", f64),
        ("quad", vp), ("weight", vp), ("mirror_NS", vp), ("mirror_EW", vp), ("mirror_D", vp),
        ("wall_D", f64 * 4), ("wall_U", f64 * 4), ("wall_V", f64 * 4), ("wall_T", f64 * 4),
        ("wall_P", f64 * 4),
        ("beta_n", f64 * 4), ("beta_t", f64 * 4), ("gamma_f", f64 * 4), ("alpha_p", f64 * 4),
        ("adsorb", f64 * 4), ("k_des", f64 * 4),
        ("dynamic", i32 * 4), ("constant_adsorb", i32 * 4),
        ("u_num", i32), ("v_num", i32),
        ("alpha_n", f64 * 4), ("alpha_t", f64 * 4), ("reflect", i32 * 4),
        ("iso", vp * 4), ("tri", vp * 4), ("nbr", vp * 4), ("n_tri", i32 * 4),
        ("B", f64),
    ]


class FusedBlock(C.Structure):
    """ugks_fused_block"""
    _fields_ = [
        ("d", BlockDesc), ("solve", i32),
        ("bc_type", i32 * 4), ("bc_block", i32 * 4), ("bc_face", i32 * 4), ("bc_ori", i32 * 4),
        ("bc_flip", i32 * 4),
        ("face_begin", i32), ("cell_begin", i32), ("ghost_begin", i32), ("wall_begin", i32),
        ("f", vp), ("flux_S", vp), ("flux_W", vp), ("flux_macro_S", vp), ("flux_macro_W", vp),
        ("macro", vp), ("Q", vp), ("prim_old", vp),
        ("area", vp), ("centre", vp), ("mid_side", vp), ("normal", vp), ("side_length", vp),
        ("xy", vp), ("wall_prop", vp), ("wall_cover", vp), ("wall_fluxes", vp), ("wall_dist", vp),
        ("cell_mom", vp), ("Q_next", vp), ("face_geo", vp), ("ref", vp),
        ("aux_S", vp), ("aux_W", vp), ("face_rec", vp),
    ]


class SolveState(C.Structure):
    """ugks_solve_state"""
    _fields_ = [
        ("dt", f64), ("time", f64), ("CFL", f64), ("delta_dt", f64), ("max_dt", f64),
        ("max_freq", C.c_uint64),
        ("retry", i32), ("status", i32), ("steps", i32), ("retries", i32), ("active", i32),
        ("nblocks", i32), ("first_block", i32), ("stopped", i32),
        ("residual", f64 * 4), ("stop_residual", f64), ("stop_steps", i32), ("stop_after", i32),
    ]


# ugks_solve_state.stopped (UGKS_STOP_*)
STOP_CONVERGED, STOP_STEPS, STOP_ERROR = 1, 2, 3
STOP_REASONS = {STOP_CONVERGED: "converged", STOP_STEPS: "max_steps", STOP_ERROR: "error"}


class FusedSizes(C.Structure):
    """ugks_fused_sizes"""
    _fields_ = [("n_faces", i32), ("n_cells", i32), ("n_ghost", i32), ("max_nv", i32),
                ("face_begin", i32 * 4), ("face_count", i32 * 4), ("max_axes", i32),
                ("n_segments", i32), ("seg_begin", i32 * 16), ("seg_count", i32 * 16),
                ("seg_method", i32 * 16), ("seg_max_nv", i32 * 16), ("seg_max_axes", i32 * 16),
                ("seg_variant", i32 * 16), ("cell_variant", i32), ("n_wall", i32)]


FACE_VARIANTS = 5   # UGKS_FACE_VARIANTS: 0 automatic, 1..4 forced shapes


# argument kinds of the drop-in kernels in reference order (p pointer, i int,
# d double); the C functions take (desc*, g0, g1, <args>, stream)
KERNEL_SIGNATURES = {
    "paraBC": "ppd", "clFindDT": "ppppd", "initFunctions": "ppp", "calcMacro": "pp",
    "calcQ": "ppp", "iFace": "ppppppi", "getFaceCons": "ppipii", "getAL": "ppipii",
    "getAR": "ppipii", "getPLR": "ppipppii", "initMacroFlux": "pidpppppii",
    "calcFaceQ": "ppppiii", "macroFlux": "pppppidppii", "distFlux": "ppppidppppppii",
    "accommodatingWallDist": "pippd", "wallFlux": "ppippd", "wallMassEnergyFluxes": "pppippd",
    "updateMacro": "ppppp", "UGKS_update": "pppppppdp", "getResidual": "pp",
    "edgeMassFlow": "ppppi", "edgeExchange": "ppippiiiii", "edgeExtrapolate": "pi",
    "edgeConstant": "pip", "edgeInflow": "pipppp", "edgeOutflow": "pipppp",
    "edgeMirror": "pi", "edgeBounceBack": "pi", "edgeConstGrad": "pi",
    "adsorbingWall_P1": "pipppppdp", "adsorbingWallD_P2": "pipppppd",
    "adsorbingWallS_P2": "pipppppd", "adsorbingWallCL_P2": "pipppppd",
    "xyExchange": "pipiiiiiiii", "xyExtrapolate": "pi", "cellGeom": "pppppp", "getInternal": "ppp",
}
_CT = {"p": vp, "i": C.c_int, "d": f64}

# layout of the mixed path's reference Maxwellian (UGKS_REF_*, include/ugks_b200.h)
REF_LAMBDA, REF_P0, REF_KB0, REF_MOM, REF_TAB = 0, 1, 2, 4, 32
FACE_REC = 48       # UGKS_FACE_REC

# ugks_getDT_noalloc limits and error codes (include/ugks_b200.h)
NOALLOC_MAX_CELLS = 1 << 20
ERR_TOO_LARGE = -10001
ERR_BAD_SIZE = -10002

_LIB = None


class NativeLibraryMissing(RuntimeError):
    pass


def lib():
    """The loaded library, with prototypes set.  Raises if it is absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise NativeLibraryMissing(
            "libugks_b200.so is not built (run `python -m pyugks_b200.build`); "
            "there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    for name, sig in KERNEL_SIGNATURES.items():
        fn = getattr(L, "ugks_" + name)
        fn.restype = C.c_int
        fn.argtypes = [C.POINTER(BlockDesc), C.c_size_t, C.c_size_t] + [_CT[k] for k in sig] + [vp]
    L.ugks_array_max.restype = C.c_int
    L.ugks_array_max.argtypes = [vp, C.c_size_t, vp, vp]
    L.ugks_fused_layout.restype = C.c_int
    L.ugks_fused_layout.argtypes = [C.POINTER(FusedBlock), C.c_int, C.POINTER(FusedSizes)]
    for nm in ("ugks_init_fp64", "ugks_init_mixed", "ugks_restart_fp64", "ugks_restart_mixed",
               "ugks_step_fp64", "ugks_step_mixed"):
        fn = getattr(L, nm)
        fn.restype = C.c_int
        fn.argtypes = [vp, C.c_int, C.POINTER(FusedSizes), vp, C.c_int, vp]
    L.ugks_step_profiled.restype = C.c_int
    L.ugks_step_profiled.argtypes = [C.c_int, vp, C.c_int, C.POINTER(FusedSizes), vp, C.c_int, vp, vp]
    L.ugks_step_launches.restype = C.c_int
    L.ugks_step_launches.argtypes = [C.POINTER(FusedSizes), C.c_int]
    L.ugks_residual.restype = C.c_int
    L.ugks_residual.argtypes = [vp, C.c_int, vp, C.c_int, vp]
    L.ugks_stop_check.restype = C.c_int
    L.ugks_stop_check.argtypes = [vp, C.c_int, vp]
    L.ugks_serve_steps.restype = C.c_int
    L.ugks_serve_steps.argtypes = [C.c_int, vp, C.c_int, C.POINTER(FusedSizes), vp, C.c_int, C.c_int, vp]
    L.ugks_prepare.restype = C.c_int
    L.ugks_prepare.argtypes = [C.c_int]
    L.ugks_check_copy_wait.restype = C.c_int
    L.ugks_check_copy_wait.argtypes = [vp, C.c_uint, vp, vp]
    L.ugks_getDT_noalloc.restype = C.c_int
    L.ugks_getDT_noalloc.argtypes = [C.POINTER(BlockDesc), vp, vp, vp, f64, vp, vp]
    L.ugks_version.restype = C.c_char_p
    L.ugks_abi_sizes.restype = C.c_int
    L.ugks_abi_sizes.argtypes = [C.POINTER(C.c_int64), C.c_int]
    sizes = (C.c_int64 * 7)()
    L.ugks_abi_sizes(sizes, 7)
    want = [C.sizeof(BlockDesc), C.sizeof(FusedBlock), C.sizeof(SolveState),
            FusedBlock.f.offset, SolveState.residual.offset, BlockDesc.wall_D.offset,
            C.sizeof(FusedSizes)]
    if list(sizes) != want:
        raise NativeLibraryMissing("struct layout mismatch with libugks_b200.so: %s vs %s"
                                   % (list(sizes), want))
    _LIB = L
    return L


def check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError("%s failed: CUDA error %d" % (what, -rc))
