"""Kernel programs of the oracle: ctypes bindings with the reference call shape.

TEST INFRASTRUCTURE ONLY.  Two interchangeable programs expose the reference
kernels as ``prog.<kernel>(global_size, *args)`` with the arguments in the
order of the reference ``__kernel`` signatures (``source/*.c``):

* ``RefProgram``  -- the reference's own kernels compiled for the CPU by
  ``oracle/ref_build.py`` (one library per block header, in ``oracle/_ref``);
* ``PortProgram`` -- the plain-C restatement ``oracle/ugks_port.c`` with the
  header constants passed at run time.

numpy arrays pass as pointers, Python ints as ``int``, floats as ``double``.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ugks_setup as us  # noqa: E402

# argument kinds per kernel (p: pointer, i: int, d: double), reference order
SIGNATURES = {
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
_CT = {"p": C.c_void_p, "i": C.c_int, "d": C.c_double}


def _arg(kind, a):
    if kind == "p":
        if isinstance(a, np.ndarray):
            assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
            return a.ctypes.data_as(C.c_void_p)
        return a
    return a


class _Program:
    def __init__(self, lib, prefix, bind=None):
        self._lib = lib
        self._prefix = prefix
        self._bind = bind or ()
        self._fns = {}

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        sig = SIGNATURES[name]
        fn = self._fns.get(name)
        if fn is None:
            fn = getattr(self._lib, self._prefix + name)
            fn.restype = None
            fn.argtypes = [C.c_void_p] * len(self._bind) + [C.c_size_t, C.c_size_t] + [_CT[k] for k in sig]
            self._fns[name] = fn

        def call(gsize, *args):
            assert len(args) == len(sig), (name, len(args), len(sig))
            g0 = int(gsize[0])
            g1 = int(gsize[1]) if len(gsize) > 1 else 1
            fn(*self._bind, g0, g1, *[_arg(k, a) for k, a in zip(sig, args)])

        return call


# ---------------------------------------------------------------------------
# the compiled reference
# ---------------------------------------------------------------------------

class RefProgram(_Program):
    """The reference kernels of one block (``oracle/_ref``)."""

    def __init__(self, const: us.Constants, block: dict, block_id: int, threads: int | None = None):
        import ref_build as rb
        so = None
        if os.path.isdir(os.path.join(rb.reference_root(), "source")):
            so = rb.build_and_index(const, block, block_id)
        else:
            so = rb.find_built(const, block, block_id)
        if so is None:
            raise FileNotFoundError("compiled reference for this block is not available")
        lib = C.CDLL(so)
        super().__init__(lib, "ref_")
        self.so = so
        if threads is not None:
            lib.ref_set_threads(int(threads))


def reference_available(const, block, block_id) -> bool:
    import ref_build as rb
    if os.path.isdir(os.path.join(rb.reference_root(), "source")):
        return True
    return rb.find_built(const, block, block_id) is not None


# ---------------------------------------------------------------------------
# the C restatement
# ---------------------------------------------------------------------------

PORT_SO = os.path.join(HERE, "_build", "libugks_port.so")


def build_port(force: bool = False) -> str:
    """Compile ``oracle/ugks_port.c`` into ``oracle/_build`` (gcc)."""
    src = os.path.join(HERE, "ugks_port.c")
    hdr = os.path.join(HERE, "ugks_port.h")
    if (not force and os.path.exists(PORT_SO) and
            os.path.getmtime(PORT_SO) >= max(os.path.getmtime(src), os.path.getmtime(hdr))):
        return PORT_SO
    os.makedirs(os.path.dirname(PORT_SO), exist_ok=True)
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off",
           "-fopenmp", src, "-o", PORT_SO + ".tmp", "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(PORT_SO + ".tmp", PORT_SO)
    return PORT_SO


class _PortParams(C.Structure):
    _fields_ = [
        ("ni", C.c_int), ("nj", C.c_int), ("Ni", C.c_int), ("Nj", C.c_int), ("ghost", C.c_int),
        ("Nv", C.c_int), ("flux_method", C.c_int), ("relax_type", C.c_int),
        ("PI", C.c_double), ("Pr", C.c_double), ("umax", C.c_double), ("vmax", C.c_double),
        ("Kn_eff", C.c_double), ("gam", C.c_double), ("B", C.c_double), ("K", C.c_double),
        ("omega", C.c_double),
        ("quad", C.c_void_p), ("weight", C.c_void_p),
        ("mirror_NS", C.c_void_p), ("mirror_EW", C.c_void_p), ("mirror_D", C.c_void_p),
        ("wall_D", C.c_double * 4), ("wall_U", C.c_double * 4), ("wall_V", C.c_double * 4),
        ("wall_T", C.c_double * 4), ("wall_P", C.c_double * 4),
        ("beta_n", C.c_double * 4), ("beta_t", C.c_double * 4), ("gamma_f", C.c_double * 4),
        ("alpha_p", C.c_double * 4), ("dynamic", C.c_int * 4), ("constant_adsorb", C.c_int * 4),
        ("adsorb", C.c_double * 4), ("k_des", C.c_double * 4),
        ("alpha_n", C.c_double * 4), ("alpha_t", C.c_double * 4),
        ("iso", C.c_void_p * 4), ("tri", C.c_void_p * 4), ("nbr", C.c_void_p * 4), ("n_tri", C.c_int * 4),
    ]


class PortProgram(_Program):
    """The C restatement bound to one block's header constants."""

    _lib = None

    def __init__(self, const: us.Constants, block: dict, block_id: int):
        if PortProgram._lib is None:
            PortProgram._lib = C.CDLL(build_port())
        G = const.ghost
        p = _PortParams()
        p.ni, p.nj = block["ni"], block["nj"]
        p.Ni, p.Nj = block["ni"] + 2 * G, block["nj"] + 2 * G
        p.ghost, p.Nv = G, const.Nv
        p.flux_method, p.relax_type = const.flux_code, const.relax_type
        p.PI, p.Pr, p.umax, p.vmax = const.PI, const.Pr, const.umax, const.vmax
        p.Kn_eff, p.gam, p.B, p.K, p.omega = const.Kn_eff, const.gam, const.B, const.K, const.omega
        # keep the tables alive with the program
        self._tables = [np.ascontiguousarray(const.quad, dtype=np.float64),
                        np.ascontiguousarray(const.weight, dtype=np.float64),
                        np.ascontiguousarray(const.mirror_NS, dtype=np.int64),
                        np.ascontiguousarray(const.mirror_EW, dtype=np.int64),
                        np.ascontiguousarray(const.mirror_D, dtype=np.int64)]
        p.quad, p.weight, p.mirror_NS, p.mirror_EW, p.mirror_D = [t.ctypes.data for t in self._tables]
        for f, bc in enumerate(block["bc"]):
            D, U, V, T, P = us.wall_values(bc)
            p.wall_D[f], p.wall_U[f], p.wall_V[f], p.wall_T[f], p.wall_P[f] = D, U, V, T, P
            if bc["type"] == us.ADSORBING:
                p.beta_n[f] = us.e15(bc.get("beta_n", 0.0))
                p.beta_t[f] = us.e15(bc.get("beta_t", 0.0))
                p.gamma_f[f] = us.e15(bc["gamma_f"])
                p.alpha_p[f] = us.e15(bc["alpha_p"])
                p.dynamic[f] = int(bc.get("dynamic", 1))
                p.constant_adsorb[f] = 1 if np.ndim(bc["adsorb"]) == 0 else 0
                p.adsorb[f] = float("%g" % bc["adsorb"]) if np.ndim(bc["adsorb"]) == 0 else 0.0
                p.k_des[f] = float(bc.get("k_des", 0.0))
                p.alpha_n[f] = us.e15(bc.get("alpha_n", 0.0))
                p.alpha_t[f] = us.e15(bc.get("alpha_t", 0.0))
                if np.ndim(bc["adsorb"]) != 0:
                    pts, tri, nbr = us.isotherm_tables(bc["adsorb"])
                    self._tables += [pts, tri, nbr]
                    p.iso[f], p.tri[f], p.nbr[f] = pts.ctypes.data, tri.ctypes.data, nbr.ctypes.data
                    p.n_tri[f] = tri.shape[0]
            else:
                p.beta_n[f] = p.beta_t[f] = p.gamma_f[f] = p.alpha_p[f] = -1.0
                p.alpha_n[f] = p.alpha_t[f] = -1.0
                p.dynamic[f] = -1
        self._params = p
        super().__init__(PortProgram._lib, "port_", bind=(C.cast(C.pointer(p), C.c_void_p),))
