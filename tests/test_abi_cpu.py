"""The C ABI library loads without a GPU, exports every entry point that
include/ugks_b200.h declares, and agrees with the Python struct layouts."""
import ctypes
import os
import re

from pyugks_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(ugks_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 40
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match():
    L = _lib.lib()  # raises on a layout mismatch
    assert L.ugks_version().startswith(b"ugks_b200")


def test_kernel_table_covers_reference_kernels():
    # every reference kernel of the time-step path has a drop-in entry point
    path_kernels = {"iFace", "getFaceCons", "getAL", "getAR", "getPLR", "initMacroFlux", "calcFaceQ",
                    "macroFlux", "distFlux", "accommodatingWallDist", "wallFlux",
                    "wallMassEnergyFluxes", "updateMacro", "UGKS_update", "getResidual",
                    "edgeMassFlow", "calcQ", "calcMacro", "initFunctions", "clFindDT", "paraBC",
                    "edgeExchange", "edgeExtrapolate", "edgeConstant", "edgeInflow", "edgeOutflow",
                    "edgeMirror", "edgeBounceBack", "edgeConstGrad", "adsorbingWall_P1",
                    "adsorbingWallD_P2"}
    assert path_kernels <= set(_lib.KERNEL_SIGNATURES)
    assert {"ugks_" + k for k in path_kernels} <= declared_symbols()
