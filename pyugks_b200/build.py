"""Build recipe for libugks_b200.so (sm_100a), compiled in-tree.

``python -m pyugks_b200.build`` (or ``build()``) runs nvcc on every
``csrc/*.cu`` into ``pyugks_b200/libugks_b200.so``; the library is rebuilt
only when a source or header is newer than it.

``python -m pyugks_b200.build --checked`` (``build(checked=True)``) builds
``libugks_b200_checked.so`` with ``-DUGKS_CHECKED=1``: every work item of the
fused kernels is checked against its block, and a failed check sets the
solve's status to 9 and skips the item.  Point ``UGKS_LIB_PATH`` at it to run
with the checks.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libugks_b200.so")
LIB_CHECKED = os.path.join(HERE, "libugks_b200_checked.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-lineinfo",
              "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


# the geometry set-up keeps every product and sum separately rounded
FILE_FLAGS = {"ugks_geometry.cu": ["-fmad=false"]}


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def deps():
    return (sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def needs_build(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(p) > t for p in deps())


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    lib = LIB_CHECKED if checked else LIB
    if not force and not needs_build(lib):
        return lib
    nvcc = os.environ.get("NVCC", "nvcc")
    objs = []
    bdir = os.path.join(HERE, "_build_checked" if checked else "_build")
    os.makedirs(bdir, exist_ok=True)
    extra = ["-DUGKS_CHECKED=1"] if checked else []
    for src in sources():
        obj = os.path.join(bdir, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc, *NVCC_FLAGS, *extra, *FILE_FLAGS.get(os.path.basename(src), []), "-I",
               os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = lib + ".tmp"
    subprocess.run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static",
                    *objs, "-o", tmp], check=True)
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv))
