"""Recipe: compile the reference's own OpenCL C kernels for the CPU.

TEST INFRASTRUCTURE ONLY (oracle).  Reads the pyUGKS kernel sources where they
lie (``<reference>/source/*.c``), never copies them into this repository, and
writes everything it generates into ``oracle/_ref/`` (git-ignored): one shared
library per distinct block header, plus a JSON manifest of the kernel
signatures so that ``oracle/refprog.py`` can call them through ctypes.

Steps, restating the reference's own source assembly:

1. ``SourceLoader`` (``source/source_CL.py:11-58``): read the kernel files and
   hoist every line holding ``#define`` into one "definitions" block.
2. ``genHeader`` (``ugks_CL.py:20-400``): emit the per-block constants, BC
   macros and velocity tables.  The only change is syntax: vector literals are
   written as ``make_doubleN(...)`` calls so that the text is valid C++.
3. Concatenate in the reference's compile order (``ugks_CL.py:423-424``):
   header, definitions, clFunctions, clAdsorb, clKernel, clUGKS,
   clGhostRoutines, after rewriting the six ``(doubleN)(...)`` literal lines of
   the kernel sources to ``make_doubleN(...)``.
4. Append, per ``__kernel``, an ``extern "C"`` launcher that walks the NDRange
   (work-group size 1, ``LOCAL_SIZE 1``) with OpenMP over work-groups.
5. ``g++ -O3 -fopenmp -ffp-contract=off`` with ``oracle/opencl_shim.hpp``.
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
# the pyUGKS checkout: $UGKS_REFERENCE, else a directory named "reference"
# beside this repository's root
DEFAULT_REFERENCE = os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference"))

sys.path.insert(0, HERE)
import ugks_setup as us  # noqa: E402

SOURCE_ORDER = ["clError.c", "clFunctions.c", "clAdsorb.c", "clKernel.c",
                "clGhostRoutines.c", "clUGKS.c"]           # source_CL.py:18-19
COMPILE_ORDER = ["clFunctions.c", "clAdsorb.c", "clKernel.c", "clUGKS.c",
                 "clGhostRoutines.c"]                      # ugks_CL.py:423-424
FACE_NAMES = ["north", "east", "south", "west"]
WALL_NAMES = ["N", "E", "S", "W"]


def reference_root() -> str:
    return os.environ.get("UGKS_REFERENCE", DEFAULT_REFERENCE)


def load_sources(root: str):
    """SourceLoader restated: hoist ``#define`` lines, keep the rest."""
    src = {}
    defines = []
    for name in SOURCE_ORDER:
        with open(os.path.join(root, "source", name)) as fh:
            lines = fh.readlines()
        these = [ln for ln in lines if "#define" in ln]
        for ln in these:
            lines.remove(ln)
        defines += these
        src[name] = "".join(lines)
    src["definitions"] = "".join(defines)
    return src


_VEC_LITERAL = re.compile(r"\((double|int)([2348])\)\s*\(")


def rewrite_literals(text: str) -> str:
    """``(double2)(a, b)`` -> ``make_double2(a, b)`` (C++ would read the
    former as a cast of a comma expression)."""
    return _VEC_LITERAL.sub(lambda m: "make_%s%s(" % (m.group(1), m.group(2)), text)


def gen_header(const: us.Constants, block: dict, block_id: int) -> str:
    """genHeader restated for one block (``ugks_CL.py:20-400``)."""
    G = const.ghost
    ni, nj = block["ni"], block["nj"]
    Ni, Nj = ni + 2 * G, nj + 2 * G
    fm = const.flux_code
    stencil = 5 if fm == 1 else 3
    mid = 2 if fm == 1 else 1
    t = const.text
    s = []
    a = s.append
    a("#define LOCAL_SIZE 1\n")
    a("#define LOCAL_LOOP_LENGTH %d\n" % const.Nv)
    for k, v in [("NI", Ni), ("NJ", Nj), ("ni", ni), ("nj", nj), ("NV", const.Nv),
                 ("NX", Ni + 1), ("NY", Nj + 1), ("IMIN", G), ("IMAX", ni + G - 1),
                 ("JMIN", G), ("JMAX", nj + G - 1), ("GHOST", G)]:
        a("#define %s %d\n" % (k, v))
    a("#define SOUTH 0\n#define WEST 1\n#define GNORTH 0\n#define GEAST 1\n"
      "#define GSOUTH 2\n#define GWEST 3\n")
    a("#define BLOCK %d\n#define FLUX_METHOD %d\n#define STENCIL_LENGTH %d\n"
      "#define MID_STENCIL %d\n\n" % (block_id, fm, stencil, mid))
    a("#define PI %s\n" % t["PI"])
    a("#define Pr %s\n" % t["Pr"])
    a("#define umax %s\n" % t["umax"])
    a("#define vmax %s\n" % t["vmax"])
    a("#define Kn_eff %s\n" % t["Kn_eff"])
    a("#define gam %s\n" % t["gam"])
    a("#define B %s\n" % t["B"])
    a("#define K %s\n" % t["K"])
    a("#define OMEGA %s\n" % t["OMEGA"])
    a("#define RELAX_TYPE %s\n" % t["RELAX_TYPE"])
    a("#define CFL %s\n\n" % t["CFL"])
    bcs = block["bc"]

    def per_face(key, fmt, default="-1"):
        vals = []
        for bc in bcs:
            vals.append(fmt % bc.get(key, 0) if bc["type"] == us.ADSORBING else default)
        return ", ".join(vals)

    a("const double BETA_N[4] = {%s};\n" % per_face("beta_n", "%0.15e"))
    a("const double BETA_T[4] = {%s};\n" % per_face("beta_t", "%0.15e"))
    a("const double GAMMA_F[4] = {%s};\n" % per_face("gamma_f", "%0.15e"))
    a("const double ALPHA_P[4] = {%s};\n" % per_face("alpha_p", "%0.15e"))
    a("const double ALPHA_N[4] = {%s};\n" % per_face("alpha_n", "%0.15e"))
    a("const double ALPHA_T[4] = {%s};\n" % per_face("alpha_t", "%0.15e"))
    a("const int DYNAMIC_VARTHETA[4] = {%s};\n" % ", ".join(
        "%i" % bc.get("dynamic", 1) if bc["type"] == us.ADSORBING else "-1" for bc in bcs))
    n_tri = [0, 0, 0, 0]
    for bci, bc in enumerate(bcs):
        fn = FACE_NAMES[bci]
        if bc["type"] == us.ADSORBING and np.ndim(bc["adsorb"]) != 0:
            pts, tri, nbr = us.isotherm_tables(bc["adsorb"])
            a("#define CONSTANT_ADSORB_%s 0\n" % fn)
            a("#define ADSORB_%s 0.0\n" % fn)
            a("const double4 ISO_%s[%d] = {%s};\n" % (fn, len(pts), ", ".join(
                "make_double4(%0.15e, %0.15e, %0.15e, 0)" % tuple(r[:3]) for r in pts)))
            a("const int4 TRI_%s[%d] = {%s};\n" % (fn, len(tri), ", ".join(
                "make_int4(%d, %d, %d, 0)" % tuple(r[:3]) for r in tri)))
            a("const int4 NBR_%s[%d] = {%s};\n" % (fn, len(nbr), ", ".join(
                "make_int4(%d, %d, %d, 0)" % tuple(r[:3]) for r in nbr)))
            n_tri[bci] = len(tri)
            continue
        if bc["type"] == us.ADSORBING:
            ads = bc["adsorb"]
            if ads > 1.0 or ads <= 0.0:
                raise RuntimeError("Boundary condition equilibrium adsorption out of bounds")
            a("#define CONSTANT_ADSORB_%s 1\n" % fn)
            a("#define ADSORB_%s %g\n" % (fn, ads))
        else:
            a("#define CONSTANT_ADSORB_%s 0\n" % fn)
            a("#define ADSORB_%s 0.0\n" % fn)
        a("const double4 ISO_%s[1] = {make_double4(-1,-1,-1,-1)};\n" % fn)
        a("const int4 TRI_%s[1] = {make_int4(-1,-1,-1,-1)};\n" % fn)
        a("const int4 NBR_%s[1] = {make_int4(-1,-1,-1,-1)};\n" % fn)
    a("const int N_TRI[4] = {%d, %d, %d, %d};\n" % tuple(n_tri))
    has = {"D": False, "CL": False, "S": False, "DA": False}
    for bc in bcs:
        if bc["type"] == us.DIFFUSE:
            has["D"] = True
        elif bc["type"] == us.ADSORBING:
            rt = bc.get("reflect_type", "S")
            has["S" if rt == "S" else ("DA" if rt == "D" else "CL")] = True
    a("#define HAS_DIFFUSE_WALL %d\n" % has["D"])
    a("#define HAS_ADSORBING_CL_WALL %d\n" % has["CL"])
    a("#define HAS_ADSORBING_SPECULAR_WALL %d\n" % has["S"])
    a("#define HAS_ADSORBING_DIFFUSE_WALL %d\n" % has["DA"])
    for i, bc in enumerate(bcs):
        w = us.wall_text(bc)
        for k in "DUVTP":
            a("#define WALL_%s_%s %s\n" % (WALL_NAMES[i], k, w[k]))
    a("const double2 QUAD[%d] = {" % const.Nv)
    a(",\n".join("make_double2(%0.15e, %0.15e)" % (q[0], q[1]) for q in const.quad))
    a("};\n\n")
    a("const double WEIGHT[%d] = {" % const.Nv)
    a(", ".join("%0.15e" % w for w in const.weight))
    a("};\n\n")
    for name, arr in [("mirror_NS", const.mirror_NS), ("mirror_EW", const.mirror_EW),
                      ("mirror_D", const.mirror_D)]:
        a("const size_t %s[%d] = {%s};\n" % (name, const.Nv, ", ".join(str(int(x)) for x in arr)))
    return "".join(s)


_KERNEL_SIG = re.compile(r"__kernel\s+void\s+(\w+)\s*\(([^)]*)\)", re.S)


def kernel_signatures(text: str):
    """[(name, [(ctype, argname), ...])] for every ``__kernel`` in ``text``."""
    out = []
    for m in _KERNEL_SIG.finditer(text):
        params = []
        for p in m.group(2).split(","):
            p = " ".join(p.replace("__global", "").split())
            name = re.findall(r"\w+", p)[-1]
            ctype = p[: p.rfind(name)].strip().replace(" *", "*")
            params.append((ctype, name))
        out.append((m.group(1), params))
    return out


def assemble(const: us.Constants, block: dict, block_id: int, root: str):
    src = load_sources(root)
    body = ""
    split = "\n//++++++++++++++++++++++++++++++++++++++++++++++++++++++\n"
    body += split + src["definitions"]
    for name in COMPILE_ORDER:
        body += split + rewrite_literals(src[name])
    header = gen_header(const, block, block_id)
    # only the kernels that survive the header's #if switches get a launcher
    pre = subprocess.run(["g++", "-E", "-P", "-x", "c++", "-"], input=header + body,
                         capture_output=True, text=True, check=True).stdout
    sigs = kernel_signatures(pre)
    launch = ["\n// ---- NDRange launchers (work-group size 1) ----\n"]
    for name, params in sigs:
        plist = ", ".join("%s %s" % (t, n) for t, n in params)
        args = ", ".join(n for _, n in params)
        launch.append(
            'extern "C" void ref_%s(size_t g0, size_t g1, %s) {\n'
            "  #pragma omp parallel for collapse(2) schedule(static)\n"
            "  for (size_t i = 0; i < g0; ++i)\n"
            "    for (size_t j = 0; j < g1; ++j) {\n"
            "      ocl_gid[0] = i; ocl_gid[1] = j; ocl_gid[2] = 0;\n"
            "      %s(%s);\n"
            "    }\n}\n" % (name, plist, name, args))
    launch.append('#include <omp.h>\nextern "C" void ref_set_threads(int n) { omp_set_num_threads(n); }\n'
                  'extern "C" int ref_get_threads(void) { return omp_get_max_threads(); }\n')
    text = ('#include "%s"\n' % os.path.join(HERE, "opencl_shim.hpp")) + header + body + "".join(launch)
    manifest = {name: [t for t, _ in params] for name, params in sigs}
    return text, manifest


def build_block(const: us.Constants, block: dict, block_id: int, root: str | None = None):
    """Compile (or reuse) the reference program for one block.  Returns the
    path of the shared library; its manifest sits beside it as ``.json``."""
    root = root or reference_root()
    if not os.path.isdir(os.path.join(root, "source")):
        raise FileNotFoundError("reference sources not found under %s" % root)
    text, manifest = assemble(const, block, block_id, root)
    key = hashlib.sha1(text.encode()).hexdigest()[:16]
    os.makedirs(REF_OUT, exist_ok=True)
    so = os.path.join(REF_OUT, "ugks_ref_%s.so" % key)
    if not os.path.exists(so):
        cpp = os.path.join(REF_OUT, "ugks_ref_%s.cpp" % key)
        with open(cpp, "w") as fh:
            fh.write(text)
        cmd = ["g++", "-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
               "-ffp-contract=off", "-fno-strict-aliasing", "-w", cpp, "-o", so + ".tmp"]
        subprocess.run(cmd, check=True)
        os.replace(so + ".tmp", so)
        with open(so[:-3] + ".json", "w") as fh:
            json.dump(manifest, fh)
    return so


def find_built(const: us.Constants, block: dict, block_id: int):
    """Path of an already-built library for this block, or None.  Used where
    the reference sources are absent (the library was built elsewhere and
    travelled with the tree); matched through the recorded header hash."""
    idx = os.path.join(REF_OUT, "index.json")
    if not os.path.exists(idx):
        return None
    with open(idx) as fh:
        table = json.load(fh)
    so = table.get(header_key(const, block, block_id))
    if so and os.path.exists(os.path.join(REF_OUT, so)):
        return os.path.join(REF_OUT, so)
    return None


def header_key(const: us.Constants, block: dict, block_id: int) -> str:
    return hashlib.sha1(gen_header(const, block, block_id).encode()).hexdigest()[:16]


def build_and_index(const: us.Constants, block: dict, block_id: int, root: str | None = None):
    so = build_block(const, block, block_id, root)
    idx = os.path.join(REF_OUT, "index.json")
    table = {}
    if os.path.exists(idx):
        with open(idx) as fh:
            table = json.load(fh)
    table[header_key(const, block, block_id)] = os.path.basename(so)
    with open(idx, "w") as fh:
        json.dump(table, fh, indent=1)
    return so
