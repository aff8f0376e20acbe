"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs pyUGKS's own OpenCL kernels, compiled for the CPU by oracle/ref_build.py
from the reference sources (so it needs them: $UGKS_REFERENCE, else a
directory "reference" beside the repository root), driven by the oracle's restatement of the reference step
sequence (oracle/host.py), and stores macroscopic fields (rho, U, V, T, qx,
qy), dt and time at several step counts -- plus the full interior f for the
small cases -- as compressed .npz files:

    python tests/golden/make_golden.py

Cases:
  cavity8      8x8 cavity, 9x9 velocities on [-4,4]^2, vanLeer        (f, steps 1/10/50)
  multiblock8  2x2 blocks of 8x8, 9x9 velocities on [-5,5]^2, WENO5, CFL 0.3
               (f, steps 1/10/30)
  channel8     2-block adsorbing channel 8x8, Langmuir desorption, CFL 0.3
               (f + coverage, 1/10/30)
  channel8_specular / channel8_cl
               channel8 with specular (adsorbingWallS_P2) or Cercignani-Lampis
               (adsorbingWallCL_P2, alpha_n 0.5, alpha_t 0.7) re-emission
  channel8_isotherm
               channel8 with a tabulated Langmuir isotherm (configs.langmuir_table)
  cavity8_minmod
               cavity8 with the minmod (NND) limiter, FLUX_METHOD 3, CFL 0.5
  rotated8     two blocks joined NORTH to EAST, grids turned 90 degrees
               (configs.rotated_pair)
  flipped8     two blocks joined NORTH to NORTH with misaligned corners and
               orientation 1 (configs.flipped_pair)
  mirror8      one block whose S, W and E faces connect to themselves with
               FLIP_NS, FLIP_EW and FLIP_D (configs.mirror_cavity)
  periodic8    Couette flow, periodic in x through a PERIODIC (code 5) face
               (configs.periodic_couette)
  open8        channel with a CONSTANT inlet and an OUTFLOW outlet
               (configs.open_channel)
  cavity32     the 32x32 cavity, 25x25 velocities on [-4,4]^2, vanLeer, Kn 0.075,
               CFL 0.8, lid 0.15 (fields at steps 1/10/100/1000)
  multiblock_cfl03_divergence (only when named: about an hour on 8 cores)
               the benchmarked 2x2-block WENO5 cavity at CFL 0.3 run by the
               reference until its NaN flag: a trajectory every 25 steps
  cavity32_perturbed
               the same case run by the reference a second time with f
               multiplied by (1 + 1e-14 N(0,1)) after start-up (fields at
               steps 100 and 1000): the scheme amplifies round-off after ~100
               steps, and this run measures by how much
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import host  # noqa: E402
from pyugks_b200 import configs  # noqa: E402

CASES = {
    "cavity8": (lambda: configs.cavity(n=8, m=8, vlim=4.0), (1, 10, 50), True),
    "multiblock8": (lambda: configs.cavity_multiblock(nb=2, n=8, m=8), (1, 10, 30), True),
    "channel8": (lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.0), (1, 10, 30), True),
    "cavity32": (lambda: configs.cavity(n=32, m=24, vlim=4.0), (1, 10, 100, 1000), False),
    "channel8_specular": (lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.0, reflect_type="S"),
                          (1, 10, 30), True),
    "channel8_cl": (lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.0, reflect_type="CL", alpha_n=0.5,
                                            alpha_t=0.7), (1, 10, 30), True),
    "channel8_isotherm": (lambda: configs.channel(nblocks=2, n=8, m=8, k_des=0.0,
                                                  adsorb=configs.langmuir_table()), (1, 10, 30), True),
    "cavity8_minmod": (lambda: configs.cavity(n=8, m=8, vlim=4.0, flux_method="minmod", CFL=0.5),
                       (1, 10, 50), True),
    "rotated8": (lambda: configs.rotated_pair(n=8, m=8), (1, 10, 30), True),
    "flipped8": (lambda: configs.flipped_pair(n=8, m=8), (1, 10, 30), True),
    "mirror8": (lambda: configs.mirror_cavity(n=8, m=8), (1, 10, 30), True),
    "periodic8": (lambda: configs.periodic_couette(n=8, m=8), (1, 10, 30), True),
    "open8": (lambda: configs.open_channel(n=8, m=8), (1, 10, 30), True),
}


def record(sim, with_f):
    out = {"dt": np.array(sim.dt), "time": np.array(sim.time)}
    for k, fl in enumerate(sim.fields()):
        for name, arr in fl.items():
            out["b%d_%s" % (k, name)] = arr
    if with_f:
        for k, f in enumerate(sim.interior_f()):
            out["b%d_f" % k] = f
        for k, b in enumerate(sim.blocks):
            out["b%d_cover" % k] = b.wall_cover.copy()
    return out


def perturbed_envelope(name, steps, amp=1e-14, seed=0):
    """The reference against itself: the same case with f multiplied by
    (1 + amp N(0,1)) after start-up.  The field differences at `steps` are
    the round-off envelope of the reference scheme for this case."""
    make = CASES[name][0]
    a = host.OracleSim(make(), "ref", threads=os.cpu_count())
    b = host.OracleSim(make(), "ref", threads=os.cpu_count())
    rng = np.random.default_rng(seed)
    for blk in b.blocks:
        blk.f *= 1.0 + amp * rng.standard_normal(blk.f.shape)
    out = {}
    done = 0
    for s in steps:
        while done < s:
            a.one_step()
            b.one_step()
            done += 1
        for k, (x, y) in enumerate(zip(a.fields(), b.fields())):
            for key in x:
                out["s%d_b%d_%s" % (s, k, key)] = y[key]
    return out


def divergence_trajectory(every=25, limit=2000, CFL=0.3):
    """The benchmarked 2x2-block WENO5 cavity (bench.workload("multiblock"))
    run by the reference's kernels at the given CFL until a NaN or `limit`
    steps: per `every` steps dt, max |U|, max T, min rho and min f (over
    interior cells and velocities), and the step the NaN flag was raised."""
    from bench import workload
    case = workload("multiblock")[0][0]
    case["CFL"] = CFL
    sim = host.OracleSim(case, "ref", threads=os.cpu_count())
    rows, nan_step = [], -1
    for s in range(1, limit + 1):
        if sim.one_step():
            nan_step = s
            break
        if s % every == 0:
            fl = sim.fields()
            rows.append([s, sim.dt, max(float(np.max(np.abs(f["U"]))) for f in fl),
                         max(float(np.max(f["T"])) for f in fl), min(float(np.min(f["rho"])) for f in fl),
                         min(float(np.min(b.f[b.G:-b.G, b.G:-b.G, :, 0])) for b in sim.blocks)])
    return {"rows": np.array(rows), "nan_step": np.array(nan_step), "CFL": np.array(CFL)}


def main(names=None):
    for name, (make, steps, with_f) in CASES.items():
        if names and name not in names:
            continue
        sim = host.OracleSim(make(), "ref", threads=os.cpu_count())
        data = {}
        done = 0
        for s in steps:
            while done < s:
                sim.one_step()
                done += 1
            for k, v in record(sim, with_f).items():
                data["s%d_%s" % (s, k)] = v
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **data)
        print(path, os.path.getsize(path))
    if names and "multiblock_cfl03_divergence" in names:
        path = os.path.join(HERE, "multiblock_cfl03_divergence.npz")
        np.savez_compressed(path, **divergence_trajectory())
        print(path, os.path.getsize(path))
    if not names or "cavity32_perturbed" in names:
        path = os.path.join(HERE, "cavity32_perturbed.npz")
        np.savez_compressed(path, **perturbed_envelope("cavity32", (100, 1000)))
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main(sys.argv[1:])
