// ugks_kernels.cu -- drop-in CUDA kernels with the pyUGKS kernel-call surface.
//
// One entry point per OpenCL __kernel of the time-step path (declared in
// include/ugks_b200.h with the reference file:line).  Launch shape: one CTA
// of VT threads per reference work-group (the (g0, g1) NDRange, flattened);
// the threads of a CTA stride over the Nv velocities, so every velocity loop
// of the reference (LOCAL_LOOP_LENGTH iterations of LOCAL_SIZE work-items)
// becomes coalesced 16-byte (h, b) loads and the __local tree reductions
// become warp-shuffle block sums.  Kernels without a velocity loop run one
// thread per work-item.
#include <cuda_runtime.h>
#include <stddef.h>

#include "ugks_device.cuh"

using namespace ugks;

namespace {

constexpr int VT = 128;  // threads per velocity-parallel CTA

inline int launch_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -(int)e;
}
inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }
inline unsigned grid_of(size_t g0, size_t g1) { return (unsigned)(g0 * g1); }
inline unsigned grid_threads(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ void work_group(size_t g1, size_t &a, size_t &b) {
  a = blockIdx.x / g1;
  b = blockIdx.x % g1;
}

__device__ __forceinline__ bool face_range(const ugks_block_desc &d, int face, size_t mi,
                                           size_t mj, int off_top) {
  return ((face == SOUTH) && (mi < (size_t)d.ni) && (mj < (size_t)(d.nj + 1 - off_top))) ||
         ((face == WEST) && (mi < (size_t)(d.ni + 1 - off_top)) && (mj < (size_t)d.nj));
}

// ---------------------------------------------------------------------------
// iFace (clUGKS.c:110-199)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(VT) k_iFace(ugks_block_desc d, size_t g1, const double *Fin,
                                              double *iface_f, double *fsigma,
                                              const double *centre, const double *mid_side,
                                              const double *normal, int face) {
  size_t mi, mj;
  work_group(g1, mi, mj);
  if (!(((face == SOUTH) && (mi < (size_t)d.ni) && (mj < (size_t)d.nj + 1)) ||
        ((face == WEST) && (mi < (size_t)d.ni + 1) && (mj < (size_t)d.nj))))
    return;
  const long gi = mi + d.ghost, gj = mj + d.ghost;
  const V2 n = ld2(normal, faceidx(d, gi, gj, face));
  const V2 mid = ld2(mid_side, faceidx(d, gi, gj, face));
  const int L = d.flux_method == 1 ? 5 : 3, MID = d.flux_method == 1 ? 2 : 1;
  // the stencil cells for delta = 1 (flow into +normal) and delta = 0
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 uv = face_velocity(d, v, n);
    int delta = (int)((ocl_sign(uv.x) + 1) / 2);
    double fh[5], fb[5];
    V2 c[5];
#pragma unroll
    for (int s = 0; s < 5; ++s) {
      if (s >= L) break;
      long si, sj;
      if (face == SOUTH) {
        si = gi;
        sj = delta ? gj - MID - 1 + s : gj + MID - s;
      } else {
        si = delta ? gi - MID - 1 + s : gi + MID - s;
        sj = gj;
      }
      V2 f = ld2(Fin, fidx(d, si, sj, v));
      fh[s] = f.x;
      fb[s] = f.y;
      c[s] = ld2(centre, gidx(d, si, sj));
    }
    double dx = mid.x - c[MID].x, dy = mid.y - c[MID].y;
    double dist = sqrt(dx * dx + dy * dy);
    V2 sig;
    if (d.flux_method == 0) {
      double ax = c[MID].x - c[MID - 1].x, ay = c[MID].y - c[MID - 1].y;
      double l1 = sqrt(ax * ax + ay * ay);
      sig.x = vanleer((fh[MID] - fh[MID - 1]) / l1, (fh[MID + 1] - fh[MID]) / l1);
      sig.y = vanleer((fb[MID] - fb[MID - 1]) / l1, (fb[MID + 1] - fb[MID]) / l1);
    } else if (d.flux_method == 1) {
      sig.x = weno5(fh[0], fh[1], fh[2], fh[3], fh[4], dist);
      sig.y = weno5(fb[0], fb[1], fb[2], fb[3], fb[4], dist);
    } else {
      sig.x = (fh[1] + 0.5 * minmod(fh[2] - fh[1], fh[1] - fh[0]) - fh[1]) / dist;
      sig.y = (fb[1] + 0.5 * minmod(fb[2] - fb[1], fb[1] - fb[0]) - fb[1]) / dist;
    }
    st2(iface_f, fidx(d, gi, gj, v), v2(fh[MID] + sig.x * dist, fb[MID] + sig.y * dist));
    st2(fsigma, fidx(d, gi, gj, v), sig);
  }
}

// conserved moments of f in the frame of face normal n (getFaceCons/getAL/getAR)
__device__ __forceinline__ P4 frame_moments(const ugks_block_desc &d, const double *f, size_t base,
                                            V2 n, double *scratch) {
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 fv = ld2(f, base + v);
    V2 uv = face_velocity(d, v, n);
    m[0] += fv.x;
    m[1] += uv.x * fv.x;
    m[2] += uv.y * fv.x;
    m[3] += 0.5 * ((uv.x * uv.x + uv.y * uv.y) * fv.x + fv.y);
  }
  block_sum<4>(m, scratch);
  return p4(m[0], m[1], m[2], m[3]);
}

// which: 0 getFaceCons (iface f at the face), 1 getAL (left cell), 2 getAR (right cell)
__global__ void __launch_bounds__(VT) k_face_moments(ugks_block_desc d, size_t g1, const double *f,
                                                     const double *normal, int face, double *out,
                                                     int off_bot, int off_top, int which) {
  __shared__ double scratch[4 * VT / 32];
  size_t a, b;
  work_group(g1, a, b);
  size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
  if (!face_range(d, face, mi, mj, off_top)) return;
  long gi = mi + d.ghost, gj = mj + d.ghost;
  V2 n = ld2(normal, faceidx(d, gi, gj, face));
  long ci = which == 1 ? gi - face : gi, cj = which == 1 ? gj - (1 - face) : gj;
  P4 m = frame_moments(d, f, fidx(d, ci, cj, 0), n, scratch);
  if (threadIdx.x == 0) st4(out, gidx(d, gi, gj), m);
}

// ---------------------------------------------------------------------------
// getPLR (clUGKS.c:401-442), initMacroFlux (clUGKS.c:446-518)
// ---------------------------------------------------------------------------
__global__ void k_getPLR(ugks_block_desc d, size_t g0, size_t g1, const double *centre,
                         const double *mid_side, int face, double *primary, double *gaL,
                         double *gaR, int off_bot, int off_top) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= g0 * g1) return;
  size_t mi = t / g1 + face * off_bot, mj = t % g1 + (1 - face) * off_bot;
  if (!face_range(d, face, mi, mj, off_top)) return;
  long gi = mi + d.ghost, gj = mj + d.ghost;
  P4 w = ld4(primary, gidx(d, gi, gj));
  P4 prim = to_primary(d, w);
  V2 mid = ld2(mid_side, faceidx(d, gi, gj, face));
  V2 cl = ld2(centre, gidx(d, gi - face, gj - (1 - face)));
  V2 cr = ld2(centre, gidx(d, gi, gj));
  double dl = sqrt((mid.x - cl.x) * (mid.x - cl.x) + (mid.y - cl.y) * (mid.y - cl.y));
  double dr = sqrt((mid.x - cr.x) * (mid.x - cr.x) + (mid.y - cr.y) * (mid.y - cr.y));
  P4 wl = ld4(gaL, gidx(d, gi, gj)), wr = ld4(gaR, gidx(d, gi, gj));
  st4(gaL, gidx(d, gi, gj),
      micro_slope(d, prim, p4((w.s0 - wl.s0) / dl, (w.s1 - wl.s1) / dl, (w.s2 - wl.s2) / dl,
                              (w.s3 - wl.s3) / dl)));
  st4(gaR, gidx(d, gi, gj),
      micro_slope(d, prim, p4((wr.s0 - w.s0) / dr, (wr.s1 - w.s1) / dr, (wr.s2 - w.s2) / dr,
                              (wr.s3 - w.s3) / dr)));
  st4(primary, gidx(d, gi, gj), prim);
}

__device__ __forceinline__ P4 g0_macro_flux(const ugks_block_desc &d, P4 prim, P4 aL, P4 aR,
                                            double dt, P4 &aT, double Mxi[3], double Mt[5]) {
  double Mu[MNUM], Mv[MTUM], MuL[MNUM], MuR[MNUM];
  moments_u(d, prim, Mu, Mv, Mxi, MuL, MuR);
  P4 sw = scale(-prim.s0, add(moment_au(aL, MuL, Mv, Mxi, 1, 0), moment_au(aR, MuR, Mv, Mxi, 1, 0)));
  aT = micro_slope(d, prim, sw);
  time_weights(relax_time(d, prim), dt, Mt);
  P4 r = add(add(scale(Mt[0], moment_uv(Mu, Mv, Mxi, 1, 0, 0)),
                 scale(Mt[1], add(moment_au(aL, MuL, Mv, Mxi, 2, 0), moment_au(aR, MuR, Mv, Mxi, 2, 0)))),
             scale(Mt[2], moment_au(aT, Mu, Mv, Mxi, 1, 0)));
  return scale(prim.s0, r);
}

__global__ void k_initMacroFlux(ugks_block_desc d, size_t g0, size_t g1, double *flux_macro,
                                int face, double dt, const double *primary, const double *gaL,
                                const double *gaR, double *gaT, double *gMxi, int off_bot,
                                int off_top) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= g0 * g1) return;
  size_t mi = t / g1 + face * off_bot, mj = t % g1 + (1 - face) * off_bot;
  if (!face_range(d, face, mi, mj, off_top)) return;
  long gi = mi + d.ghost, gj = mj + d.ghost;
  P4 aT;
  double Mxi[3], Mt[5];
  P4 fm = g0_macro_flux(d, ld4(primary, gidx(d, gi, gj)), ld4(gaL, gidx(d, gi, gj)),
                        ld4(gaR, gidx(d, gi, gj)), dt, aT, Mxi, Mt);
  size_t k = gidx(d, gi, gj);
  gMxi[3 * k] = Mxi[0];
  gMxi[3 * k + 1] = Mxi[1];
  gMxi[3 * k + 2] = Mxi[2];
  st4(gaT, k, aT);
  st4(flux_macro, k, fm);
}

// ---------------------------------------------------------------------------
// calcFaceQ (clUGKS.c:522-585), macroFlux (587-681), distFlux (683-772)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(VT) k_calcFaceQ(ugks_block_desc d, size_t g1, const double *iface_f,
                                                  const double *primary, const double *normal,
                                                  double *faceQ, int face, int off_bot, int off_top) {
  __shared__ double scratch[2 * VT / 32];
  size_t a, b;
  work_group(g1, a, b);
  size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
  if (!face_range(d, face, mi, mj, off_top)) return;
  long gi = mi + d.ghost, gj = mj + d.ghost;
  V2 n = ld2(normal, faceidx(d, gi, gj, face));
  P4 prim = ld4(primary, gidx(d, gi, gj));
  double q[2] = {0.0, 0.0};
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 f = ld2(iface_f, fidx(d, gi, gj, v));
    V2 uv = face_velocity(d, v, n);
    double cx = uv.x - prim.s1, cy = uv.y - prim.s2, c2 = cx * cx + cy * cy;
    q[0] += 0.5 * (cx * (c2 * f.x + (f.y / d.K)));
    q[1] += 0.5 * (cy * (c2 * f.x + (f.y / d.K)));
  }
  block_sum<2>(q, scratch);
  if (threadIdx.x == 0) st2(faceQ, gidx(d, gi, gj), v2(q[0], q[1]));
}

__global__ void __launch_bounds__(VT) k_macroFlux(ugks_block_desc d, size_t g1, const double *flux_f,
                                                  const double *fsigma, double *flux_macro,
                                                  const double *normal, const double *side_length,
                                                  int face, double dt, const double *primary,
                                                  const double *faceQ, int off_bot, int off_top) {
  __shared__ double scratch[4 * VT / 32];
  size_t a, b;
  work_group(g1, a, b);
  size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
  if (!face_range(d, face, mi, mj, off_top)) return;
  long gi = mi + d.ghost, gj = mj + d.ghost;
  V2 n = ld2(normal, faceidx(d, gi, gj, face));
  P4 prim = ld4(primary, gidx(d, gi, gj));
  double Mt[5];
  time_weights(relax_time(d, prim), dt, Mt);
  V2 Q = ld2(faceQ, gidx(d, gi, gj));
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 uv = face_velocity(d, v, n);
    V2 F0 = shakhov(d, prim, Q, uv, maxwellian(d, prim, uv, v));
    V2 fd = ld2(flux_f, fidx(d, gi, gj, v));
    V2 fs = ld2(fsigma, fidx(d, gi, gj, v));
    double u = uv.x, w = uv.y, uu = u * u + w * w;
    acc[0] += Mt[0] * u * F0.x + Mt[3] * u * fd.x - Mt[4] * u * u * fs.x;
    acc[1] += Mt[0] * u * u * F0.x + Mt[3] * u * u * fd.x - Mt[4] * u * u * u * fs.x;
    acc[2] += Mt[0] * w * u * F0.x + Mt[3] * w * u * fd.x - Mt[4] * w * u * u * fs.x;
    acc[3] += Mt[0] * 0.5 * (u * uu * F0.x + u * F0.y) + Mt[3] * 0.5 * (u * uu * fd.x + u * fd.y) -
              Mt[4] * 0.5 * (u * u * uu * fs.x + u * u * fs.y);
  }
  block_sum<4>(acc, scratch);
  if (threadIdx.x == 0) {
    size_t k = gidx(d, gi, gj);
    P4 out = add(p4(acc[0], acc[1], acc[2], acc[3]), ld4(flux_macro, k));
    V2 m = to_global(v2(out.s1, out.s2), n);
    out.s1 = m.x;
    out.s2 = m.y;
    st4(flux_macro, k, scale(side_length[faceidx(d, gi, gj, face)], out));
  }
}

// per-velocity UGKS flux (clUGKS.c:751-763) given the face state
__device__ __forceinline__ V2 ugks_dist_flux(const ugks_block_desc &d, P4 prim, P4 aL, P4 aR,
                                             P4 aT, double Mxi2, const double Mt[5], V2 Q, V2 uv,
                                             int v, V2 fd, V2 fs) {
  int delta = (int)((ocl_sign(uv.x) + 1) / 2);
  V2 f0 = maxwellian(d, prim, uv, v);
  V2 F0 = shakhov(d, prim, Q, uv, f0);
  double u = uv.x, w = uv.y, uu = u * u + w * w;
  P4 a = delta ? aL : aR;
  double ph = a.s0 * f0.x + a.s1 * u * f0.x + a.s2 * w * f0.x + 0.5 * a.s3 * (uu * f0.x + f0.y);
  double pb = a.s0 * f0.y + a.s1 * u * f0.y + a.s2 * w * f0.y + 0.5 * a.s3 * (uu * f0.y + Mxi2 * f0.x);
  double th = aT.s0 * f0.x + aT.s1 * u * f0.x + aT.s2 * w * f0.x + 0.5 * aT.s3 * (uu * f0.x + f0.y);
  double tb = aT.s0 * f0.y + aT.s1 * u * f0.y + aT.s2 * w * f0.y + 0.5 * aT.s3 * (uu * f0.y + Mxi2 * f0.x);
  double hx = Mt[0] * u * (f0.x + F0.x) + Mt[1] * (u * u) * ph + Mt[2] * u * th + Mt[3] * u * fd.x -
              Mt[4] * (u * u) * fs.x;
  double hy = Mt[0] * u * (f0.y + F0.y) + Mt[1] * (u * u) * pb + Mt[2] * u * tb + Mt[3] * u * fd.y -
              Mt[4] * (u * u) * fs.y;
  return v2(hx, hy);
}

__global__ void __launch_bounds__(VT) k_distFlux(ugks_block_desc d, size_t g1, double *flux_f,
                                                 const double *fsigma, const double *normal,
                                                 const double *side_length, int face, double dt,
                                                 const double *primary, const double *gaL,
                                                 const double *gaR, const double *gaT,
                                                 const double *gMxi, const double *faceQ,
                                                 int off_bot, int off_top) {
  size_t a, b;
  work_group(g1, a, b);
  size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
  if (!face_range(d, face, mi, mj, off_top)) return;
  long gi = mi + d.ghost, gj = mj + d.ghost;
  size_t k = gidx(d, gi, gj);
  P4 prim = ld4(primary, k), aL = ld4(gaL, k), aR = ld4(gaR, k), aT = ld4(gaT, k);
  double Mxi2 = gMxi[3 * k + 2], Mt[5];
  time_weights(relax_time(d, prim), dt, Mt);
  V2 n = ld2(normal, faceidx(d, gi, gj, face));
  V2 Q = ld2(faceQ, k);
  double len = side_length[faceidx(d, gi, gj, face)];
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    size_t kv = fidx(d, gi, gj, v);
    V2 h = ugks_dist_flux(d, prim, aL, aR, aT, Mxi2, Mt, Q, face_velocity(d, v, n), v,
                          ld2(flux_f, kv), ld2(fsigma, kv));
    st2(flux_f, kv, v2(len * h.x, len * h.y));
  }
}

// ---------------------------------------------------------------------------
// walls: accommodatingWallDist (clUGKS.c:774-906), wallFlux (910-1011),
// wallMassEnergyFluxes (1019-1147)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void wall_face(const ugks_block_desc &d, int face, long &gi, long &gj,
                                          long &ci, int &rot, int &fid) {
  switch (face) {
    case GNORTH: ci = gi; gi += d.ghost; gj += d.Nj - d.ghost; rot = -1; fid = SOUTH; break;
    case GEAST: ci = gj; gi += d.Ni - d.ghost; gj += d.ghost; rot = -1; fid = WEST; break;
    case GSOUTH: ci = gi; gi += d.ghost; gj += d.ghost; rot = 1; fid = SOUTH; break;
    default: ci = gj; gi += d.ghost; gj += d.ghost; rot = 1; fid = WEST; break;
  }
}
__device__ __forceinline__ bool wall_range(const ugks_block_desc &d, int fid, long gi, long gj) {
  return ((fid == SOUTH) && ((size_t)(gi - d.ghost) < (size_t)d.ni)) ||
         ((fid == WEST) && ((size_t)(gj - d.ghost) < (size_t)d.nj));
}

__global__ void __launch_bounds__(VT) k_accommodatingWallDist(ugks_block_desc d, size_t g1,
                                                              const double *normal, int face,
                                                              const double *wall_prop,
                                                              double *flux_f) {
  __shared__ double scratch[2 * VT / 32];
  size_t a, b;
  work_group(g1, a, b);
  long gi = a, gj = b, ci;
  int rot, fid;
  wall_face(d, face, gi, gj, ci, rot, fid);
  if (!wall_range(d, fid, gi, gj)) return;
  V2 n = ld2(normal, faceidx(d, gi, gj, fid));
  P4 wall = ld4(wall_prop, ci * 4 + face);
  V2 wl = to_local(v2(wall.s1, wall.s2), n);
  wall.s1 = wl.x;
  wall.s2 = wl.y;
  double s[2] = {0.0, 0.0};
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 uv = face_velocity(d, v, n);
    V2 fd = ld2(flux_f, fidx(d, gi, gj, v));
    int delta = upwind_flag(uv.x, rot);
    s[0] += uv.x * (1 - delta) * fd.x;
    s[1] -= uv.x * delta * maxwellian(d, wall, uv, v).x;
  }
  block_sum<2>(s, scratch);
  double ratio = s[0] / s[1];
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 uv = face_velocity(d, v, n);
    int delta = upwind_flag(uv.x, rot);
    size_t kv = fidx(d, gi, gj, v);
    V2 fd = ld2(flux_f, kv);
    V2 M = maxwellian(d, wall, uv, v);
    st2(flux_f, kv, v2(ratio * delta * M.x + (1 - delta) * fd.x, ratio * delta * M.y + (1 - delta) * fd.y));
  }
}

__global__ void __launch_bounds__(VT) k_wallFlux(ugks_block_desc d, size_t g1, const double *normal,
                                                 const double *side_length, int face,
                                                 double *flux_f, double *flux_macro, double dt) {
  __shared__ double scratch[4 * VT / 32];
  size_t a, b;
  work_group(g1, a, b);
  long gi = a, gj = b, ci;
  int rot, fid;
  wall_face(d, face, gi, gj, ci, rot, fid);
  if (!wall_range(d, fid, gi, gj)) return;
  V2 n = ld2(normal, faceidx(d, gi, gj, fid));
  double len = side_length[faceidx(d, gi, gj, fid)];
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 uv = face_velocity(d, v, n);
    size_t kv = fidx(d, gi, gj, v);
    V2 wd = ld2(flux_f, kv);
    st2(flux_f, kv, v2(uv.x * wd.x * len * dt, uv.x * wd.y * len * dt));
    m[0] += uv.x * wd.x;
    m[1] += uv.x * uv.x * wd.x;
    m[2] += uv.x * uv.y * wd.x;
    m[3] += 0.5 * uv.x * ((uv.x * uv.x + uv.y * uv.y) * wd.x + wd.y);
  }
  block_sum<4>(m, scratch);
  if (threadIdx.x == 0) {
    V2 g = to_global(v2(m[1], m[2]), n);
    st4(flux_macro, gidx(d, gi, gj), scale(dt * len, p4(m[0], g.x, g.y, m[3])));
  }
}

__global__ void __launch_bounds__(VT) k_wallMassEnergyFluxes(ugks_block_desc d, size_t g1,
                                                             const double *normal, int face,
                                                             const double *flux_f,
                                                             double *wall_flux) {
  __shared__ double scratch[8 * VT / 32];
  size_t a, b;
  work_group(g1, a, b);
  long gi = a, gj = b, ci;
  int rot, fid;
  wall_face(d, face, gi, gj, ci, rot, fid);
  if (!wall_range(d, fid, gi, gj)) return;
  V2 n = ld2(normal, faceidx(d, gi, gj, fid));
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 uv = face_velocity(d, v, n);
    int delta = upwind_flag(uv.x, rot);
    V2 wd = ld2(flux_f, fidx(d, gi, gj, v));
    double uu = uv.x * uv.x + uv.y * uv.y;
    double ix = (1 - delta) * wd.x, iy = (1 - delta) * wd.y, ox = delta * wd.x, oy = delta * wd.y;
    s[0] += ix; s[1] += uv.x * ix; s[2] += uv.y * ix; s[3] += 0.5 * (uu * ix + iy);
    s[4] += ox; s[5] += uv.x * ox; s[6] += uv.y * ox; s[7] += 0.5 * (uu * ox + oy);
  }
  block_sum<8>(s, scratch);
  if (threadIdx.x == 0) {
    double *w = wall_flux + 8 * (ci * 4 + face);
    w[0] = -rot * s[0]; w[1] = rot * s[4]; w[2] = -rot * s[1]; w[3] = rot * s[5];
    w[4] = -rot * s[2]; w[5] = rot * s[6]; w[6] = -rot * s[3]; w[7] = rot * s[7];
  }
}

// ---------------------------------------------------------------------------
// cell kernels: updateMacro (clUGKS.c:1158-1187), UGKS_update (1189-1257),
// getResidual (1259-1277), calcQ / calcMacro / initFunctions (clKernel.c)
// ---------------------------------------------------------------------------
__global__ void k_updateMacro(ugks_block_desc d, size_t g0, size_t g1, const double *fmS,
                              const double *fmW, const double *area, double *macro,
                              double *residual) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= g0 * g1) return;
  size_t mi = t / g1, mj = t % g1;
  if (!(mi < (size_t)d.ni && mj < (size_t)d.nj)) return;
  long gi = mi + d.ghost, gj = mj + d.ghost;
  P4 old = ld4(macro, midx(d, mi, mj));
  P4 w = to_conserved(d, old);
  double A = area[gidx(d, gi, gj)];
  P4 s0 = ld4(fmS, gidx(d, gi, gj)), s1 = ld4(fmS, gidx(d, gi, gj + 1));
  P4 w0 = ld4(fmW, gidx(d, gi, gj)), w1 = ld4(fmW, gidx(d, gi + 1, gj));
  P4 nw = p4(w.s0 + (s0.s0 - s1.s0 + w0.s0 - w1.s0) / A, w.s1 + (s0.s1 - s1.s1 + w0.s1 - w1.s1) / A,
             w.s2 + (s0.s2 - s1.s2 + w0.s2 - w1.s2) / A, w.s3 + (s0.s3 - s1.s3 + w0.s3 - w1.s3) / A);
  st4(macro, midx(d, mi, mj), to_primary(d, nw));
  st4(residual, midx(d, mi, mj), old);
}

__global__ void __launch_bounds__(VT) k_UGKS_update(ugks_block_desc d, size_t g1, double *Fin,
                                                    const double *fS, const double *fW,
                                                    const double *area, const double *macro,
                                                    const double *gQ, const double *residual,
                                                    double dt, double *flag) {
  size_t mi, mj;
  work_group(g1, mi, mj);
  long gi = mi + d.ghost, gj = mj + d.ghost;
  P4 prim_old = ld4(residual, midx(d, mi, mj));
  double tau_old = relax_time(d, prim_old);
  V2 Q = ld2(gQ, midx(d, mi, mj));
  P4 prim = ld4(macro, midx(d, mi, mj));
  double tau = relax_time(d, prim);
  double A = area[gidx(d, gi, gj)];
  bool nan = false;
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 e = quad_at(d, v);
    V2 fo = shakhov_eq(d, prim_old, Q, e, v);
    V2 fn = shakhov_eq(d, prim, Q, e, v);
    size_t kv = fidx(d, gi, gj, v);
    V2 f = ld2(Fin, kv);
    V2 a0 = ld2(fS, kv), a1 = ld2(fS, fidx(d, gi, gj + 1, v));
    V2 b0 = ld2(fW, kv), b1 = ld2(fW, fidx(d, gi + 1, gj, v));
    double flh = (a0.x - a1.x + b0.x - b1.x) / A, flb = (a0.y - a1.y + b0.y - b1.y) / A;
    double rh = fn.x / tau + (fo.x - f.x) / tau_old, rb = fn.y / tau + (fo.y - f.y) / tau_old;
    double den = 1.0 + 0.5 * dt / tau;
    V2 out = v2((f.x + flh + 0.5 * dt * rh) / den, (f.y + flb + 0.5 * dt * rb) / den);
    nan |= isnan(out.x) || isnan(out.y);
    st2(Fin, kv, out);
  }
  if (nan) flag[0] = 1.0;
}

__global__ void k_getResidual(ugks_block_desc d, size_t g0, size_t g1, const double *macro,
                              double *residual) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= g0 * g1) return;
  size_t mi = t / g1, mj = t % g1;
  if (!(mi < (size_t)d.ni && mj < (size_t)d.nj)) return;
  for (int k = 0; k < 4; ++k) {
    double x = macro[4 * midx(d, mi, mj) + k] - residual[4 * midx(d, mi, mj) + k];
    residual[4 * midx(d, mi, mj) + k] = x * x;
  }
}

__global__ void k_edgeMassFlow(ugks_block_desc d, size_t g0, const double *macro,
                               const double *normal, const double *side_length, double *mdot,
                               int this_face) {
  size_t ci = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (ci >= g0) return;
  long mi, mj, gi, gj;
  int face;
  double dir;
  if (this_face == GNORTH) { mi = ci; mj = d.nj - 1; gi = d.ghost + ci; gj = d.Nj - d.ghost; face = SOUTH; dir = 1; }
  else if (this_face == GEAST) { mi = d.ni - 1; mj = ci; gi = d.Ni - d.ghost; gj = d.ghost + ci; face = WEST; dir = 1; }
  else if (this_face == GSOUTH) { mi = ci; mj = 0; gi = d.ghost + ci; gj = d.ghost; face = SOUTH; dir = -1; }
  else { mi = 0; mj = ci; gi = d.ghost; gj = d.ghost + ci; face = WEST; dir = -1; }
  V2 n = ld2(normal, faceidx(d, gi, gj, face));
  double len = side_length[faceidx(d, gi, gj, face)];
  P4 m = ld4(macro, midx(d, mi, mj));
  mdot[ci * 4 + this_face] = (dir * n.x * m.s1 + dir * n.y * m.s2) * m.s0 * len;
}

__global__ void __launch_bounds__(VT) k_calcQ(ugks_block_desc d, size_t g1, const double *Fin,
                                              const double *macro, double *gQ) {
  __shared__ double scratch[2 * VT / 32];
  size_t mi, mj;
  work_group(g1, mi, mj);
  if (!(mi < (size_t)d.ni && mj < (size_t)d.nj)) return;
  long gi = mi + d.ghost, gj = mj + d.ghost;
  P4 prim = ld4(macro, midx(d, mi, mj));
  double q[2] = {0.0, 0.0};
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 f = ld2(Fin, fidx(d, gi, gj, v));
    V2 e = quad_at(d, v);
    double cx = e.x - prim.s1, cy = e.y - prim.s2, c2 = cx * cx + cy * cy;
    q[0] += 0.5 * (cx * (c2 * f.x + (f.y / d.K)));
    q[1] += 0.5 * (cy * (c2 * f.x + (f.y / d.K)));
  }
  block_sum<2>(q, scratch);
  if (threadIdx.x == 0) st2(gQ, midx(d, mi, mj), v2(q[0], q[1]));
}

__global__ void __launch_bounds__(VT) k_calcMacro(ugks_block_desc d, size_t g1, const double *Fin,
                                                  double *macro) {
  __shared__ double scratch[4 * VT / 32];
  size_t mi, mj;
  work_group(g1, mi, mj);
  if (!(mi < (size_t)d.ni && mj < (size_t)d.nj)) return;
  long gi = mi + d.ghost, gj = mj + d.ghost;
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 f = ld2(Fin, fidx(d, gi, gj, v));
    V2 e = quad_at(d, v);
    m[0] += f.x;
    m[1] += e.x * f.x;
    m[2] += e.y * f.x;
    m[3] += 0.5 * ((e.x * e.x + e.y * e.y) * f.x + f.y);
  }
  block_sum<4>(m, scratch);
  if (threadIdx.x == 0) st4(macro, midx(d, mi, mj), to_primary(d, p4(m[0], m[1], m[2], m[3])));
}

__global__ void __launch_bounds__(VT) k_initFunctions(ugks_block_desc d, size_t g1, double *Fin,
                                                      const double *macro, const double *gQ) {
  size_t mi, mj;
  work_group(g1, mi, mj);
  if (!(mi < (size_t)d.ni && mj < (size_t)d.nj)) return;
  long gi = mi + d.ghost, gj = mj + d.ghost;
  P4 prim = ld4(macro, midx(d, mi, mj));
  V2 Q = ld2(gQ, midx(d, mi, mj));
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x)
    st2(Fin, fidx(d, gi, gj, v), shakhov_eq(d, prim, Q, quad_at(d, v), v));
}

// clFindDT (clKernel.c:224-308): cfl_frequency of ugks_device.cuh per cell
__global__ void k_clFindDT(ugks_block_desc d, size_t g0, size_t g1, const double *xy,
                           const double *area, const double *macro, double *time_step, double Kn) {
  size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= g0 * g1) return;
  long mi = t / g1, mj = t % g1;
  time_step[midx(d, mi, mj)] = cfl_frequency(d, xy, area, ld4(macro, midx(d, mi, mj)), mi, mj, Kn);
}

__global__ void k_array_max(const double *x, size_t n, double *out) {
  __shared__ double sm[32];
  double m = -INFINITY;
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, x[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = sm[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sm[w]);
    out[0] = r;
  }
}

__global__ void k_paraBC(ugks_block_desc d, size_t g0, double *wall_prop) {
  size_t ci = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (ci >= g0) return;
  for (int f = 0; f < 4; ++f) {
    bool ns = (f == GNORTH || f == GSOUTH);
    if (ns ? !(ci < (size_t)d.ni) : !(ci < (size_t)d.nj)) continue;
    double l = (d.wall_P[f] != -1) ? d.wall_P[f] / d.wall_D[f] : d.wall_T[f];
    st4(wall_prop, ci * 4 + f, p4(d.wall_D[f], d.wall_U[f], d.wall_V[f], l));
  }
}

// ---------------------------------------------------------------------------
// ghost-cell kernels (clGhostRoutines.c)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void ghost_cell(const ugks_block_desc &d, int face, long &gi, long &gj) {
  switch (face) {
    case GNORTH: gi += d.ghost; gj += d.Nj - d.ghost; break;
    case GEAST: gi += d.Ni - d.ghost; gj += d.ghost; break;
    case GSOUTH: gi += d.ghost; break;
    default: gj += d.ghost; break;
  }
}

}  // namespace

namespace {

__device__ __forceinline__ void face_corners(int face, int NI, int NJ, int G, int &a1i, int &a1j,
                                             int &a2i, int &a2j) {
  switch (face) {
    case GNORTH: a1i = G; a1j = NJ - G; a2i = NI - G; a2j = NJ - G; break;
    case GEAST: a1i = NI - G; a1j = G; a2i = NI - G; a2j = NJ - G; break;
    case GSOUTH: a1i = G; a1j = G; a2i = NI - G; a2j = G; break;
    default: a1i = G; a1j = G; a2i = G; a2j = NJ - G; break;
  }
}

__global__ void __launch_bounds__(VT) k_edgeExchange(ugks_block_desc d, size_t g1, double *fA,
                                                     const double *xyA, int this_face,
                                                     const double *fB, const double *xyB, int NIB,
                                                     int NJB, int that_face, int ori, int flip) {
  size_t a, b;
  work_group(g1, a, b);
  const int G = d.ghost, NI = d.Ni, NJ = d.Nj;
  int a1i, a1j, a2i, a2j, b1i, b1j, b2i, b2j;
  face_corners(this_face, NI, NJ, G, a1i, a1j, a2i, a2j);
  face_corners(that_face, NIB, NJB, G, b1i, b1j, b2i, b2j);
  V2 A1 = ld2(xyA, (size_t)a1i * (NJ + 1) + a1j), A2 = ld2(xyA, (size_t)a2i * (NJ + 1) + a2j);
  V2 B1 = ld2(xyB, (size_t)b1i * (NJB + 1) + b1j), B2 = ld2(xyB, (size_t)b2i * (NJB + 1) + b2j);
  bool misalign = !(fabs(A1.x - B1.x) <= 1e-6) || !(fabs(A1.y - B1.y) <= 1e-6) ||
                  !(fabs(A2.x - B2.x) <= 1e-6) || !(fabs(A2.y - B2.y) <= 1e-6);
  long gi = a, gj = b;
  ghost_cell(d, this_face, gi, gj);
  int iB = (int)gi, jB = (int)gj;
  if (misalign && ori) {
    if (this_face == GEAST || this_face == GWEST) jB = (NJ - 1) - jB;
    else iB = (NI - 1) - iB;
  }
  swap_cell_index(NI, NJ, G, this_face, iB, jB, that_face, NIB, NJB);
  if (iB < 0 || iB >= NIB || jB < 0 || jB >= NJB) return;  // connection does not map
  const double2 *src = reinterpret_cast<const double2 *>(fB) + ((size_t)iB * NJB + jB) * (size_t)d.Nv;
  double2 *dst = reinterpret_cast<double2 *>(fA) + fidx(d, gi, gj, 0);
  const int32_t *perm = flip == FLIP_NS ? d.mirror_NS : (flip == FLIP_D ? d.mirror_D : d.mirror_EW);
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) dst[v] = src[flip == NO_FLIP ? v : perm[v]];
}

__global__ void __launch_bounds__(VT) k_edgeExtrapolate(ugks_block_desc d, size_t g1, double *Fin,
                                                        int this_face) {
  size_t a, b;
  work_group(g1, a, b);
  long gi = a, gj = b, ei, ej;
  ghost_cell(d, this_face, gi, gj);
  switch (this_face) {
    case GNORTH: ei = gi; ej = d.Nj - d.ghost - 1; break;
    case GEAST: ei = d.Ni - d.ghost - 1; ej = gj; break;
    case GSOUTH: ei = gi; ej = d.ghost; break;
    default: ei = d.ghost; ej = gj; break;
  }
  double2 *F = reinterpret_cast<double2 *>(Fin);
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) F[fidx(d, gi, gj, v)] = F[fidx(d, ei, ej, v)];
}

__global__ void __launch_bounds__(VT) k_edgeConstant(ugks_block_desc d, size_t g1, double *Fin,
                                                     int this_face, const double *wall_prop) {
  size_t a, b;
  work_group(g1, a, b);
  long gi = a, gj = b;
  size_t ci = (this_face == GNORTH || this_face == GSOUTH) ? a : b;
  ghost_cell(d, this_face, gi, gj);
  P4 prim = ld4(wall_prop, ci * 4 + this_face);
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x)
    st2(Fin, fidx(d, gi, gj, v), shakhov_eq(d, prim, v2(0.0, 0.0), quad_at(d, v), v));
}

__global__ void __launch_bounds__(VT) k_edgeInOut(ugks_block_desc d, size_t g1, double *Fin,
                                                  int this_face, const double *normal,
                                                  const double *macro, const double *gQ,
                                                  const double *wall_prop, int outflow) {
  size_t a, b;
  work_group(g1, a, b);
  long gi = a, gj = b, ei, ej, noi, noj;
  size_t ci;
  int face;
  ghost_cell(d, this_face, gi, gj);
  switch (this_face) {
    case GNORTH: ci = a; ei = gi; ej = d.Nj - d.ghost - 1; noi = gi; noj = gj; face = SOUTH; break;
    case GEAST: ci = b; ei = d.Ni - d.ghost - 1; ej = gj; noi = gi; noj = gj; face = WEST; break;
    case GSOUTH: ci = a; ei = gi; ej = d.ghost; noi = ei; noj = ej; face = SOUTH; break;
    default: ci = b; ei = d.ghost; ej = gj; noi = ei; noj = ej; face = WEST; break;
  }
  P4 prim = ld4(wall_prop, ci * 4 + this_face);
  V2 Q = ld2(gQ, midx(d, ei - d.ghost, ej - d.ghost));
  P4 gm = ld4(macro, midx(d, ei - d.ghost, ej - d.ghost));
  V2 uv = to_local(v2(gm.s1, gm.s2), ld2(normal, faceidx(d, noi, noj, face)));
  gm.s1 = uv.x;
  gm.s2 = uv.y;
  if (outflow) {
    gm.s3 = gm.s0 / (prim.s0 / prim.s3);
  } else {
    gm.s0 = prim.s0;
    gm.s3 = prim.s3;
  }
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x)
    st2(Fin, fidx(d, gi, gj, v), shakhov_eq(d, gm, Q, quad_at(d, v), v));
}

__global__ void __launch_bounds__(VT) k_edgeMirror(ugks_block_desc d, size_t g1, double *Fin,
                                                   int this_face, int bounce) {
  size_t a, b;
  work_group(g1, a, b);
  long gi = a, gj = b, mi, mj;
  ghost_cell(d, this_face, gi, gj);
  const int32_t *perm;
  switch (this_face) {
    case GNORTH: mi = gi; mj = 2 * (d.Nj - d.ghost) - gj - 1; perm = d.mirror_NS; break;
    case GEAST: mi = 2 * (d.Ni - d.ghost) - gi - 1; mj = gj; perm = d.mirror_EW; break;
    case GSOUTH: mi = gi; mj = 2 * d.ghost - gj - 1; perm = d.mirror_NS; break;
    default: mi = 2 * d.ghost - gi - 1; mj = gj; perm = d.mirror_EW; break;
  }
  if (bounce) perm = d.mirror_D;
  double2 *F = reinterpret_cast<double2 *>(Fin);
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) F[fidx(d, gi, gj, v)] = F[fidx(d, mi, mj, perm[v])];
}

__global__ void __launch_bounds__(VT) k_edgeConstGrad(ugks_block_desc d, size_t g1, double *Fin,
                                                      int this_face) {
  size_t a, b;
  work_group(g1, a, b);
  long gi = a, gj = b, ei0, ej0, ei1, ej1;
  double m;
  ghost_cell(d, this_face, gi, gj);
  switch (this_face) {
    case GNORTH: ei1 = gi; ej1 = d.Nj - d.ghost - 1; ei0 = ei1; ej0 = ej1 - 1; m = (double)(gj - ej1); break;
    case GEAST: ei1 = d.Ni - d.ghost - 1; ej1 = gj; ei0 = ei1 - 1; ej0 = ej1; m = (double)(gi - ei1); break;
    case GSOUTH: ei1 = gi; ej1 = d.ghost; ei0 = ei1; ej0 = ej1 + 1; m = (double)(ej1 - gj); break;
    default: ei1 = d.ghost; ej1 = gj; ei0 = ei1 + 1; ej0 = ej1; m = (double)(ei1 - gi); break;
  }
  double2 *F = reinterpret_cast<double2 *>(Fin);
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    double2 f0 = F[fidx(d, ei0, ej0, v)], f1 = F[fidx(d, ei1, ej1, v)];
    // unfused multiply and add: the same rounding as the reference
    F[fidx(d, gi, gj, v)] = make_double2(__dadd_rn(f1.x, __dmul_rn(m, __dsub_rn(f1.x, f0.x))),
                                         __dadd_rn(f1.y, __dmul_rn(m, __dsub_rn(f1.y, f0.y))));
  }
}

// ---------------------------------------------------------------------------
// adsorbing wall: adsorbingWall_P1 (clAdsorb.c:253-482), adsorbingWallD_P2
// (clAdsorb.c:821-975)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(VT) k_adsorbingWall_P1(ugks_block_desc d, size_t g1,
                                                         const double *normal, int face,
                                                         double *wall_cover, double *wall_dist,
                                                         const double *flux_f, const double *macro,
                                                         double dt, double *flag) {
  __shared__ double scratch[3 * VT / 32];
  __shared__ double correct_sh;
  size_t a, b;
  work_group(g1, a, b);
  long gi = a, gj = b, ci;
  int rot, fid;
  wall_face(d, face, gi, gj, ci, rot, fid);
  size_t mc;  // the cell beside the wall face
  switch (face) {
    case GNORTH: mc = midx(d, ci, gj - d.ghost - 1); break;
    case GEAST: mc = midx(d, gi - d.ghost - 1, ci); break;
    case GSOUTH: mc = midx(d, ci, gj - d.ghost); break;
    default: mc = midx(d, gi - d.ghost, ci); break;
  }
  const double T = 1.0 / macro[4 * mc + 3], D = macro[4 * mc];
  if (!wall_range(d, fid, gi, gj)) return;
  V2 n = ld2(normal, faceidx(d, gi, gj, fid));
  double *cover = wall_cover + 4 * (ci * 4 + face);
  const double theta = cover[0];
  const double gf = d.gamma_f[face];
  double s[3] = {0.0, 0.0, 0.0};  // reflected, adsorbed, flux seen by the Langmuir reaction
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 uv = face_velocity(d, v, n);
    V2 fd = ld2(flux_f, fidx(d, gi, gj, v));
    int delta = upwind_flag(uv.x, rot);
    double k = -rot * uv.x * (1 - delta);
    V2 total = v2(k * fd.x, k * fd.y);
    double beta = sticking(d, uv, T, face);
    V2 ads = v2(beta * total.x * gf * (1.0 - theta), beta * total.y * gf * (1.0 - theta));
    double fs = ocl_sign(total.x);
    if ((fs * ads.x) > (fs * total.x)) ads = total;
    V2 refl = v2(total.x - ads.x, total.y - ads.y);
    s[0] += refl.x;
    s[1] += ads.x;
    s[2] += beta * total.x;
    st2(wall_dist, (size_t)ci * d.Nv + v, v2(refl.x / uv.x, refl.y / uv.x));
  }
  block_sum<3>(s, scratch);
  if (threadIdx.x == 0) {
    double ads_final = s[1], dvt = 0.0, des = 0.0;
    bool ok = true;
    if (gf > 0.0) {
      if (d.dynamic[face] == 1) {
        dvt = dt * d.alpha_p[face] * s[1];
        if (dvt > (1 - theta)) {
          dvt = 1 - theta;
          ads_final = dvt / dt * d.alpha_p[face];  // the reference's form (clAdsorb.c:420)
        }
      }
      if (d.k_des[face] > 0.0) {
        // first-order desorption k_des * theta (no counterpart in the reference)
        des = d.k_des[face] * theta / d.alpha_p[face];
      } else {
        // Langmuir desorption with the equilibrium coverage of the isotherm
        const V2 veq = vartheta_langmuir(d, D, T, face);
        if (veq.y == 1.0) {
          flag[0] = 4.0;  // outside the tabulated isotherm
          ok = false;
        } else {
          des = gf * (1.0 / veq.x - 1.0) * s[2] * theta;
        }
      }
      if (ok) {
        if (d.dynamic[face] == 1) {
          dvt -= dt * d.alpha_p[face] * des;
          if ((theta + dvt) < 0.0) des = theta / (dt * d.alpha_p[face]);
        }
      }
    }
    double correct = 1.0;
    if (ok) {
      double refl_final = s[0] + s[1] - ads_final;
      correct = refl_final / s[0];
      cover[0] += dvt;
      cover[1] = refl_final;
      cover[2] = ads_final;
      cover[3] = des;
    }
    correct_sh = correct;
  }
  __syncthreads();
  const double c = correct_sh;
  if (c != 1.0)
    for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
      size_t k = (size_t)ci * d.Nv + v;
      V2 w = ld2(wall_dist, k);
      st2(wall_dist, k, v2(w.x * c, w.y * c));
    }
}

// getInternal (clKernel.c:314-375): one work group per interior cell;
// directional temperatures (Tx, Ty, Tz, T) and stress (xx, xy, yy, 0) from
// the moments of f
__global__ void __launch_bounds__(VT) k_getInternal(ugks_block_desc d, size_t g1, const double *Fin, double *Txyz,
                                                    double *Stress) {
  __shared__ double scratch[7 * VT / 32];
  size_t a, b;
  work_group(g1, a, b);
  if (!(a < (size_t)d.ni && b < (size_t)d.nj)) return;
  const long gi = a + d.ghost, gj = b + d.ghost;
  double m[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // D, M1, M2, M4, M5, M6, H
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    const V2 uv = quad_at(d, v);
    const V2 f = ld2(Fin, fidx(d, gi, gj, v));
    m[0] += f.x;
    m[1] += uv.x * f.x;
    m[2] += uv.y * f.x;
    m[3] += uv.x * uv.x * f.x;
    m[4] += uv.y * uv.y * f.x;
    m[5] += uv.x * uv.y * f.x;
    m[6] += f.y;
  }
  block_sum<7>(m, scratch);
  if (threadIdx.x == 0) {
    const double D = m[0], U = m[1] / D, V = m[2] / D;
    const double Tx = 2 * (m[3] / D - U * U), Ty = 2 * (m[4] / D - V * V), Tz = 2 * (m[6] / D);
    const double T = (Tx + Ty + Tz) / d.B;
    const size_t k = midx(d, a, b);
    st4(Txyz, k, p4(Tx, Ty, Tz, T));
    st4(Stress, k, p4(m[3] - D * (U * U + T / 2.0), m[5] - D * (U * V + T / 2.0), m[4] - D * (V * V + T / 2.0), 0.0));
  }
}

// adsorbingWallS_P2 (clAdsorb.c:656-816) and adsorbingWallCL_P2
// (clAdsorb.c:488-651): the reflected part of the incoming flux (wall_dist,
// per incoming velocity, from adsorbingWall_P1) is re-emitted specularly,
// through the velocity mirrored about the wall, or through the
// Cercignani-Lampis kernel (an O(Nv^2) sum over incoming velocities); then,
// as for diffuse re-emission, scaled to the reflected flux and the desorbed
// particles added
template <int KIND>
__global__ void __launch_bounds__(VT) k_adsorbingWallSCL_P2(ugks_block_desc d, size_t g1,
                                                            const double *normal, int face,
                                                            const double *wall_prop,
                                                            const double *wall_cover,
                                                            const double *wall_dist, double *flux_f) {
  __shared__ double scratch[VT / 32];
  size_t a, b;
  work_group(g1, a, b);
  long gi = a, gj = b, ci;
  int rot, fid;
  wall_face(d, face, gi, gj, ci, rot, fid);
  if (!wall_range(d, fid, gi, gj)) return;
  V2 n = ld2(normal, faceidx(d, gi, gj, fid));
  P4 wall = ld4(wall_prop, ci * 4 + face);
  V2 wl = to_local(v2(wall.s1, wall.s2), n);
  wall.s1 = wl.x;
  wall.s2 = wl.y;
  const double *cover = wall_cover + 4 * (ci * 4 + face);
  const double refl = cover[1];
  double ratio = 1.0;
  if (refl > 0.0) {
    double s[1] = {0.0};
    const double an = d.alpha_n[face], at = d.alpha_t[face], Tw = 1.0 / wall.s3;
    for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
      V2 uv = face_velocity(d, v, n);
      int delta = upwind_flag(uv.x, rot);
      V2 out = v2(0.0, 0.0);
      if (delta) {
        if (KIND == UGKS_REFLECT_SPECULAR) {
          const int mv = fid == WEST ? d.mirror_EW[v] : d.mirror_NS[v];
          out = ld2(wall_dist, (size_t)ci * d.Nv + mv);
        } else {
          for (int va = 0; va < d.Nv; ++va) {
            const V2 uv_in = face_velocity(d, va, n);
            if (!upwind_flag(uv_in.x, rot) && uv_in.x != 0.0) {
              const V2 c = cercignani_lampis(d.PI, uv_in, uv, ld2(wall_dist, (size_t)ci * d.Nv + va), an, at, Tw,
                                             wall.s3);
              out.x += c.x;
              out.y += c.y;
            }
          }
          out.x *= d.weight[v];
          out.y *= d.weight[v];
        }
      }
      size_t kv = fidx(d, gi, gj, v);
      V2 fd = ld2(flux_f, kv);
      st2(flux_f, kv, v2(delta * out.x + (1 - delta) * fd.x, delta * out.y + (1 - delta) * fd.y));
      s[0] += rot * uv.x * out.x;
    }
    block_sum<1>(s, scratch);
    ratio = refl / s[0];
  }
  const double des = cover[3], ads = cover[2];
  const int account = ((des == 0.0) && (ads > 0.0) && (refl == 0.0)) ? 1 : 0;
  P4 wd = wall;
  wd.s0 = 2 * des * sqrt(d.PI * wall.s3);
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 uv = face_velocity(d, v, n);
    int delta = upwind_flag(uv.x, rot);
    size_t kv = fidx(d, gi, gj, v);
    V2 fd = ld2(flux_f, kv);
    double sc = 1 - delta * (1 - ratio);
    fd.x *= sc;
    fd.y *= sc;
    V2 M = maxwellian(d, wd, uv, v);
    fd.x += delta * M.x;
    fd.y += delta * M.y;
    fd.x -= account * delta * fd.x;
    fd.y -= account * delta * fd.y;
    st2(flux_f, kv, fd);
  }
}

__global__ void __launch_bounds__(VT) k_adsorbingWallD_P2(ugks_block_desc d, size_t g1,
                                                          const double *normal, int face,
                                                          const double *wall_prop,
                                                          const double *wall_cover,
                                                          double *flux_f) {
  __shared__ double scratch[VT / 32];
  size_t a, b;
  work_group(g1, a, b);
  long gi = a, gj = b, ci;
  int rot, fid;
  wall_face(d, face, gi, gj, ci, rot, fid);
  if (!wall_range(d, fid, gi, gj)) return;
  V2 n = ld2(normal, faceidx(d, gi, gj, fid));
  P4 wall = ld4(wall_prop, ci * 4 + face);
  V2 wl = to_local(v2(wall.s1, wall.s2), n);
  wall.s1 = wl.x;
  wall.s2 = wl.y;
  const double *cover = wall_cover + 4 * (ci * 4 + face);
  const double refl = cover[1];
  double ratio = 1.0;
  if (refl > 0.0) {
    double s[1] = {0.0};
    for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
      V2 uv = face_velocity(d, v, n);
      int delta = upwind_flag(uv.x, rot);
      V2 dif = delta ? maxwellian(d, wall, uv, v) : v2(0.0, 0.0);
      size_t kv = fidx(d, gi, gj, v);
      V2 fd = ld2(flux_f, kv);
      st2(flux_f, kv, v2(delta * dif.x + (1 - delta) * fd.x, delta * dif.y + (1 - delta) * fd.y));
      s[0] += rot * uv.x * dif.x;
    }
    block_sum<1>(s, scratch);
    ratio = refl / s[0];
  }
  const double des = cover[3], ads = cover[2];
  const int account = ((des == 0.0) && (ads > 0.0) && (refl == 0.0)) ? 1 : 0;
  P4 wd = wall;
  wd.s0 = 2 * des * sqrt(d.PI * wall.s3);
  for (int v = threadIdx.x; v < d.Nv; v += blockDim.x) {
    V2 uv = face_velocity(d, v, n);
    int delta = upwind_flag(uv.x, rot);
    size_t kv = fidx(d, gi, gj, v);
    V2 fd = ld2(flux_f, kv);
    double sc = 1 - delta * (1 - ratio);
    fd.x *= sc;
    fd.y *= sc;
    V2 M = maxwellian(d, wd, uv, v);
    fd.x += delta * M.x;
    fd.y += delta * M.y;
    fd.x -= account * delta * fd.x;
    fd.y -= account * delta * fd.y;
    st2(flux_f, kv, fd);
  }
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
#define VEL_LAUNCH(kernel, ...)                                                       \
  do {                                                                                \
    if (g0 * g1 == 0) return 0;                                                       \
    kernel<<<grid_of(g0, g1), VT, 0, S(stream)>>>(*d, g1, __VA_ARGS__);               \
    return launch_status();                                                           \
  } while (0)
#define PT_LAUNCH(kernel, n, ...)                                                     \
  do {                                                                                \
    if ((n) == 0) return 0;                                                           \
    kernel<<<grid_threads((n), 128), 128, 0, S(stream)>>>(*d, __VA_ARGS__);           \
    return launch_status();                                                           \
  } while (0)

extern "C" {

const char *ugks_version(void) { return "ugks_b200 0.2 (sm_100a)"; }

int ugks_abi_sizes(int64_t *out, int n) {
  const int64_t v[7] = {(int64_t)sizeof(ugks_block_desc), (int64_t)sizeof(ugks_fused_block),
                        (int64_t)sizeof(ugks_solve_state), (int64_t)offsetof(ugks_fused_block, f),
                        (int64_t)offsetof(ugks_solve_state, residual),
                        (int64_t)offsetof(ugks_block_desc, wall_D), (int64_t)sizeof(ugks_fused_sizes)};
  for (int i = 0; i < n && i < 7; ++i) out[i] = v[i];
  return 7;
}

int ugks_iFace(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin, double *iface_f,
               double *fsigma, const double *centre, const double *mid_side, const double *normal,
               int face, void *stream) {
  VEL_LAUNCH(k_iFace, Fin, iface_f, fsigma, centre, mid_side, normal, face);
}
int ugks_getFaceCons(const ugks_block_desc *d, size_t g0, size_t g1, const double *iface_f,
                     const double *normal, int face, double *primary, int off_bot, int off_top,
                     void *stream) {
  VEL_LAUNCH(k_face_moments, iface_f, normal, face, primary, off_bot, off_top, 0);
}
int ugks_getAL(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin,
               const double *normal, int face, double *gaL, int off_bot, int off_top,
               void *stream) {
  VEL_LAUNCH(k_face_moments, Fin, normal, face, gaL, off_bot, off_top, 1);
}
int ugks_getAR(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin,
               const double *normal, int face, double *gaR, int off_bot, int off_top,
               void *stream) {
  VEL_LAUNCH(k_face_moments, Fin, normal, face, gaR, off_bot, off_top, 2);
}
int ugks_getPLR(const ugks_block_desc *d, size_t g0, size_t g1, const double *centre,
                const double *mid_side, int face, double *primary, double *gaL, double *gaR,
                int off_bot, int off_top, void *stream) {
  PT_LAUNCH(k_getPLR, g0 * g1, g0, g1, centre, mid_side, face, primary, gaL, gaR, off_bot, off_top);
}
int ugks_initMacroFlux(const ugks_block_desc *d, size_t g0, size_t g1, double *flux_macro,
                       int face, double dt, const double *primary, const double *gaL,
                       const double *gaR, double *gaT, double *gMxi, int off_bot, int off_top,
                       void *stream) {
  PT_LAUNCH(k_initMacroFlux, g0 * g1, g0, g1, flux_macro, face, dt, primary, gaL, gaR, gaT, gMxi,
            off_bot, off_top);
}
int ugks_calcFaceQ(const ugks_block_desc *d, size_t g0, size_t g1, const double *iface_f,
                   const double *primary, const double *normal, double *faceQ, int face,
                   int off_bot, int off_top, void *stream) {
  VEL_LAUNCH(k_calcFaceQ, iface_f, primary, normal, faceQ, face, off_bot, off_top);
}
int ugks_macroFlux(const ugks_block_desc *d, size_t g0, size_t g1, const double *flux_f,
                   const double *fsigma, double *flux_macro, const double *normal,
                   const double *side_length, int face, double dt, const double *primary,
                   const double *faceQ, int off_bot, int off_top, void *stream) {
  VEL_LAUNCH(k_macroFlux, flux_f, fsigma, flux_macro, normal, side_length, face, dt, primary, faceQ,
             off_bot, off_top);
}
int ugks_distFlux(const ugks_block_desc *d, size_t g0, size_t g1, double *flux_f,
                  const double *fsigma, const double *normal, const double *side_length, int face,
                  double dt, const double *primary, const double *gaL, const double *gaR,
                  const double *gaT, const double *gMxi, const double *faceQ, int off_bot,
                  int off_top, void *stream) {
  VEL_LAUNCH(k_distFlux, flux_f, fsigma, normal, side_length, face, dt, primary, gaL, gaR, gaT, gMxi,
             faceQ, off_bot, off_top);
}
int ugks_accommodatingWallDist(const ugks_block_desc *d, size_t g0, size_t g1,
                               const double *normal, int face, const double *wall_prop,
                               double *flux_f, double dt, void *stream) {
  (void)dt;
  VEL_LAUNCH(k_accommodatingWallDist, normal, face, wall_prop, flux_f);
}
int ugks_wallFlux(const ugks_block_desc *d, size_t g0, size_t g1, const double *normal,
                  const double *side_length, int face, double *flux_f, double *flux_macro,
                  double dt, void *stream) {
  VEL_LAUNCH(k_wallFlux, normal, side_length, face, flux_f, flux_macro, dt);
}
int ugks_wallMassEnergyFluxes(const ugks_block_desc *d, size_t g0, size_t g1,
                              const double *normal, const double *side_length, const double *area,
                              int face, const double *flux_f, double *wall_flux, double dt,
                              void *stream) {
  (void)side_length; (void)area; (void)dt;
  VEL_LAUNCH(k_wallMassEnergyFluxes, normal, face, flux_f, wall_flux);
}
int ugks_updateMacro(const ugks_block_desc *d, size_t g0, size_t g1, const double *fmS,
                     const double *fmW, const double *area, double *macro, double *residual,
                     void *stream) {
  PT_LAUNCH(k_updateMacro, g0 * g1, g0, g1, fmS, fmW, area, macro, residual);
}
int ugks_UGKS_update(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin,
                     const double *fS, const double *fW, const double *area, const double *macro,
                     const double *gQ, const double *residual, double dt, double *flag,
                     void *stream) {
  VEL_LAUNCH(k_UGKS_update, Fin, fS, fW, area, macro, gQ, residual, dt, flag);
}
int ugks_getResidual(const ugks_block_desc *d, size_t g0, size_t g1, const double *macro,
                     double *residual, void *stream) {
  PT_LAUNCH(k_getResidual, g0 * g1, g0, g1, macro, residual);
}
int ugks_edgeMassFlow(const ugks_block_desc *d, size_t g0, size_t g1, const double *macro,
                      const double *normal, const double *side_length, double *mdot,
                      int this_face, void *stream) {
  (void)g1;
  PT_LAUNCH(k_edgeMassFlow, g0, g0, macro, normal, side_length, mdot, this_face);
}
int ugks_calcQ(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin,
               const double *macro, double *gQ, void *stream) {
  VEL_LAUNCH(k_calcQ, Fin, macro, gQ);
}
int ugks_calcMacro(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin,
                   double *macro, void *stream) {
  VEL_LAUNCH(k_calcMacro, Fin, macro);
}
int ugks_initFunctions(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin,
                       const double *macro, const double *gQ, void *stream) {
  VEL_LAUNCH(k_initFunctions, Fin, macro, gQ);
}
int ugks_clFindDT(const ugks_block_desc *d, size_t g0, size_t g1, const double *xy,
                  const double *area, const double *macro, double *time_step, double Kn,
                  void *stream) {
  PT_LAUNCH(k_clFindDT, g0 * g1, g0, g1, xy, area, macro, time_step, Kn);
}
int ugks_array_max(const double *x, size_t n, double *out, void *stream) {
  if (n == 0) return 0;
  k_array_max<<<1, 1024, 0, S(stream)>>>(x, n, out);
  return launch_status();
}
int ugks_paraBC(const ugks_block_desc *d, size_t g0, size_t g1, const double *para_def,
                double *wall_prop, double t, void *stream) {
  (void)g1; (void)para_def; (void)t;
  PT_LAUNCH(k_paraBC, g0, g0, wall_prop);
}
int ugks_edgeExchange(const ugks_block_desc *d, size_t g0, size_t g1, double *fA,
                      const double *xyA, int this_face, const double *fB, const double *xyB,
                      int NIB, int NJB, int that_face, int ori, int flip, void *stream) {
  VEL_LAUNCH(k_edgeExchange, fA, xyA, this_face, fB, xyB, NIB, NJB, that_face, ori, flip);
}
int ugks_edgeExtrapolate(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin,
                         int this_face, void *stream) {
  VEL_LAUNCH(k_edgeExtrapolate, Fin, this_face);
}
int ugks_edgeConstant(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin, int this_face,
                      const double *wall_prop, void *stream) {
  VEL_LAUNCH(k_edgeConstant, Fin, this_face, wall_prop);
}
int ugks_edgeInflow(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin, int this_face,
                    const double *normal, const double *macro, const double *gQ,
                    const double *wall_prop, void *stream) {
  VEL_LAUNCH(k_edgeInOut, Fin, this_face, normal, macro, gQ, wall_prop, 0);
}
int ugks_edgeOutflow(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin, int this_face,
                     const double *normal, const double *macro, const double *gQ,
                     const double *wall_prop, void *stream) {
  VEL_LAUNCH(k_edgeInOut, Fin, this_face, normal, macro, gQ, wall_prop, 1);
}
int ugks_edgeMirror(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin, int this_face,
                    void *stream) {
  VEL_LAUNCH(k_edgeMirror, Fin, this_face, 0);
}
int ugks_edgeBounceBack(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin,
                        int this_face, void *stream) {
  VEL_LAUNCH(k_edgeMirror, Fin, this_face, 1);
}
int ugks_edgeConstGrad(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin, int this_face,
                       void *stream) {
  VEL_LAUNCH(k_edgeConstGrad, Fin, this_face);
}
int ugks_adsorbingWall_P1(const ugks_block_desc *d, size_t g0, size_t g1, const double *normal,
                          int face, const double *wall_prop, double *wall_cover, double *wall_dist,
                          const double *flux_f, const double *macro, double dt, double *flag,
                          void *stream) {
  (void)wall_prop;
  VEL_LAUNCH(k_adsorbingWall_P1, normal, face, wall_cover, wall_dist, flux_f, macro, dt, flag);
}
int ugks_adsorbingWallD_P2(const ugks_block_desc *d, size_t g0, size_t g1, const double *normal,
                           int face, const double *wall_prop, const double *wall_cover,
                           const double *wall_dist, double *flux_f, const double *macro,
                           double dt, void *stream) {
  (void)wall_dist; (void)macro; (void)dt;
  VEL_LAUNCH(k_adsorbingWallD_P2, normal, face, wall_prop, wall_cover, flux_f);
}
int ugks_getInternal(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin, double *Txyz,
                     double *Stress, void *stream) {
  VEL_LAUNCH(k_getInternal, Fin, Txyz, Stress);
}
int ugks_adsorbingWallS_P2(const ugks_block_desc *d, size_t g0, size_t g1, const double *normal,
                           int face, const double *wall_prop, const double *wall_cover,
                           const double *wall_dist, double *flux_f, const double *macro,
                           double dt, void *stream) {
  (void)macro; (void)dt;
  VEL_LAUNCH(k_adsorbingWallSCL_P2<UGKS_REFLECT_SPECULAR>, normal, face, wall_prop, wall_cover, wall_dist, flux_f);
}
int ugks_adsorbingWallCL_P2(const ugks_block_desc *d, size_t g0, size_t g1, const double *normal,
                            int face, const double *wall_prop, const double *wall_cover,
                            const double *wall_dist, double *flux_f, const double *macro,
                            double dt, void *stream) {
  (void)macro; (void)dt;
  VEL_LAUNCH(k_adsorbingWallSCL_P2<UGKS_REFLECT_CL>, normal, face, wall_prop, wall_cover, wall_dist, flux_f);
}

}  // extern "C"
