// ugks_device.cuh -- device physics of the UGKS time step (FP64 arithmetic).
//
// Each helper restates one function of the pyUGKS OpenCL sources
// (file:line at each definition).  The header constants the reference baked
// in with #define come from ugks_block_desc.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ugks_b200.h"

namespace ugks {

constexpr int SOUTH = 0, WEST = 1;
constexpr int GNORTH = 0, GEAST = 1, GSOUTH = 2, GWEST = 3;
constexpr int NO_FLIP = 0, FLIP_NS = 1, FLIP_D = 2, FLIP_EW = 3;
// boundary condition codes (geom/geom_bc_defs.py:27-37)
constexpr int BC_ADJACENT = 0, BC_EXTRAPOLATE_OUT = 1, BC_CONSTANT = 2, BC_REFLECT = 3,
              BC_DIFFUSE = 4, BC_PERIODIC = 5, BC_INFLOW = 6, BC_OUTFLOW = 7,
              BC_ADSORBING = 8, BC_BOUNCE_BACK = 9;
constexpr int MNUM = 7, MTUM = 5;

struct V2 { double x, y; };
// (rho, U, V, lambda) or conserved (rho, rho U, rho V, E)
struct P4 { double s0, s1, s2, s3; };

__device__ __forceinline__ V2 v2(double x, double y) { V2 r; r.x = x; r.y = y; return r; }
__device__ __forceinline__ P4 p4(double a, double b, double c, double e) {
  P4 r; r.s0 = a; r.s1 = b; r.s2 = c; r.s3 = e; return r;
}
__device__ __forceinline__ P4 add(P4 a, P4 b) {
  return p4(a.s0 + b.s0, a.s1 + b.s1, a.s2 + b.s2, a.s3 + b.s3);
}
__device__ __forceinline__ P4 scale(double s, P4 a) { return p4(s * a.s0, s * a.s1, s * a.s2, s * a.s3); }

__device__ __forceinline__ P4 ld4(const double *a, size_t k) {
  const double2 *p = reinterpret_cast<const double2 *>(a + 4 * k);
  double2 x = p[0], y = p[1];
  return p4(x.x, x.y, y.x, y.y);
}
__device__ __forceinline__ void st4(double *a, size_t k, P4 v) {
  double2 *p = reinterpret_cast<double2 *>(a + 4 * k);
  p[0] = make_double2(v.s0, v.s1);
  p[1] = make_double2(v.s2, v.s3);
}
__device__ __forceinline__ V2 ld2(const double *a, size_t k) {
  double2 x = reinterpret_cast<const double2 *>(a)[k];
  return v2(x.x, x.y);
}
__device__ __forceinline__ void st2(double *a, size_t k, V2 v) {
  reinterpret_cast<double2 *>(a)[k] = make_double2(v.x, v.y);
}

// index helpers for the reference layouts (clKernel.c:4-26)
__device__ __forceinline__ size_t fidx(const ugks_block_desc &d, long i, long j, long v) {
  return ((size_t)i * d.Nj + (size_t)j) * d.Nv + (size_t)v;
}
__device__ __forceinline__ size_t gidx(const ugks_block_desc &d, long i, long j) {
  return (size_t)i * d.Nj + (size_t)j;
}
__device__ __forceinline__ size_t faceidx(const ugks_block_desc &d, long i, long j, int f) {
  return ((size_t)i * d.Nj + (size_t)j) * 2 + f;
}
__device__ __forceinline__ size_t midx(const ugks_block_desc &d, long i, long j) {
  return (size_t)i * d.nj + (size_t)j;
}

// Reciprocal by Newton-Raphson: the hardware's approximate reciprocal
// (rcp.approx.ftz.f64, PTX ISA) refined by two iterations y <- y + y (1 - x y),
// each of which squares the relative error; for normal finite x != 0 the
// result is within 1 ulp of 1/x (checked against 1/x by the GPU tests).
__device__ __forceinline__ double nr_rcp(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// OpenCL sign(): +-1, keeps signed zero, 0 for NaN
__device__ __forceinline__ double ocl_sign(double a) {
  return a > 0.0 ? 1.0 : (a < 0.0 ? -1.0 : (a == 0.0 ? a : 0.0));
}
// upwind flag (sign(u)*rot + 1)/2 truncated to int: 1 for u*rot > 0 else 0
__device__ __forceinline__ int upwind_flag(double u, int rot) {
  return (int)((ocl_sign(u) * rot + 1) / 2);
}

// relaxTime (clFunctions.c:8-32)
__device__ __forceinline__ double relax_time(const ugks_block_desc &d, P4 prim) {
  double p = pow(prim.s3, 1.0 - d.omega);
  switch (d.relax_type) {
    case 0: return (d.Kn_eff / prim.s0) * 0.79788456080286541 * p;
    case 1: return (5. / 8.) * (d.Kn_eff / prim.s0) * sqrt(d.PI) * p;
    case 3: return (d.Kn_eff / prim.s0) * 2.2567583341910251 * p;
    default: return (d.Kn_eff / prim.s0) * p;
  }
}

// interfaceVelocity (clFunctions.c:191-209)
__device__ __forceinline__ V2 face_velocity(const ugks_block_desc &d, int v, V2 n) {
  double2 e = reinterpret_cast<const double2 *>(d.quad)[v];
  return v2(e.x * n.x + e.y * n.y, e.x * (-n.y) + e.y * n.x);
}
__device__ __forceinline__ V2 quad_at(const ugks_block_desc &d, int v) {
  double2 e = reinterpret_cast<const double2 *>(d.quad)[v];
  return v2(e.x, e.y);
}
// toGlobal / toLocal (clFunctions.c:215-250)
__device__ __forceinline__ V2 to_global(V2 in, V2 n) {
  return v2(n.x * in.x + (-n.y) * in.y, n.y * in.x + n.x * in.y);
}
__device__ __forceinline__ V2 to_local(V2 in, V2 n) {
  return v2(in.x * n.x + in.y * n.y, in.x * (-n.y) + in.y * n.x);
}

// fM (clFunctions.c:49-58): weighted Maxwellian (h, b)
__device__ __forceinline__ V2 maxwellian(const ugks_block_desc &d, P4 prim, V2 uv, int v) {
  double cx = uv.x - prim.s1, cy = uv.y - prim.s2;
  double h = prim.s0 * (prim.s3 / d.PI) * exp(-prim.s3 * (cx * cx + cy * cy));
  double b = (h * d.K) / (2.0 * prim.s3);
  double w = d.weight[v];
  return v2(w * h, w * b);
}
// fS (clFunctions.c:64-77)
__device__ __forceinline__ V2 shakhov(const ugks_block_desc &d, P4 prim, V2 Q, V2 uv, V2 M) {
  double cx = uv.x - prim.s1, cy = uv.y - prim.s2;
  double s = 0.8 * (1 - d.Pr) * (prim.s3 * prim.s3) / prim.s0 * (cx * Q.x + cy * Q.y);
  double part = 2 * prim.s3 * (cx * cx + cy * cy);
  return v2((s * (part - 4)) * M.x, (s * (part - 2)) * M.y);
}
// fEQ (clFunctions.c:79-86)
__device__ __forceinline__ V2 shakhov_eq(const ugks_block_desc &d, P4 prim, V2 Q, V2 uv, int v) {
  V2 M = maxwellian(d, prim, uv, v);
  V2 S = shakhov(d, prim, Q, uv, M);
  return v2(M.x + S.x, M.y + S.y);
}

// clFindDT (clKernel.c:224-308): the CFL frequency (dx u + dy v) / A of
// interior cell (mi, mj) with macro state m (rho, U, V, lambda); Kn is the
// host's unrounded Kn that ugks_block.py:1421 passes.  The drop-in kernel,
// the fused cell and set-up passes and the allocation-free query all call it.
__device__ __forceinline__ double cfl_frequency(const ugks_block_desc &d, const double *xy,
                                                const double *area, P4 m, long mi, long mj,
                                                double Kn) {
  const long G = d.ghost, NY = d.Nj + 1;
  const V2 a = ld2(xy, (mi + 1 + G) * NY + mj + G), b = ld2(xy, (mi + 1 + G) * NY + mj + 1 + G);
  const V2 c = ld2(xy, (mi + G) * NY + mj + 1 + G), e = ld2(xy, (mi + G) * NY + mj + G);
  const double dx = fmax(fmax(fmax(fabs(a.x - b.x), fabs(c.x - b.x)), fmax(fabs(c.x - e.x), fabs(a.x - e.x))),
                         fmax(fabs(c.x - a.x), fabs(b.x - e.x)));
  const double dy = fmax(fmax(fmax(fabs(a.y - b.y), fabs(c.y - b.y)), fmax(fabs(c.y - e.y), fabs(a.y - e.y))),
                         fmax(fabs(c.y - a.y), fabs(b.y - e.y)));
  const double sos = sqrt(0.5 * d.gam / m.s3);
  const double lo_u = fmin(d.umax, fabs(m.s1) + sos), lo_v = fmin(d.vmax, fabs(m.s2) + sos);
  const double hi_u = fmax(d.umax, fabs(m.s1) + sos), hi_v = fmax(d.vmax, fabs(m.s2) + sos);
  const double sc = (erf(10 * (Kn - 1e-3)) + 1) / 2.0;
  const double u = sc * (hi_u - lo_u) + lo_u, v = sc * (hi_v - lo_v) + lo_v;
  return (dx * u + dy * v) / area[gidx(d, mi + G, mj + G)];
}

// getPrimary / getConserved / microSlope (clUGKS.c:16-45)
__device__ __forceinline__ P4 to_primary(const ugks_block_desc &d, P4 w) {
  P4 p = w;
  p.s3 = 0.5 * w.s0 / (d.gam - 1.0) / (w.s3 - 0.5 * (w.s1 * w.s1 + w.s2 * w.s2) / w.s0);
  p.s1 = w.s1 / w.s0;
  p.s2 = w.s2 / w.s0;
  return p;
}
__device__ __forceinline__ P4 to_conserved(const ugks_block_desc &d, P4 p) {
  P4 w = p;
  w.s3 = 0.5 * p.s0 / p.s3 / (d.gam - 1.0) + 0.5 * p.s0 * (p.s1 * p.s1 + p.s2 * p.s2);
  w.s1 = p.s1 * p.s0;
  w.s2 = p.s2 * p.s0;
  return w;
}
__device__ __forceinline__ P4 micro_slope(const ugks_block_desc &d, P4 prim, P4 sw) {
  const double K = d.K;
  P4 a;
  a.s3 = 4.0 * (prim.s3 * prim.s3) / (K + 2) / prim.s0 *
         (2.0 * sw.s3 - 2.0 * prim.s1 * sw.s1 - 2.0 * prim.s2 * sw.s2 +
          sw.s0 * ((prim.s1 * prim.s1 + prim.s2 * prim.s2) - 0.5 * (K + 2) / prim.s3));
  a.s2 = 2.0 * prim.s3 / prim.s0 * (sw.s2 - prim.s2 * sw.s0) - prim.s2 * a.s3;
  a.s1 = 2.0 * prim.s3 / prim.s0 * (sw.s1 - prim.s1 * sw.s0) - prim.s1 * a.s3;
  a.s0 = sw.s0 / prim.s0 - prim.s1 * a.s1 - prim.s2 * a.s2 -
         0.5 * ((prim.s1 * prim.s1) + (prim.s2 * prim.s2) + 0.5 * (K + 2) / prim.s3) * a.s3;
  return a;
}

// momentU (clUGKS.c:47-80)
__device__ inline void moments_u(const ugks_block_desc &d, P4 prim, double Mu[MNUM],
                                 double Mv[MTUM], double Mxi[3], double MuL[MNUM],
                                 double MuR[MNUM]) {
  double sl = sqrt(prim.s3);
  double g = 0.5 * exp(-prim.s3 * (prim.s1 * prim.s1)) / sqrt(d.PI * prim.s3);
  MuL[0] = 0.5 * erfc(-sl * prim.s1);
  MuL[1] = prim.s1 * MuL[0] + g;
  MuR[0] = 0.5 * erfc(sl * prim.s1);
  MuR[1] = prim.s1 * MuR[0] - g;
#pragma unroll
  for (int i = 2; i < MNUM; ++i) {
    MuL[i] = prim.s1 * MuL[i - 1] + 0.5 * (i - 1) * MuL[i - 2] / prim.s3;
    MuR[i] = prim.s1 * MuR[i - 1] + 0.5 * (i - 1) * MuR[i - 2] / prim.s3;
  }
#pragma unroll
  for (int i = 0; i < MNUM; ++i) Mu[i] = MuL[i] + MuR[i];
  Mv[0] = 1.0;
  Mv[1] = prim.s2;
#pragma unroll
  for (int i = 2; i < MTUM; ++i) Mv[i] = prim.s2 * Mv[i - 1] + 0.5 * (i - 1) * Mv[i - 2] / prim.s3;
  Mxi[0] = 1.0;
  Mxi[1] = 0.5 * d.K / prim.s3;
  Mxi[2] = (d.K * d.K + 2.0 * d.K) / (4.0 * prim.s3 * prim.s3);
}
// moment_uv (clUGKS.c:82-93)
__device__ __forceinline__ P4 moment_uv(const double *Mu, const double *Mv, const double *Mxi,
                                        int a, int b, int dd) {
  return p4(Mu[a] * Mv[b] * Mxi[dd / 2], Mu[a + 1] * Mv[b] * Mxi[dd / 2],
            Mu[a] * Mv[b + 1] * Mxi[dd / 2],
            0.5 * (Mu[a + 2] * Mv[b] * Mxi[dd / 2] + Mu[a] * Mv[b + 2] * Mxi[dd / 2] +
                   Mu[a] * Mv[b] * Mxi[(dd + 2) / 2]));
}
// moment_au (clUGKS.c:95-104)
__device__ __forceinline__ P4 moment_au(P4 a, const double *Mu, const double *Mv,
                                        const double *Mxi, int al, int be) {
  P4 r = scale(a.s0, moment_uv(Mu, Mv, Mxi, al + 0, be + 0, 0));
  r = add(r, scale(a.s1, moment_uv(Mu, Mv, Mxi, al + 1, be + 0, 0)));
  r = add(r, scale(a.s2, moment_uv(Mu, Mv, Mxi, al + 0, be + 1, 0)));
  r = add(r, scale(0.5 * a.s3, moment_uv(Mu, Mv, Mxi, al + 2, be + 0, 0)));
  r = add(r, scale(0.5 * a.s3, moment_uv(Mu, Mv, Mxi, al + 0, be + 2, 0)));
  r = add(r, scale(0.5 * a.s3, moment_uv(Mu, Mv, Mxi, al + 0, be + 0, 2)));
  return r;
}
// time-integration weights (clUGKS.c:497-503)
__device__ __forceinline__ void time_weights(double tau, double dt, double Mt[5]) {
  double e = exp(-dt / tau);
  Mt[3] = tau * (1.0 - e);
  Mt[4] = -tau * dt * e + tau * Mt[3];
  Mt[0] = dt - Mt[3];
  Mt[1] = -tau * Mt[0] + Mt[4];
  Mt[2] = (dt * dt) / 2.0 - tau * Mt[0];
}

// limiters (clFunctions.c:255-353)
__device__ __forceinline__ double vanleer(double s1, double s2) {
  return (ocl_sign(s1) + ocl_sign(s2)) * (fabs(s1) * fabs(s2)) / (fabs(s1) + fabs(s2) + 1e-16);
}
__device__ __forceinline__ double weno5(double S0, double S1, double S2, double S3, double S4,
                                        double dx) {
  const double eps = 1E-16;
  double t1, t2;
  t1 = S0 - 2.0 * S1 + S2;
  t2 = S0 - 4.0 * S1 + 3.0 * S2;
  double B0 = (13.0 / 12.0) * t1 * t1 + 0.25 * t2 * t2;
  t1 = S1 - 2.0 * S2 + S3;
  t2 = S1 - S3;
  double B1 = (13.0 / 12.0) * t1 * t1 + 0.25 * t2 * t2;
  t1 = S2 - 2.0 * S3 + S4;
  t2 = 3.0 * S2 - 4.0 * S3 + S4;
  double B2 = (13.0 / 12.0) * t1 * t1 + 0.25 * t2 * t2;
  t1 = eps + B0; double a0 = 0.1 / (t1 * t1);
  t1 = eps + B1; double a1 = 0.6 / (t1 * t1);
  t1 = eps + B2; double a2 = 0.3 / (t1 * t1);
  double s = a0 + a1 + a2;
  double f0 = (1. / 3.) * S0 - (7. / 6.) * S1 + (11. / 6.) * S2;
  double f1 = -(1. / 6.) * S1 + (5. / 6.) * S2 + (1. / 3.) * S3;
  double f2 = (1. / 3.) * S2 + (5. / 6.) * S3 - (1. / 6.) * S4;
  double fL = (a0 / s) * f0 + (a1 / s) * f1 + (a2 / s) * f2;
  return (fL - S2) / dx;
}
__device__ __forceinline__ double minmod(double a, double b) {
  double out = 0.0;
  if ((fabs(a) < fabs(b)) && (a * b > 0)) out = a;
  else if ((fabs(b) < fabs(a)) && (a * b > 0)) out = b;
  else if (a == b) out = a;
  return out;
}

// stickingProbability (clAdsorb.c:6-16)
__device__ __forceinline__ double sticking(const ugks_block_desc &d, V2 uv, double T, int face) {
  double nrm = 1.0 - d.beta_n[face] * exp(-uv.x * uv.x / T);
  double tan_ = 1.0 - d.beta_t[face] * (1.0 - exp(-uv.y * uv.y / T));
  return nrm * tan_;
}

// distance_from_segment, intersect, get_tri, interpolate, vartheta_langmuir
// (clAdsorb.c:18-247): equilibrium coverage at (P = rho T / 2, T) from a
// tabulated isotherm by a walk through its Delaunay triangulation, starting at
// triangle 0; intersect works in single precision as the reference does.
// Returns (theta, 1 when the point lies outside the table).
__device__ __forceinline__ double iso_segment_distance(V2 a, V2 b, V2 c) {
  const double r_num = (c.x - a.x) * (b.x - a.x) + (c.y - a.y) * (b.y - a.y);
  const double r_den = (b.x - a.x) * (b.x - a.x) + (b.y - a.y) * (b.y - a.y);
  const double r = r_num / r_den;
  const double s = ((a.y - c.y) * (b.x - a.x) - (a.x - c.x) * (b.y - a.y)) / r_den;
  const double line = fabs(s) * sqrt(r_den);
  if ((r >= 0) && (r <= 1)) return line;
  const double d1 = (c.x - a.x) * (c.x - a.x) + (c.y - a.y) * (c.y - a.y);
  const double d2 = (c.x - b.x) * (c.x - b.x) + (c.y - b.y) * (c.y - b.y);
  return d1 < d2 ? sqrt(d1) : sqrt(d2);
}
__device__ __forceinline__ int iso_intersect(V2 a, V2 b, V2 c, V2 d) {
  const float den = (float)((d.y - c.y) * (b.x - a.x) - (d.x - c.x) * (b.y - a.y));
  const float num1 = (float)((d.x - c.x) * (a.y - c.y) - (d.y - c.y) * (a.x - c.x));
  const float num2 = (float)((b.x - a.x) * (a.y - c.y) - (b.y - a.y) * (a.x - c.x));
  const float u1 = __fdiv_rn(num1, den), u2 = __fdiv_rn(num2, den);
  if (den == 0.0f) return 0;
  if (u1 < 0 || u1 > 1 || u2 < 0 || u2 > 1) return 0;
  return 1;
}
__device__ inline V2 vartheta_langmuir(const ugks_block_desc &d, double D, double T, int face) {
  if (d.constant_adsorb[face]) return v2(d.adsorb[face], 0.0);
  const double *iso = d.iso[face];
  const int32_t *tri = d.tri[face], *nbr = d.nbr[face];
  const V2 xy = v2(0.5 * D * T, T);
  auto pt = [&](int k) { return v2(iso[4 * k], iso[4 * k + 1]); };
  int id = 0, outside = 0;
  for (int counter = 0; counter < d.n_tri[face]; ++counter) {
    const int32_t *t = tri + 4 * id;
    const V2 a = pt(t[0]), b = pt(t[1]), c = pt(t[2]);
    const V2 start = v2((1.0 / 3.0) * (a.x + b.x + c.x), (1.0 / 3.0) * (a.y + b.y + c.y));
    const int hz = iso_intersect(a, b, start, xy), hx = iso_intersect(b, c, start, xy),
              hy = iso_intersect(c, a, start, xy);
    if ((hx + hy + hz) == 0) break;
    const int32_t *nb = nbr + 4 * id;
    if (hx) {
      if (nb[0] == -1) { outside = 1; break; }
      if (iso_segment_distance(b, c, xy) < 1e-12) break;
      id = nb[0];
    } else if (hy) {
      if (nb[1] == -1) { outside = 1; break; }
      if (iso_segment_distance(c, a, xy) < 1e-12) break;
      id = nb[1];
    } else {
      if (nb[2] == -1) { outside = 1; break; }
      if (iso_segment_distance(a, b, xy) < 1e-12) break;
      id = nb[2];
    }
  }
  const int32_t *t = tri + 4 * id;
  const double *A = iso + 4 * t[0], *Bp = iso + 4 * t[1], *Cp = iso + 4 * t[2];
  const double den = (Bp[1] - Cp[1]) * (A[0] - Cp[0]) + (Cp[0] - Bp[0]) * (A[1] - Cp[1]);
  const double L1 = ((Bp[1] - Cp[1]) * (xy.x - Cp[0]) + (Cp[0] - Bp[0]) * (xy.y - Cp[1])) / den;
  const double L2 = ((Cp[1] - A[1]) * (xy.x - Cp[0]) + (A[0] - Cp[0]) * (xy.y - Cp[1])) / den;
  const double L3 = 1 - L1 - L2;
  return v2(L1 * A[2] + L2 * Bp[2] + L3 * Cp[2], (double)outside);
}

// Cercignani-Lampis scattering (scatterNormal, scatterTangential,
// CercignaniLampis: clFunctions.c:146-185), I0 from the CUDA math library
__device__ __forceinline__ double scatter_normal(double c_in, double c_out, double an, double Tw) {
  return (2.0 / (an * Tw)) * fabs(c_out) * cyl_bessel_i0(((2 * sqrt(1 - an)) / (an * Tw)) * c_in * c_out) *
         exp(-(c_out * c_out + (1 - an) * c_in * c_in) / (an * Tw));
}
__device__ __forceinline__ double scatter_tangential(double PI, double c_in, double c_out, double at,
                                                     double Tw) {
  const double a = c_out - (1 - at) * c_in;
  return (1.0 / sqrt(PI * at * (2 - at) * Tw)) * exp(-(a * a) / (at * (2 - at) * Tw));
}
// contribution of incoming velocity uv_in (distribution f_in) to outgoing
// uv_out, with the (h, b) closure term added (clAdsorb.c:568-569)
__device__ __forceinline__ V2 cercignani_lampis(double PI, V2 uv_in, V2 uv_out, V2 f_in, double an, double at,
                                                double Tw, double lam_w) {
  const double k = fabs(uv_in.x / uv_out.x) * scatter_normal(uv_in.x, uv_out.x, an, Tw) *
                   scatter_tangential(PI, uv_in.y, uv_out.y, at, Tw);
  V2 r = v2(k * f_in.x, k * f_in.y);
  r.y *= (1 - at) * (1 - at);
  r.y += 0.5 * at * (2 - at) / lam_w * r.x;
  return r;
}

// ---------------------------------------------------------------------------
// block-wide sums: every thread passes N partial sums and receives the totals.
// `scratch` is shared memory of at least N * (blockDim.x / 32) doubles.
// ---------------------------------------------------------------------------
template <int N>
__device__ __forceinline__ void block_sum(double (&x)[N], double *scratch) {
#pragma unroll
  for (int k = 0; k < N; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x[k] += __shfl_xor_sync(0xffffffffu, x[k], o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();  // scratch may still be read by a previous call
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) scratch[k * nw + warp] = x[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += scratch[k * nw + w];
    x[k] = s;
  }
}

// Sums N <= 16 values over the 32 lanes of a warp by halving butterflies: at
// each exchange a lane keeps half of its values and adds the partner lane's
// copies of that half, so that P - 1 + (5 - log2 P) exchanges (P = N rounded
// up to a power of 2) replace the 5 N of one butterfly per value.  On return
// the 2^S lanes from k << S on (S = spread_shift<N>()) hold the total of
// value k.
template <int N>
__device__ __forceinline__ constexpr int spread_width() {
  return N <= 1 ? 1 : (N <= 2 ? 2 : (N <= 4 ? 4 : (N <= 8 ? 8 : 16)));
}
template <int N>
__device__ __forceinline__ constexpr int spread_shift() {
  return N <= 1 ? 5 : (N <= 2 ? 4 : (N <= 4 ? 3 : (N <= 8 ? 2 : 1)));
}
template <int C, int O, int P>
__device__ __forceinline__ void spread_step(double (&v)[P], unsigned lane) {
  if constexpr (O >= 1) {
    if constexpr (C > 1) {
      constexpr int H = C / 2;
      const bool hi = (lane & O) != 0;
#pragma unroll
      for (int k = 0; k < H; ++k) {
        const double keep = hi ? v[k + H] : v[k], send = hi ? v[k] : v[k + H];
        v[k] = keep + __shfl_xor_sync(0xffffffffu, send, O);
      }
      spread_step<H, O / 2, P>(v, lane);
    } else {
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], O);
      spread_step<1, O / 2, P>(v, lane);
    }
  }
}
template <int N>
__device__ __forceinline__ double warp_spread_sum(const double (&x)[N]) {
  static_assert(N >= 1 && N <= 16, "at most 16 values");
  constexpr int P = spread_width<N>();
  double v[P];
#pragma unroll
  for (int k = 0; k < P; ++k) v[k] = k < N ? x[k] : 0.0;
  spread_step<P, 16, P>(v, threadIdx.x & 31);
  return v[0];
}

// block_sum with halving butterflies inside each warp: the same totals in
// another order of summation, in 2 (P - 1) + 2 (5 - log2 P) shuffles per warp
// instead of 10 N
template <int N>
__device__ __forceinline__ void block_sum_spread(double (&x)[N], double *scratch) {
  const double t = warp_spread_sum<N>(x);
  constexpr int S = spread_shift<N>();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();  // scratch may still be read by a previous call
  if ((lane & ((1 << S) - 1)) == 0 && (lane >> S) < N) scratch[(lane >> S) * nw + warp] = t;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += scratch[k * nw + w];
    x[k] = s;
  }
}
// the same, with the totals only on thread 0
template <int N>
__device__ __forceinline__ void block_sum_spread_to0(double (&x)[N], double *scratch) {
  const double t = warp_spread_sum<N>(x);
  constexpr int S = spread_shift<N>();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if ((lane & ((1 << S) - 1)) == 0 && (lane >> S) < N) scratch[(lane >> S) * nw + warp] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += scratch[k * nw + w];
      x[k] = s;
    }
  }
}

// ---------------------------------------------------------------------------
// bulk asynchronous copies (the TMA engine, sm_90+): rows of global memory
// into shared memory, completed on an mbarrier; waits are polled with a bound
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// the barrier initialisations visible to the bulk-copy engine
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// order this thread's generic shared-memory accesses before later bulk copies
// into the same memory
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// bytes (a multiple of 16; both addresses 16-byte aligned) from global src to
// shared dst, completing `bytes` of the barrier's transaction count
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// true once the barrier's phase of the given parity has completed; false
// after `limit` waits.  UGKS_MBAR_TRY_WAIT: each wait is a try_wait that
// suspends the thread for at most about a microsecond; else a test_wait poll
// followed by a 32 ns sleep.
#ifndef UGKS_MBAR_TRY_WAIT
#define UGKS_MBAR_TRY_WAIT 1
#endif
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
#if UGKS_MBAR_TRY_WAIT
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(1000u)
        : "memory");
    if (done) return true;
#else
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    __nanosleep(32);
#endif
  }
  return false;
}

// (h, b) pairs stored as double2 or float2
template <typename T> struct Store;
template <> struct Store<double> {
  using vec = double2;
  __device__ __forceinline__ static V2 load(const void *base, size_t k) {
    double2 x = reinterpret_cast<const double2 *>(base)[k];
    return v2(x.x, x.y);
  }
  __device__ __forceinline__ static void store(void *base, size_t k, V2 v) {
    reinterpret_cast<double2 *>(base)[k] = make_double2(v.x, v.y);
  }
  // the value a store followed by a load gives back
  __device__ __forceinline__ static V2 as_stored(V2 v) { return v; }
};
template <> struct Store<float> {
  using vec = float2;
  __device__ __forceinline__ static V2 load(const void *base, size_t k) {
    float2 x = reinterpret_cast<const float2 *>(base)[k];
    return v2((double)x.x, (double)x.y);
  }
  __device__ __forceinline__ static void store(void *base, size_t k, V2 v) {
    reinterpret_cast<float2 *>(base)[k] = make_float2((float)v.x, (float)v.y);
  }
  __device__ __forceinline__ static V2 as_stored(V2 v) {
    return v2((double)(float)v.x, (double)(float)v.y);
  }
};

__device__ __forceinline__ void rot90(int &i, int &j, int n, int Ni, int Nj) {
  for (int a = 0; a < n; a++) {
    int t = i;
    i = Nj - j - 1;
    j = t;
    t = Ni; Ni = Nj; Nj = t;
  }
}

// getSwapIndex for cell indices (clGhostRoutines.c:47-138 with v == 0);
// also used by the fused ghost kernel
__device__ __forceinline__ void swap_cell_index(int NI, int NJ, int G, int this_face, int &iB, int &jB,
                                     int that_face, int NIB, int NJB) {
  switch (this_face) {
    case GEAST:
      if (that_face == GEAST) { iB = (NI - 1) - iB; iB += NIB - 2 * G; }
      else if (that_face == GWEST) { iB -= NI - 2 * G; }
      else if (that_face == GNORTH) { rot90(iB, jB, 3, NI, NJ); jB += NJB - 2 * G; }
      else { rot90(iB, jB, 1, NI, NJ); jB -= NI - 2 * G; }
      break;
    case GWEST:
      if (that_face == GWEST) { iB = (NI - 1) - iB; iB -= NI - 2 * G; }
      else if (that_face == GEAST) { iB += NIB - 2 * G; }
      else if (that_face == GNORTH) { rot90(iB, jB, 1, NI, NJ); jB += NJB - 2 * G; }
      else { rot90(iB, jB, 3, NI, NJ); jB -= NI - 2 * G; }
      break;
    case GNORTH:
      if (that_face == GNORTH) { jB = (NJ - 1) - jB; jB += NJB - 2 * G; }
      else if (that_face == GSOUTH) { jB -= NJ - 2 * G; }
      else if (that_face == GEAST) { rot90(iB, jB, 1, NI, NJ); iB += NIB - 2 * G; }
      else { rot90(iB, jB, 3, NI, NJ); iB -= NJ - 2 * G; }
      break;
    default:
      if (that_face == GSOUTH) { jB = (NJ - 1) - jB; jB -= NJ - 2 * G; }
      else if (that_face == GNORTH) { jB += NJB - 2 * G; }
      else if (that_face == GEAST) { rot90(iB, jB, 3, NI, NJ); iB += NIB - 2 * G; }
      else { rot90(iB, jB, 1, NI, NJ); iB -= NJ - 2 * G; }
      break;
  }
}


}  // namespace ugks
