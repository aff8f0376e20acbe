/* ugks_port.c -- TEST INFRASTRUCTURE ONLY (oracle; never linked into the product).
 *
 * Sequential C restatement of the pyUGKS OpenCL kernels on the UGKS time-step
 * path.  Every port_<name> walks the reference NDRange (g0 x g1 work-groups,
 * one work-item each, so every __local reduction of the reference is the plain
 * sequential sum over velocity written here) and takes the reference kernel's
 * arguments in the reference order, after the parameter struct and the range.
 * Built with -ffp-contract=off so that no multiply-add is fused.
 */
#include "ugks_port.h"

#include <math.h>
#include <string.h>

typedef struct { double x, y; } d2;
typedef struct { double s0, s1, s2, s3; } d4;

#define PP const ugks_port_params *P
/* f-like arrays: [(i*Nj + j)*Nv + v] pairs (clKernel.c:4) */
#define FIDX(i, j, v) ((((size_t)(i)) * P->Nj + (size_t)(j)) * P->Nv + (size_t)(v))
/* ghosted per-cell arrays: [i*Nj + j] (clKernel.c:17-18) */
#define GIDX(i, j) (((size_t)(i)) * P->Nj + (size_t)(j))
/* per-face geometry: [(i*Nj + j)*2 + face] (clKernel.c:19-21) */
#define FACEIDX(i, j, f) ((((size_t)(i)) * P->Nj + (size_t)(j)) * 2 + (size_t)(f))
/* interior per-cell arrays: [i*nj + j] (clKernel.c:10-14) */
#define MIDX(i, j) (((size_t)(i)) * P->nj + (size_t)(j))

enum { SOUTH = 0, WEST = 1 };
enum { GNORTH = 0, GEAST = 1, GSOUTH = 2, GWEST = 3 };
enum { NO_FLIP = 0, FLIP_NS = 1, FLIP_D = 2, FLIP_EW = 3 };
#define ERR_NAN 1.0
#define ERR_CLAMPING_ADSORB_ISOTHERM 4.0

static inline d2 ld2(const double *a, size_t k) { d2 r = {a[2 * k], a[2 * k + 1]}; return r; }
static inline void st2(double *a, size_t k, d2 v) { a[2 * k] = v.x; a[2 * k + 1] = v.y; }
static inline d4 ld4(const double *a, size_t k) {
  d4 r = {a[4 * k], a[4 * k + 1], a[4 * k + 2], a[4 * k + 3]};
  return r;
}
static inline void st4(double *a, size_t k, d4 v) {
  a[4 * k] = v.s0; a[4 * k + 1] = v.s1; a[4 * k + 2] = v.s2; a[4 * k + 3] = v.s3;
}
static inline d4 zero4(void) { d4 r = {0.0, 0.0, 0.0, 0.0}; return r; }

/* OpenCL sign(): +-1, signed zero kept, 0 for NaN */
static inline double ocl_sign(double a) {
  if (a > 0.0) return 1.0;
  if (a < 0.0) return -1.0;
  if (a == 0.0) return a;
  return 0.0;
}

/* relaxTime (clFunctions.c:8-32): prim = (rho, U, V, lambda) */
static double relax_time(PP, d4 prim) {
  double p = pow(prim.s3, 1.0 - P->omega);
  switch (P->relax_type) {
    case 0: return (P->Kn_eff / prim.s0) * 0.79788456080286541 * p;
    case 1: return (5. / 8.) * (P->Kn_eff / prim.s0) * sqrt(P->PI) * p;
    case 3: return (P->Kn_eff / prim.s0) * 2.2567583341910251 * p;
    default: return (P->Kn_eff / prim.s0) * p;
  }
}

/* interfaceVelocity (clFunctions.c:191-209): global velocity v in the
   (normal, tangent) frame of a face with unit normal n, tangent (-n.y, n.x) */
static inline d2 face_velocity(PP, size_t v, d2 n) {
  double ex = P->quad[2 * v], ey = P->quad[2 * v + 1];
  d2 uv;
  uv.x = ex * n.x + ey * n.y;
  uv.y = ex * (-n.y) + ey * n.x;
  return uv;
}
static inline d2 quad_at(PP, size_t v) { d2 e = {P->quad[2 * v], P->quad[2 * v + 1]}; return e; }

/* toGlobal / toLocal (clFunctions.c:215-250) */
static inline d2 to_global(d2 in, d2 n) {
  double tx = -n.y, ty = n.x;
  d2 out;
  out.x = ((n.x * in.x) * 1.0 + (n.y * in.x) * 0.0) + ((tx * in.y) * 1.0 + (ty * in.y) * 0.0);
  out.y = ((n.x * in.x) * 0.0 + (n.y * in.x) * 1.0) + ((tx * in.y) * 0.0 + (ty * in.y) * 1.0);
  return out;
}
static inline d2 to_local(d2 in, d2 n) {
  d2 out;
  out.x = in.x * n.x + in.y * n.y;
  out.y = in.x * (-n.y) + in.y * n.x;
  return out;
}

/* fM (clFunctions.c:49-58): weighted Maxwellian (h, b) */
static inline d2 maxwellian(PP, d4 prim, d2 uv, size_t v) {
  double cx = uv.x - prim.s1, cy = uv.y - prim.s2;
  double h = prim.s0 * (prim.s3 / P->PI) * exp(-prim.s3 * (cx * cx + cy * cy));
  double b = (h * P->K) / (2.0 * prim.s3);
  d2 r = {P->weight[v] * h, P->weight[v] * b};
  return r;
}

/* fS (clFunctions.c:64-77): Shakhov correction for Maxwellian M */
static inline d2 shakhov(PP, d4 prim, d2 Q, d2 uv, d2 M) {
  double cx = uv.x - prim.s1, cy = uv.y - prim.s2;
  double s = 0.8 * (1 - P->Pr) * (prim.s3 * prim.s3) / prim.s0 * (cx * Q.x + cy * Q.y);
  double part = 2 * prim.s3 * (cx * cx + cy * cy);
  d2 r = {(s * (part - 4)) * M.x, (s * (part - 2)) * M.y};
  return r;
}

/* fEQ (clFunctions.c:79-86) */
static inline d2 shakhov_eq(PP, d4 prim, d2 Q, d2 uv, size_t v) {
  d2 M = maxwellian(P, prim, uv, v);
  d2 S = shakhov(P, prim, Q, uv, M);
  d2 r = {M.x + S.x, M.y + S.y};
  return r;
}

/* getPrimary / getConserved / microSlope (clUGKS.c:16-45) */
static d4 to_primary(PP, d4 w) {
  d4 p = w;
  p.s3 = 0.5 * w.s0 / (P->gam - 1.0) / (w.s3 - 0.5 * (w.s1 * w.s1 + w.s2 * w.s2) / w.s0);
  p.s1 = w.s1 / w.s0;
  p.s2 = w.s2 / w.s0;
  return p;
}
static d4 to_conserved(PP, d4 p) {
  d4 w = p;
  w.s3 = 0.5 * p.s0 / p.s3 / (P->gam - 1.0) + 0.5 * p.s0 * (p.s1 * p.s1 + p.s2 * p.s2);
  w.s1 = p.s1 * p.s0;
  w.s2 = p.s2 * p.s0;
  return w;
}
static d4 micro_slope(PP, d4 prim, d4 sw) {
  double K = P->K;
  d4 a;
  a.s3 = 4.0 * (prim.s3 * prim.s3) / (K + 2) / prim.s0 *
         (2.0 * sw.s3 - 2.0 * prim.s1 * sw.s1 - 2.0 * prim.s2 * sw.s2 +
          sw.s0 * ((prim.s1 * prim.s1 + prim.s2 * prim.s2) - 0.5 * (K + 2) / prim.s3));
  a.s2 = 2.0 * prim.s3 / prim.s0 * (sw.s2 - prim.s2 * sw.s0) - prim.s2 * a.s3;
  a.s1 = 2.0 * prim.s3 / prim.s0 * (sw.s1 - prim.s1 * sw.s0) - prim.s1 * a.s3;
  a.s0 = sw.s0 / prim.s0 - prim.s1 * a.s1 - prim.s2 * a.s2 -
         0.5 * ((prim.s1 * prim.s1) + (prim.s2 * prim.s2) + 0.5 * (K + 2) / prim.s3) * a.s3;
  return a;
}

/* momentU (clUGKS.c:47-80): half-range and full moments of the Maxwellian */
#define MNUM 7
#define MTUM 5
static void moments_u(PP, d4 prim, double Mu[MNUM], double Mv[MTUM], double Mxi[3],
                      double MuL[MNUM], double MuR[MNUM]) {
  MuL[0] = 0.5 * erfc(-sqrt(prim.s3) * prim.s1);
  MuL[1] = prim.s1 * MuL[0] + 0.5 * exp(-prim.s3 * (prim.s1 * prim.s1)) / sqrt(P->PI * prim.s3);
  MuR[0] = 0.5 * erfc(sqrt(prim.s3) * prim.s1);
  MuR[1] = prim.s1 * MuR[0] - 0.5 * exp(-prim.s3 * (prim.s1 * prim.s1)) / sqrt(P->PI * prim.s3);
  for (int i = 2; i < MNUM; ++i) {
    MuL[i] = prim.s1 * MuL[i - 1] + 0.5 * (i - 1) * MuL[i - 2] / prim.s3;
    MuR[i] = prim.s1 * MuR[i - 1] + 0.5 * (i - 1) * MuR[i - 2] / prim.s3;
  }
  for (int i = 0; i < MNUM; ++i) Mu[i] = MuL[i] + MuR[i];
  Mv[0] = 1.0;
  Mv[1] = prim.s2;
  for (int i = 2; i < MTUM; ++i) Mv[i] = prim.s2 * Mv[i - 1] + 0.5 * (i - 1) * Mv[i - 2] / prim.s3;
  Mxi[0] = 1.0;
  Mxi[1] = 0.5 * P->K / prim.s3;
  Mxi[2] = (P->K * P->K + 2.0 * P->K) / (4.0 * prim.s3 * prim.s3);
}

/* moment_uv (clUGKS.c:82-93): <u^a v^b xi^d psi> */
static d4 moment_uv(const double *Mu, const double *Mv, const double *Mxi, int a, int b, int d) {
  d4 m;
  m.s0 = Mu[a] * Mv[b] * Mxi[d / 2];
  m.s1 = Mu[a + 1] * Mv[b] * Mxi[d / 2];
  m.s2 = Mu[a] * Mv[b + 1] * Mxi[d / 2];
  m.s3 = 0.5 * (Mu[a + 2] * Mv[b] * Mxi[d / 2] + Mu[a] * Mv[b + 2] * Mxi[d / 2] +
                Mu[a] * Mv[b] * Mxi[(d + 2) / 2]);
  return m;
}
static inline d4 add4(d4 a, d4 b) { d4 r = {a.s0 + b.s0, a.s1 + b.s1, a.s2 + b.s2, a.s3 + b.s3}; return r; }
static inline d4 scale4(double s, d4 a) { d4 r = {s * a.s0, s * a.s1, s * a.s2, s * a.s3}; return r; }

/* moment_au (clUGKS.c:95-104): <a u^alpha v^beta psi> */
static d4 moment_au(d4 a, const double *Mu, const double *Mv, const double *Mxi, int al, int be) {
  d4 r = scale4(a.s0, moment_uv(Mu, Mv, Mxi, al + 0, be + 0, 0));
  r = add4(r, scale4(a.s1, moment_uv(Mu, Mv, Mxi, al + 1, be + 0, 0)));
  r = add4(r, scale4(a.s2, moment_uv(Mu, Mv, Mxi, al + 0, be + 1, 0)));
  r = add4(r, scale4(0.5 * a.s3, moment_uv(Mu, Mv, Mxi, al + 2, be + 0, 0)));
  r = add4(r, scale4(0.5 * a.s3, moment_uv(Mu, Mv, Mxi, al + 0, be + 2, 0)));
  r = add4(r, scale4(0.5 * a.s3, moment_uv(Mu, Mv, Mxi, al + 0, be + 0, 2)));
  return r;
}

/* time-integration weights Mt[0..4] (clUGKS.c:497-503) */
static void time_weights(double tau, double dt, double Mt[5]) {
  Mt[3] = tau * (1.0 - exp(-dt / tau));
  Mt[4] = -tau * dt * exp(-dt / tau) + tau * Mt[3];
  Mt[0] = dt - Mt[3];
  Mt[1] = -tau * Mt[0] + Mt[4];
  Mt[2] = (dt * dt) / 2.0 - tau * Mt[0];
}

/* limiters (clFunctions.c:255-353) */
static inline double vanleer1(double s1, double s2) {
  return (ocl_sign(s1) + ocl_sign(s2)) * (fabs(s1) * fabs(s2)) / (fabs(s1) + fabs(s2) + 1e-16);
}
static double weno5_1(const double *S, double dx) {
  const double eps = 1E-16;
  double t1, t2, B0, B1, B2, a0, a1, a2, w0, w1, w2, f0, f1, f2;
  t1 = S[0] - 2.0 * S[1] + S[2];
  t2 = S[0] - 4.0 * S[1] + 3.0 * S[2];
  B0 = (13.0 / 12.0) * t1 * t1 + 0.25 * t2 * t2;
  t1 = S[1] - 2.0 * S[2] + S[3];
  t2 = S[1] - S[3];
  B1 = (13.0 / 12.0) * t1 * t1 + 0.25 * t2 * t2;
  t1 = S[2] - 2.0 * S[3] + S[4];
  t2 = 3.0 * S[2] - 4.0 * S[3] + S[4];
  B2 = (13.0 / 12.0) * t1 * t1 + 0.25 * t2 * t2;
  t1 = eps + B0; a0 = 0.1 / (t1 * t1);
  t1 = eps + B1; a1 = 0.6 / (t1 * t1);
  t1 = eps + B2; a2 = 0.3 / (t1 * t1);
  t1 = a0 + a1 + a2;
  w0 = a0 / t1; w1 = a1 / t1; w2 = a2 / t1;
  f0 = (1. / 3.) * S[0] - (7. / 6.) * S[1] + (11. / 6.) * S[2];
  f1 = -(1. / 6.) * S[1] + (5. / 6.) * S[2] + (1. / 3.) * S[3];
  f2 = (1. / 3.) * S[2] + (5. / 6.) * S[3] - (1. / 6.) * S[4];
  double fL = w0 * f0 + w1 * f1 + w2 * f2;
  return (fL - S[2]) / dx;
}
static double minmod(double a, double b) {
  double out = 0.0;
  if ((fabs(a) < fabs(b)) && (a * b > 0)) out = a;
  else if ((fabs(b) < fabs(a)) && (a * b > 0)) out = b;
  else if (a == b) out = a;
  else if (a * b <= 0) out = 0;
  return out;
}
static double nnd1(const double *S, double dx) {
  double ip = S[1] + 0.5 * minmod(S[2] - S[1], S[1] - S[0]);
  return (ip - S[1]) / dx;
}

/* -------------------------------------------------------------------------
 * iFace (clUGKS.c:110-199): upwind reconstruction of f at every face of one
 * direction.  face==SOUTH: faces (mi < ni, mj < nj+1); WEST: (ni+1, nj).
 * ---------------------------------------------------------------------- */
void port_iFace(PP, size_t g0, size_t g1, const double *Fin, double *iface_f, double *fsigma,
                const double *centre, const double *mid_side, const double *normal, int face) {
  const int L = P->flux_method == 1 ? 5 : 3, MID = P->flux_method == 1 ? 2 : 1;
  for (size_t mi = 0; mi < g0; ++mi)
    for (size_t mj = 0; mj < g1; ++mj) {
      if (!(((face == SOUTH) && (mi < (size_t)P->ni) && (mj < (size_t)P->nj + 1)) ||
            ((face == WEST) && (mi < (size_t)P->ni + 1) && (mj < (size_t)P->nj))))
        continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d2 n = ld2(normal, FACEIDX(gi, gj, face));
      d2 mid = ld2(mid_side, FACEIDX(gi, gj, face));
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 uv = face_velocity(P, v, n);
        int delta = (int)((ocl_sign(uv.x) + 1) / 2);
        double fh[5], fb[5];
        d2 c[5];
        for (int s = 0; s < L; ++s) {
          long si, sj;
          if (face == SOUTH) {
            si = (long)gi;
            sj = delta * ((long)gj - MID - 1 + s) + (1 - delta) * ((long)gj + MID - s);
          } else {
            si = delta * ((long)gi - MID - 1 + s) + (1 - delta) * ((long)gi + MID - s);
            sj = (long)gj;
          }
          d2 f = ld2(Fin, FIDX(si, sj, v));
          fh[s] = f.x;
          fb[s] = f.y;
          c[s] = ld2(centre, GIDX(si, sj));
        }
        double ddx = mid.x - c[MID].x, ddy = mid.y - c[MID].y;
        double dist = sqrt(ddx * ddx + ddy * ddy);
        d2 sig;
        if (P->flux_method == 0) {
          double ax = c[MID].x - c[MID - 1].x, ay = c[MID].y - c[MID - 1].y;
          double bx = c[MID - 1].x - c[MID].x, by = c[MID - 1].y - c[MID].y;
          double l1 = sqrt(ax * ax + ay * ay), l2 = sqrt(bx * bx + by * by);
          double s1h = (fh[MID] - fh[MID - 1]) / l1, s1b = (fb[MID] - fb[MID - 1]) / l1;
          double s2h = (fh[MID + 1] - fh[MID]) / l2, s2b = (fb[MID + 1] - fb[MID]) / l2;
          sig.x = vanleer1(s1h, s2h);
          sig.y = vanleer1(s1b, s2b);
        } else if (P->flux_method == 1) {
          sig.x = weno5_1(fh, dist);
          sig.y = weno5_1(fb, dist);
        } else {
          sig.x = nnd1(fh, dist);
          sig.y = nnd1(fb, dist);
        }
        d2 out = {fh[MID] + sig.x * dist, fb[MID] + sig.y * dist};
        st2(iface_f, FIDX(gi, gj, v), out);
        st2(fsigma, FIDX(gi, gj, v), sig);
      }
    }
}

/* face range used by the face-moment kernels (clUGKS.c:218-225) */
static int face_in_range(PP, int face, size_t mi, size_t mj, int off_top) {
  return ((face == SOUTH) && (mi < (size_t)P->ni) && (mj < (size_t)(P->nj + 1 - off_top))) ||
         ((face == WEST) && (mi < (size_t)(P->ni + 1 - off_top)) && (mj < (size_t)P->nj));
}

/* conserved moments of a distribution in the frame of face normal n */
static d4 face_frame_moments(PP, const double *f, size_t base, d2 n) {
  d4 m = zero4();
  for (size_t v = 0; v < (size_t)P->Nv; ++v) {
    d2 fv = ld2(f, base + v);
    d2 uv = face_velocity(P, v, n);
    m.s0 += fv.x;
    m.s1 += uv.x * fv.x;
    m.s2 += uv.y * fv.x;
    m.s3 += 0.5 * ((uv.x * uv.x + uv.y * uv.y) * fv.x + fv.y);
  }
  return m;
}

/* getFaceCons / getAL / getAR (clUGKS.c:209-399) */
void port_getFaceCons(PP, size_t g0, size_t g1, const double *iface_f, const double *normal, int face,
                      double *primary, int off_bot, int off_top) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
      if (!face_in_range(P, face, mi, mj, off_top)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d2 n = ld2(normal, FACEIDX(gi, gj, face));
      st4(primary, GIDX(gi, gj), face_frame_moments(P, iface_f, FIDX(gi, gj, 0), n));
    }
}
void port_getAL(PP, size_t g0, size_t g1, const double *Fin, const double *normal, int face,
                double *gaL, int off_bot, int off_top) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
      if (!face_in_range(P, face, mi, mj, off_top)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d2 n = ld2(normal, FACEIDX(gi, gj, face));
      st4(gaL, GIDX(gi, gj), face_frame_moments(P, Fin, FIDX(gi - face, gj - (1 - face), 0), n));
    }
}
void port_getAR(PP, size_t g0, size_t g1, const double *Fin, const double *normal, int face,
                double *gaR, int off_bot, int off_top) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
      if (!face_in_range(P, face, mi, mj, off_top)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d2 n = ld2(normal, FACEIDX(gi, gj, face));
      st4(gaR, GIDX(gi, gj), face_frame_moments(P, Fin, FIDX(gi, gj, 0), n));
    }
}

/* getPLR (clUGKS.c:401-442) */
void port_getPLR(PP, size_t g0, size_t g1, const double *centre, const double *mid_side, int face,
                 double *primary, double *gaL, double *gaR, int off_bot, int off_top) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
      if (!face_in_range(P, face, mi, mj, off_top)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d4 w = ld4(primary, GIDX(gi, gj));
      d4 prim = to_primary(P, w);
      d2 mid = ld2(mid_side, FACEIDX(gi, gj, face));
      d2 cl = ld2(centre, GIDX(gi - face, gj - (1 - face)));
      d2 cr = ld2(centre, GIDX(gi, gj));
      double dl = sqrt((mid.x - cl.x) * (mid.x - cl.x) + (mid.y - cl.y) * (mid.y - cl.y));
      double dr = sqrt((mid.x - cr.x) * (mid.x - cr.x) + (mid.y - cr.y) * (mid.y - cr.y));
      d4 wl = ld4(gaL, GIDX(gi, gj)), wr = ld4(gaR, GIDX(gi, gj));
      d4 sw = {(w.s0 - wl.s0) / dl, (w.s1 - wl.s1) / dl, (w.s2 - wl.s2) / dl, (w.s3 - wl.s3) / dl};
      st4(gaL, GIDX(gi, gj), micro_slope(P, prim, sw));
      d4 sr = {(wr.s0 - w.s0) / dr, (wr.s1 - w.s1) / dr, (wr.s2 - w.s2) / dr, (wr.s3 - w.s3) / dr};
      st4(gaR, GIDX(gi, gj), micro_slope(P, prim, sr));
      st4(primary, GIDX(gi, gj), prim);
    }
}

/* initMacroFlux (clUGKS.c:446-518) */
void port_initMacroFlux(PP, size_t g0, size_t g1, double *flux_macro, int face, double dt,
                        const double *primary, const double *gaL, const double *gaR, double *gaT,
                        double *gMxi, int off_bot, int off_top) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
      if (!face_in_range(P, face, mi, mj, off_top)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d4 prim = ld4(primary, GIDX(gi, gj));
      d4 aL = ld4(gaL, GIDX(gi, gj)), aR = ld4(gaR, GIDX(gi, gj));
      double Mu[MNUM], Mv[MTUM], Mxi[3], MuL[MNUM], MuR[MNUM];
      moments_u(P, prim, Mu, Mv, Mxi, MuL, MuR);
      for (int k = 0; k < 3; ++k) gMxi[3 * GIDX(gi, gj) + k] = Mxi[k];
      d4 mL = moment_au(aL, MuL, Mv, Mxi, 1, 0);
      d4 mR = moment_au(aR, MuR, Mv, Mxi, 1, 0);
      d4 sw = scale4(-prim.s0, add4(mL, mR));
      d4 aT = micro_slope(P, prim, sw);
      st4(gaT, GIDX(gi, gj), aT);
      double tau = relax_time(P, prim), Mt[5];
      time_weights(tau, dt, Mt);
      d4 m0 = moment_uv(Mu, Mv, Mxi, 1, 0, 0);
      mL = moment_au(aL, MuL, Mv, Mxi, 2, 0);
      mR = moment_au(aR, MuR, Mv, Mxi, 2, 0);
      d4 mT = moment_au(aT, Mu, Mv, Mxi, 1, 0);
      d4 r = add4(add4(scale4(Mt[0], m0), scale4(Mt[1], add4(mL, mR))), scale4(Mt[2], mT));
      st4(flux_macro, GIDX(gi, gj), scale4(prim.s0, r));
    }
}

/* calcFaceQ (clUGKS.c:522-585) */
void port_calcFaceQ(PP, size_t g0, size_t g1, const double *iface_f, const double *primary,
                    const double *normal, double *faceQ, int face, int off_bot, int off_top) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
      if (!face_in_range(P, face, mi, mj, off_top)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d2 n = ld2(normal, FACEIDX(gi, gj, face));
      d4 prim = ld4(primary, GIDX(gi, gj));
      d2 Q = {0.0, 0.0};
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 f = ld2(iface_f, FIDX(gi, gj, v));
        d2 uv = face_velocity(P, v, n);
        double cx = uv.x - prim.s1, cy = uv.y - prim.s2, c2 = cx * cx + cy * cy;
        Q.x += 0.5 * ((uv.x - prim.s1) * (c2 * f.x + (f.y / P->K)));
        Q.y += 0.5 * ((uv.y - prim.s2) * (c2 * f.x + (f.y / P->K)));
      }
      st2(faceQ, GIDX(gi, gj), Q);
    }
}

/* macroFlux (clUGKS.c:587-681) */
void port_macroFlux(PP, size_t g0, size_t g1, const double *flux_f, const double *fsigma,
                    double *flux_macro, const double *normal, const double *side_length, int face,
                    double dt, const double *primary, const double *faceQ, int off_bot, int off_top) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
      if (!face_in_range(P, face, mi, mj, off_top)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d2 n = ld2(normal, FACEIDX(gi, gj, face));
      d4 prim = ld4(primary, GIDX(gi, gj));
      double tau = relax_time(P, prim), Mt[5];
      time_weights(tau, dt, Mt);
      d2 Q = ld2(faceQ, GIDX(gi, gj));
      d4 acc = zero4();
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 uv = face_velocity(P, v, n);
        d2 F0 = shakhov(P, prim, Q, uv, maxwellian(P, prim, uv, v));
        d2 fd = ld2(flux_f, FIDX(gi, gj, v));
        d2 fs = ld2(fsigma, FIDX(gi, gj, v));
        double u = uv.x, w = uv.y, uu = uv.x * uv.x + uv.y * uv.y;
        acc.s0 += Mt[0] * u * F0.x + Mt[3] * u * fd.x - Mt[4] * u * u * fs.x;
        acc.s1 += Mt[0] * u * u * F0.x + Mt[3] * u * u * fd.x - Mt[4] * u * u * u * fs.x;
        acc.s2 += Mt[0] * w * u * F0.x + Mt[3] * w * u * fd.x - Mt[4] * w * u * u * fs.x;
        acc.s3 += Mt[0] * 0.5 * (u * uu * F0.x + u * F0.y) + Mt[3] * 0.5 * (u * uu * fd.x + u * fd.y) -
                  Mt[4] * 0.5 * (u * u * uu * fs.x + u * u * fs.y);
      }
      d4 out = add4(acc, ld4(flux_macro, GIDX(gi, gj)));
      d2 m = {out.s1, out.s2};
      m = to_global(m, n);
      out.s1 = m.x;
      out.s2 = m.y;
      st4(flux_macro, GIDX(gi, gj), scale4(side_length[FACEIDX(gi, gj, face)], out));
    }
}

/* distFlux (clUGKS.c:683-772): per-velocity time-integrated flux, written
   over the interface distribution in place */
void port_distFlux(PP, size_t g0, size_t g1, double *flux_f, const double *fsigma,
                   const double *normal, const double *side_length, int face, double dt,
                   const double *primary, const double *gaL, const double *gaR, const double *gaT,
                   const double *gMxi, const double *faceQ, int off_bot, int off_top) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t mi = a + face * off_bot, mj = b + (1 - face) * off_bot;
      if (!face_in_range(P, face, mi, mj, off_top)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d4 prim = ld4(primary, GIDX(gi, gj));
      d4 aL = ld4(gaL, GIDX(gi, gj)), aR = ld4(gaR, GIDX(gi, gj)), aT = ld4(gaT, GIDX(gi, gj));
      double Mxi2 = gMxi[3 * GIDX(gi, gj) + 2];
      double tau = relax_time(P, prim), Mt[5];
      time_weights(tau, dt, Mt);
      d2 n = ld2(normal, FACEIDX(gi, gj, face));
      d2 Q = ld2(faceQ, GIDX(gi, gj));
      double len = side_length[FACEIDX(gi, gj, face)];
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 uv = face_velocity(P, v, n);
        int delta = (int)((ocl_sign(uv.x) + 1) / 2);
        d2 f0 = maxwellian(P, prim, uv, v);
        d2 F0 = shakhov(P, prim, Q, uv, f0);
        d2 fd = ld2(flux_f, FIDX(gi, gj, v));
        d2 fs = ld2(fsigma, FIDX(gi, gj, v));
        double u = uv.x, w = uv.y, uu = uv.x * uv.x + uv.y * uv.y;
        double hx = Mt[0] * u * (f0.x + F0.x) +
                    Mt[1] * (u * u) * (aL.s0 * f0.x + aL.s1 * u * f0.x + aL.s2 * w * f0.x + 0.5 * aL.s3 * (uu * f0.x + f0.y)) * delta +
                    Mt[1] * (u * u) * (aR.s0 * f0.x + aR.s1 * u * f0.x + aR.s2 * w * f0.x + 0.5 * aR.s3 * (uu * f0.x + f0.y)) * (1 - delta) +
                    Mt[2] * u * (aT.s0 * f0.x + aT.s1 * u * f0.x + aT.s2 * w * f0.x + 0.5 * aT.s3 * (uu * f0.x + f0.y)) +
                    Mt[3] * u * fd.x - Mt[4] * (u * u) * fs.x;
        double hy = Mt[0] * u * (f0.y + F0.y) +
                    Mt[1] * (u * u) * (aL.s0 * f0.y + aL.s1 * u * f0.y + aL.s2 * w * f0.y + 0.5 * aL.s3 * (uu * f0.y + Mxi2 * f0.x)) * delta +
                    Mt[1] * (u * u) * (aR.s0 * f0.y + aR.s1 * u * f0.y + aR.s2 * w * f0.y + 0.5 * aR.s3 * (uu * f0.y + Mxi2 * f0.x)) * (1 - delta) +
                    Mt[2] * u * (aT.s0 * f0.y + aT.s1 * u * f0.y + aT.s2 * w * f0.y + 0.5 * aT.s3 * (uu * f0.y + Mxi2 * f0.x)) +
                    Mt[3] * u * fd.y - Mt[4] * (u * u) * fs.y;
        d2 out = {len * hx, len * hy};
        st2(flux_f, FIDX(gi, gj, v), out);
      }
    }
}

/* distance_from_segment, intersect, get_tri, interpolate, vartheta_langmuir
   (clAdsorb.c:18-247): equilibrium coverage from a tabulated isotherm by a
   walk through its Delaunay triangulation; intersect works in single
   precision as the reference does */
static double distance_from_segment(d2 a, d2 b, d2 c) {
  double r_num = (c.x - a.x) * (b.x - a.x) + (c.y - a.y) * (b.y - a.y);
  double r_den = (b.x - a.x) * (b.x - a.x) + (b.y - a.y) * (b.y - a.y);
  double r = r_num / r_den;
  double s = ((a.y - c.y) * (b.x - a.x) - (a.x - c.x) * (b.y - a.y)) / r_den;
  double line = fabs(s) * sqrt(r_den);
  if ((r >= 0) && (r <= 1)) return line;
  double d1 = (c.x - a.x) * (c.x - a.x) + (c.y - a.y) * (c.y - a.y);
  double d2v = (c.x - b.x) * (c.x - b.x) + (c.y - b.y) * (c.y - b.y);
  return d1 < d2v ? sqrt(d1) : sqrt(d2v);
}
static int intersect(d2 a, d2 b, d2 c, d2 d) {
  float den = (float)((d.y - c.y) * (b.x - a.x) - (d.x - c.x) * (b.y - a.y));
  float num1 = (float)((d.x - c.x) * (a.y - c.y) - (d.y - c.y) * (a.x - c.x));
  float num2 = (float)((b.x - a.x) * (a.y - c.y) - (b.y - a.y) * (a.x - c.x));
  float u1 = num1 / den;
  float u2 = num2 / den;
  if (den == 0 && num1 == 0 && num2 == 0) return 0;
  if (den == 0) return 0;
  if (u1 < 0 || u1 > 1 || u2 < 0 || u2 > 1) return 0;
  return 1;
}
static d2 iso_pt(const double *iso, int k) { d2 r = {iso[4 * k], iso[4 * k + 1]}; return r; }
static void get_tri(d2 xy, const double *pts, const int32_t *tris, int size_tri, const int32_t *nbrs, int id,
                    int *out_id, int *out_outside) {
  const double tol = 1e-12;
  int outside = 0;
  for (int counter = 0; counter < size_tri; ++counter) {
    const int32_t *t = tris + 4 * id;
    d2 a = iso_pt(pts, t[0]), b = iso_pt(pts, t[1]), c = iso_pt(pts, t[2]);
    d2 start = {(1.0 / 3.0) * (a.x + b.x + c.x), (1.0 / 3.0) * (a.y + b.y + c.y)};
    int hz = intersect(a, b, start, xy), hx = intersect(b, c, start, xy), hy = intersect(c, a, start, xy);
    if ((hx + hy + hz) == 0) break;
    const int32_t *nb = nbrs + 4 * id;
    if (hx) {
      if (nb[0] == -1) { outside = 1; break; }
      else if (distance_from_segment(b, c, xy) < tol) break;
      else id = nb[0];
    } else if (hy) {
      if (nb[1] == -1) { outside = 1; break; }
      else if (distance_from_segment(c, a, xy) < tol) break;
      else id = nb[1];
    } else if (hz) {
      if (nb[2] == -1) { outside = 1; break; }
      else if (distance_from_segment(a, b, xy) < tol) break;
      else id = nb[2];
    }
  }
  *out_id = id;
  *out_outside = outside;
}
static double iso_interpolate(d2 pt, const double *a, const double *b, const double *c) {
  double L1 = ((b[1] - c[1]) * (pt.x - c[0]) + (c[0] - b[0]) * (pt.y - c[1])) /
              ((b[1] - c[1]) * (a[0] - c[0]) + (c[0] - b[0]) * (a[1] - c[1]));
  double L2 = ((c[1] - a[1]) * (pt.x - c[0]) + (a[0] - c[0]) * (pt.y - c[1])) /
              ((b[1] - c[1]) * (a[0] - c[0]) + (c[0] - b[0]) * (a[1] - c[1]));
  double L3 = 1 - L1 - L2;
  return L1 * a[2] + L2 * b[2] + L3 * c[2];
}
static d2 vartheta_langmuir(PP, double D, double T, int face) {
  d2 v;
  if (P->constant_adsorb[face]) { v.x = P->adsorb[face]; v.y = 0.0; return v; }
  d2 pt = {0.5 * D * T, T};
  int id, outside;
  get_tri(pt, P->iso[face], P->tri[face], P->n_tri[face], P->nbr[face], 0, &id, &outside);
  const int32_t *t = P->tri[face] + 4 * id;
  v.x = iso_interpolate(pt, P->iso[face] + 4 * t[0], P->iso[face] + 4 * t[1], P->iso[face] + 4 * t[2]);
  v.y = (double)outside;
  return v;
}

/* getInternal (clKernel.c:314-375): directional temperatures and stress */
void port_getInternal(PP, size_t g0, size_t g1, const double *Fin, double *Txyz, double *Stress) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      if (!(a < (size_t)P->ni && b < (size_t)P->nj)) continue;
      size_t gi = a + P->ghost, gj = b + P->ghost;
      double D = 0.0, M1 = 0.0, M2 = 0.0, M4 = 0.0, M5 = 0.0, M6 = 0.0, H = 0.0;
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 uv = quad_at(P, v);
        d2 f = ld2(Fin, FIDX(gi, gj, v));
        D += f.x;
        M1 += uv.x * f.x;
        M2 += uv.y * f.x;
        M4 += uv.x * uv.x * f.x;
        M5 += uv.y * uv.y * f.x;
        M6 += uv.x * uv.y * f.x;
        H += f.y;
      }
      double U = M1 / D, V = M2 / D;
      double Tx = 2 * (M4 / D - U * U), Ty = 2 * (M5 / D - V * V), Tz = 2 * (H / D);
      double T = (Tx + Ty + Tz) / P->B;
      size_t m = MIDX(a, b);
      Txyz[4 * m] = Tx; Txyz[4 * m + 1] = Ty; Txyz[4 * m + 2] = Tz; Txyz[4 * m + 3] = T;
      Stress[4 * m] = M4 - D * (U * U + T / 2.0);
      Stress[4 * m + 1] = M6 - D * (U * V + T / 2.0);
      Stress[4 * m + 2] = M5 - D * (V * V + T / 2.0);
      Stress[4 * m + 3] = 0.0;
    }
}

/* wall-face addressing shared by the wall kernels (clUGKS.c:795-824) */
static void wall_face(PP, int face, size_t *gi, size_t *gj, size_t *ci, int *rot, int *face_id) {
  switch (face) {
    case GNORTH: *ci = *gi; *gi += P->ghost; *gj += P->Nj - P->ghost; *rot = -1; *face_id = SOUTH; break;
    case GEAST: *ci = *gj; *gi += P->Ni - P->ghost; *gj += P->ghost; *rot = -1; *face_id = WEST; break;
    case GSOUTH: *ci = *gi; *gi += P->ghost; *gj += P->ghost; *rot = 1; *face_id = SOUTH; break;
    default: *ci = *gj; *gi += P->ghost; *gj += P->ghost; *rot = 1; *face_id = WEST; break;
  }
}
static int wall_in_range(PP, int face_id, size_t gi, size_t gj) {
  return ((face_id == SOUTH) && ((gi - P->ghost) < (size_t)P->ni)) ||
         ((face_id == WEST) && ((gj - P->ghost) < (size_t)P->nj));
}

/* accommodatingWallDist (clUGKS.c:776-906): diffuse wall */
void port_accommodatingWallDist(PP, size_t g0, size_t g1, const double *normal, int face,
                                const double *wall_prop, double *flux_f, double dt) {
  (void)dt;
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b, ci;
      int rot, fid;
      wall_face(P, face, &gi, &gj, &ci, &rot, &fid);
      if (!wall_in_range(P, fid, gi, gj)) continue;
      d2 n = ld2(normal, FACEIDX(gi, gj, fid));
      d4 wall = ld4(wall_prop, ci * 4 + face);
      d2 wv = {wall.s1, wall.s2};
      wv = to_local(wv, n);
      wall.s1 = wv.x;
      wall.s2 = wv.y;
      double sum_out = 0.0, sum_in = 0.0;
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 uv = face_velocity(P, v, n);
        d2 fd = ld2(flux_f, FIDX(gi, gj, v));
        int delta = (int)((ocl_sign(uv.x) * rot + 1) / 2);
        sum_out += uv.x * (1 - delta) * fd.x;
        d2 wd = maxwellian(P, wall, uv, v);
        sum_in -= uv.x * delta * wd.x;
      }
      double ratio = sum_out / sum_in;
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 uv = face_velocity(P, v, n);
        int delta = (int)((ocl_sign(uv.x) * rot + 1) / 2);
        d2 fd = ld2(flux_f, FIDX(gi, gj, v));
        d2 M = maxwellian(P, wall, uv, v);
        d2 out = {ratio * delta * M.x + (1 - delta) * fd.x, ratio * delta * M.y + (1 - delta) * fd.y};
        st2(flux_f, FIDX(gi, gj, v), out);
      }
    }
}

/* wallFlux (clUGKS.c:910-1011): first-order wall flux and its moments */
void port_wallFlux(PP, size_t g0, size_t g1, const double *normal, const double *side_length,
                   int face, double *flux_f, double *flux_macro, double dt) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b, ci;
      int rot, fid;
      wall_face(P, face, &gi, &gj, &ci, &rot, &fid);
      if (!wall_in_range(P, fid, gi, gj)) continue;
      d2 n = ld2(normal, FACEIDX(gi, gj, fid));
      double len = side_length[FACEIDX(gi, gj, fid)];
      d4 m = zero4();
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 uv = face_velocity(P, v, n);
        d2 wd = ld2(flux_f, FIDX(gi, gj, v));
        d2 out = {uv.x * wd.x * len * dt, uv.x * wd.y * len * dt};
        st2(flux_f, FIDX(gi, gj, v), out);
        m.s0 += uv.x * wd.x;
        m.s1 += uv.x * uv.x * wd.x;
        m.s2 += uv.x * uv.y * wd.x;
        m.s3 += 0.5 * uv.x * ((uv.x * uv.x + uv.y * uv.y) * wd.x + wd.y);
      }
      d2 mv = {m.s1, m.s2};
      mv = to_global(mv, n);
      m.s1 = mv.x;
      m.s2 = mv.y;
      st4(flux_macro, GIDX(gi, gj), scale4(dt * len, m));
    }
}

/* wallMassEnergyFluxes (clUGKS.c:1019-1147): diagnostic in/out fluxes */
void port_wallMassEnergyFluxes(PP, size_t g0, size_t g1, const double *normal,
                               const double *side_length, const double *area, int face,
                               const double *flux_f, double *wall_flux, double dt) {
  (void)side_length; (void)area; (void)dt;
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b, ci;
      int rot, fid;
      wall_face(P, face, &gi, &gj, &ci, &rot, &fid);
      if (!wall_in_range(P, fid, gi, gj)) continue;
      d2 n = ld2(normal, FACEIDX(gi, gj, fid));
      d4 din = zero4(), dout = zero4();
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 uv = face_velocity(P, v, n);
        int delta = (int)((ocl_sign(uv.x) * rot + 1) / 2);
        d2 wd = ld2(flux_f, FIDX(gi, gj, v));
        double uu = uv.x * uv.x + uv.y * uv.y;
        d2 fi = {(1 - delta) * wd.x, (1 - delta) * wd.y};
        d2 fo = {delta * wd.x, delta * wd.y};
        din.s0 += fi.x; din.s1 += uv.x * fi.x; din.s2 += uv.y * fi.x; din.s3 += 0.5 * (uu * fi.x + fi.y);
        dout.s0 += fo.x; dout.s1 += uv.x * fo.x; dout.s2 += uv.y * fo.x; dout.s3 += 0.5 * (uu * fo.x + fo.y);
      }
      d4 mi_ = scale4(-rot, din), mo = scale4(rot, dout);
      double *w = wall_flux + 8 * (ci * 4 + face);
      w[0] = mi_.s0; w[1] = mo.s0; w[2] = mi_.s1; w[3] = mo.s1;
      w[4] = mi_.s2; w[5] = mo.s2; w[6] = mi_.s3; w[7] = mo.s3;
    }
}

/* updateMacro (clUGKS.c:1158-1187) */
void port_updateMacro(PP, size_t g0, size_t g1, const double *flux_macro_S, const double *flux_macro_W,
                      const double *area, double *macro, double *residual) {
  for (size_t mi = 0; mi < g0; ++mi)
    for (size_t mj = 0; mj < g1; ++mj) {
      if (!(mi < (size_t)P->ni && mj < (size_t)P->nj)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d4 prim_old = ld4(macro, MIDX(mi, mj));
      d4 w = to_conserved(P, prim_old);
      double A = area[GIDX(gi, gj)];
      d4 s0 = ld4(flux_macro_S, GIDX(gi, gj)), s1 = ld4(flux_macro_S, GIDX(gi, gj + 1));
      d4 w0 = ld4(flux_macro_W, GIDX(gi, gj)), w1 = ld4(flux_macro_W, GIDX(gi + 1, gj));
      d4 nw = {w.s0 + (s0.s0 - s1.s0 + w0.s0 - w1.s0) / A, w.s1 + (s0.s1 - s1.s1 + w0.s1 - w1.s1) / A,
               w.s2 + (s0.s2 - s1.s2 + w0.s2 - w1.s2) / A, w.s3 + (s0.s3 - s1.s3 + w0.s3 - w1.s3) / A};
      st4(macro, MIDX(mi, mj), to_primary(P, nw));
      st4(residual, MIDX(mi, mj), prim_old);
    }
}

/* UGKS_update (clUGKS.c:1189-1257): implicit Shakhov-BGK relaxation */
void port_UGKS_update(PP, size_t g0, size_t g1, double *Fin, const double *flux_f_S,
                      const double *flux_f_W, const double *area, const double *macro,
                      const double *gQ, const double *residual, double dt, double *flag) {
  for (size_t mi = 0; mi < g0; ++mi)
    for (size_t mj = 0; mj < g1; ++mj) {
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d4 prim_old = ld4(residual, MIDX(mi, mj));
      double tau_old = relax_time(P, prim_old);
      d2 Q = ld2(gQ, MIDX(mi, mj));
      d4 prim = ld4(macro, MIDX(mi, mj));
      double tau = relax_time(P, prim);
      double A = area[GIDX(gi, gj)];
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 e = quad_at(P, v);
        d2 fo = shakhov_eq(P, prim_old, Q, e, v);
        d2 fn = shakhov_eq(P, prim, Q, e, v);
        d2 f = ld2(Fin, FIDX(gi, gj, v));
        d2 s0 = ld2(flux_f_S, FIDX(gi, gj, v)), s1 = ld2(flux_f_S, FIDX(gi, gj + 1, v));
        d2 w0 = ld2(flux_f_W, FIDX(gi, gj, v)), w1 = ld2(flux_f_W, FIDX(gi + 1, gj, v));
        double flh = (s0.x - s1.x + w0.x - w1.x) / A, flb = (s0.y - s1.y + w0.y - w1.y) / A;
        double rh = fn.x / tau + (fo.x - f.x) / tau_old, rb = fn.y / tau + (fo.y - f.y) / tau_old;
        double den = 1.0 + 0.5 * dt / tau;
        d2 out = {(f.x + flh + 0.5 * dt * rh) / den, (f.y + flb + 0.5 * dt * rb) / den};
        if (isnan(out.x) || isnan(out.y)) flag[0] = ERR_NAN;
        st2(Fin, FIDX(gi, gj, v), out);
      }
    }
}

/* getResidual (clUGKS.c:1259-1277) */
void port_getResidual(PP, size_t g0, size_t g1, const double *macro, double *residual) {
  for (size_t mi = 0; mi < g0; ++mi)
    for (size_t mj = 0; mj < g1; ++mj) {
      if (!(mi < (size_t)P->ni && mj < (size_t)P->nj)) continue;
      for (int k = 0; k < 4; ++k) {
        double d = macro[4 * MIDX(mi, mj) + k] - residual[4 * MIDX(mi, mj) + k];
        residual[4 * MIDX(mi, mj) + k] = d * d;
      }
    }
}

/* edgeMassFlow (clUGKS.c:1282-1337) */
void port_edgeMassFlow(PP, size_t g0, size_t g1, const double *macro, const double *normal,
                       const double *side_length, double *mdot, int this_face) {
  (void)g1;
  for (size_t ci = 0; ci < g0; ++ci) {
    size_t mi, mj, gi, gj;
    int face;
    double dir;
    if (this_face == GNORTH) { mi = ci; mj = P->nj - 1; gi = P->ghost + ci; gj = P->Nj - P->ghost; face = SOUTH; dir = 1; }
    else if (this_face == GEAST) { mi = P->ni - 1; mj = ci; gi = P->Ni - P->ghost; gj = P->ghost + ci; face = WEST; dir = 1; }
    else if (this_face == GSOUTH) { mi = ci; mj = 0; gi = P->ghost + ci; gj = P->ghost; face = SOUTH; dir = -1; }
    else { mi = 0; mj = ci; gi = P->ghost; gj = P->ghost + ci; face = WEST; dir = -1; }
    d2 n = ld2(normal, FACEIDX(gi, gj, face));
    n.x *= dir; n.y *= dir;
    double len = side_length[FACEIDX(gi, gj, face)];
    d4 m = ld4(macro, MIDX(mi, mj));
    mdot[ci * 4 + this_face] = (n.x * m.s1 + n.y * m.s2) * m.s0 * len;
  }
}

/* calcQ (clKernel.c:480-543) */
void port_calcQ(PP, size_t g0, size_t g1, const double *Fin, const double *macro, double *gQ) {
  for (size_t mi = 0; mi < g0; ++mi)
    for (size_t mj = 0; mj < g1; ++mj) {
      if (!(mi < (size_t)P->ni && mj < (size_t)P->nj)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d4 prim = ld4(macro, MIDX(mi, mj));
      d2 Q = {0.0, 0.0};
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 f = ld2(Fin, FIDX(gi, gj, v));
        d2 uv = quad_at(P, v);
        double cx = uv.x - prim.s1, cy = uv.y - prim.s2, c2 = cx * cx + cy * cy;
        Q.x += 0.5 * ((uv.x - prim.s1) * (c2 * f.x + (f.y / P->K)));
        Q.y += 0.5 * ((uv.y - prim.s2) * (c2 * f.x + (f.y / P->K)));
      }
      st2(gQ, MIDX(mi, mj), Q);
    }
}

/* calcMacro (clKernel.c:414-478) */
void port_calcMacro(PP, size_t g0, size_t g1, const double *Fin, double *macro) {
  for (size_t mi = 0; mi < g0; ++mi)
    for (size_t mj = 0; mj < g1; ++mj) {
      if (!(mi < (size_t)P->ni && mj < (size_t)P->nj)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d4 m = zero4();
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 f = ld2(Fin, FIDX(gi, gj, v));
        d2 uv = quad_at(P, v);
        m.s0 += f.x;
        m.s1 += uv.x * f.x;
        m.s2 += uv.y * f.x;
        m.s3 += 0.5 * ((uv.x * uv.x + uv.y * uv.y) * f.x + f.y);
      }
      d4 p = m;
      p.s3 = 0.5 * m.s0 / (P->gam - 1.0) / (m.s3 - 0.5 * (m.s1 * m.s1 + m.s2 * m.s2) / m.s0);
      p.s1 = m.s1 / m.s0;
      p.s2 = m.s2 / m.s0;
      st4(macro, MIDX(mi, mj), p);
    }
}

/* initFunctions (clKernel.c:382-412) */
void port_initFunctions(PP, size_t g0, size_t g1, double *Fin, const double *macro, const double *gQ) {
  for (size_t mi = 0; mi < g0; ++mi)
    for (size_t mj = 0; mj < g1; ++mj) {
      if (!(mi < (size_t)P->ni && mj < (size_t)P->nj)) continue;
      size_t gi = mi + P->ghost, gj = mj + P->ghost;
      d4 prim = ld4(macro, MIDX(mi, mj));
      d2 Q = ld2(gQ, MIDX(mi, mj));
      for (size_t v = 0; v < (size_t)P->Nv; ++v)
        st2(Fin, FIDX(gi, gj, v), shakhov_eq(P, prim, Q, quad_at(P, v), v));
    }
}

/* clFindDT (clKernel.c:224-308): per-cell CFL frequency */
void port_clFindDT(PP, size_t g0, size_t g1, const double *xy, const double *area,
                   const double *macro, double *time_step, double Kn) {
  const size_t NY = P->Nj + 1;
  for (size_t mi = 0; mi < g0; ++mi)
    for (size_t mj = 0; mj < g1; ++mj) {
      size_t G = P->ghost;
      d2 a = ld2(xy, (mi + 1 + G) * NY + mj + G), b = ld2(xy, (mi + 1 + G) * NY + mj + 1 + G);
      d2 c = ld2(xy, (mi + G) * NY + mj + 1 + G), d = ld2(xy, (mi + G) * NY + mj + G);
      double dx = fabs(a.x - b.x), t;
      if ((t = fabs(c.x - b.x)) > dx) dx = t;
      if ((t = fabs(c.x - d.x)) > dx) dx = t;
      if ((t = fabs(a.x - d.x)) > dx) dx = t;
      if ((t = fabs(c.x - a.x)) > dx) dx = t;
      if ((t = fabs(b.x - d.x)) > dx) dx = t;
      double dy = fabs(a.y - b.y);
      if ((t = fabs(c.y - b.y)) > dy) dy = t;
      if ((t = fabs(c.y - d.y)) > dy) dy = t;
      if ((t = fabs(a.y - d.y)) > dy) dy = t;
      if ((t = fabs(c.y - a.y)) > dy) dy = t;
      if ((t = fabs(b.y - d.y)) > dy) dy = t;
      d4 m = ld4(macro, MIDX(mi, mj));
      double sos = sqrt(0.5 * P->gam / m.s3);
      double lo_u = fmin(P->umax, fabs(m.s1) + sos), lo_v = fmin(P->vmax, fabs(m.s2) + sos);
      double hi_u = fmax(P->umax, fabs(m.s1) + sos), hi_v = fmax(P->vmax, fabs(m.s2) + sos);
      double scale = (erf(10 * (Kn - 1e-3)) + 1) / 2.0;
      double u = scale * (hi_u - lo_u) + lo_u, v = scale * (hi_v - lo_v) + lo_v;
      time_step[MIDX(mi, mj)] = (dx * u + dy * v) / area[GIDX(mi + G, mj + G)];
    }
}

/* paraBC (clKernel.c:141-218) for constant (non-UDF) wall values */
void port_paraBC(PP, size_t g0, size_t g1, const double *para_def, double *wall_prop, double t) {
  (void)g1; (void)para_def; (void)t;
  for (size_t ci = 0; ci < g0; ++ci) {
    for (int f = 0; f < 4; ++f) {
      int ns = (f == GNORTH || f == GSOUTH);
      if (ns ? !(ci < (size_t)P->ni) : !(ci < (size_t)P->nj)) continue;
      d4 prim;
      prim.s0 = P->wall_D[f];
      prim.s1 = P->wall_U[f];
      prim.s2 = P->wall_V[f];
      prim.s3 = (P->wall_P[f] != -1) ? P->wall_P[f] / P->wall_D[f] : P->wall_T[f];
      st4(wall_prop, ci * 4 + f, prim);
    }
  }
}

/* ghost-strip addressing of the edge kernels (clGhostRoutines.c:558-587) */
static void ghost_cell(PP, int face, size_t *gi, size_t *gj) {
  switch (face) {
    case GNORTH: *gi += P->ghost; *gj += P->Nj - P->ghost; break;
    case GEAST: *gi += P->Ni - P->ghost; *gj += P->ghost; break;
    case GSOUTH: *gi += P->ghost; break;
    default: *gj += P->ghost; break;
  }
}

static void rot90(int *i, int *j, int n, int Ni, int Nj) {
  for (int a = 0; a < n; a++) {
    int t = *i;
    *i = Nj - *j - 1;
    *j = t;
    t = Ni; Ni = Nj; Nj = t;
  }
}

/* getSwapIndex for cells (clGhostRoutines.c:47-138, v == 0) */
static void swap_cell_index(PP, int this_face, int *iB, int *jB, int that_face, int NIB, int NJB) {
  const int NI = P->Ni, NJ = P->Nj, G = P->ghost;
  switch (this_face) {
    case GEAST:
      if (that_face == GEAST) { *iB = (NI - 1) - *iB; *iB += NIB - 2 * G; }
      else if (that_face == GWEST) { *iB -= NI - 2 * G; }
      else if (that_face == GNORTH) { rot90(iB, jB, 3, NI, NJ); *jB += NJB - 2 * G; }
      else { rot90(iB, jB, 1, NI, NJ); *jB -= NI - 2 * G; }
      break;
    case GWEST:
      if (that_face == GWEST) { *iB = (NI - 1) - *iB; *iB -= NI - 2 * G; }
      else if (that_face == GEAST) { *iB += NIB - 2 * G; }
      else if (that_face == GNORTH) { rot90(iB, jB, 1, NI, NJ); *jB += NJB - 2 * G; }
      else { rot90(iB, jB, 3, NI, NJ); *jB -= NI - 2 * G; }
      break;
    case GNORTH:
      if (that_face == GNORTH) { *jB = (NJ - 1) - *jB; *jB += NJB - 2 * G; }
      else if (that_face == GSOUTH) { *jB -= NJ - 2 * G; }
      else if (that_face == GEAST) { rot90(iB, jB, 1, NI, NJ); *iB += NIB - 2 * G; }
      else { rot90(iB, jB, 3, NI, NJ); *iB -= NJ - 2 * G; }
      break;
    default: /* GSOUTH */
      if (that_face == GSOUTH) { *jB = (NJ - 1) - *jB; *jB -= NJ - 2 * G; }
      else if (that_face == GNORTH) { *jB += NJB - 2 * G; }
      else if (that_face == GEAST) { rot90(iB, jB, 3, NI, NJ); *iB += NIB - 2 * G; }
      else { rot90(iB, jB, 1, NI, NJ); *iB -= NJ - 2 * G; }
      break;
  }
}

static void face_corners(int face, int NI, int NJ, int G, int *a1i, int *a1j, int *a2i, int *a2j) {
  switch (face) {
    case GNORTH: *a1i = G; *a1j = NJ - G; *a2i = NI - G; *a2j = NJ - G; break;
    case GEAST: *a1i = NI - G; *a1j = G; *a2i = NI - G; *a2j = NJ - G; break;
    case GSOUTH: *a1i = G; *a1j = G; *a2i = NI - G; *a2j = G; break;
    default: *a1i = G; *a1j = G; *a2i = G; *a2j = NJ - G; break;
  }
}

/* edgeExchange (clGhostRoutines.c:407-538): neighbour ghosts, bit-exact copy */
void port_edgeExchange(PP, size_t g0, size_t g1, double *fA, const double *xyA, int this_face,
                       const double *fB, const double *xyB, int NIB, int NJB, int that_face,
                       int ori, int flip) {
  const int G = P->ghost, NI = P->Ni, NJ = P->Nj;
  int a1i, a1j, a2i, a2j, b1i, b1j, b2i, b2j;
  face_corners(this_face, NI, NJ, G, &a1i, &a1j, &a2i, &a2j);
  face_corners(that_face, NIB, NJB, G, &b1i, &b1j, &b2i, &b2j);
  const size_t NYA = NJ + 1, NYB = NJB + 1;
  d2 A1 = ld2(xyA, a1i * NYA + a1j), A2 = ld2(xyA, a2i * NYA + a2j);
  d2 B1 = ld2(xyB, b1i * NYB + b1j), B2 = ld2(xyB, b2i * NYB + b2j);
  int misalign = !(fabs(A1.x - B1.x) <= 1e-6) || !(fabs(A1.y - B1.y) <= 1e-6) ||
                 !(fabs(A2.x - B2.x) <= 1e-6) || !(fabs(A2.y - B2.y) <= 1e-6);
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b;
      ghost_cell(P, this_face, &gi, &gj);
      int iB = (int)gi, jB = (int)gj;
      if (misalign && ori) {
        if (this_face == GEAST || this_face == GWEST) jB = (NJ - 1) - jB;
        else iB = (NI - 1) - iB;
      }
      swap_cell_index(P, this_face, &iB, &jB, that_face, NIB, NJB);
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        size_t v2 = v;
        if (flip == FLIP_NS) v2 = (size_t)P->mirror_NS[v];
        else if (flip == FLIP_D) v2 = (size_t)P->mirror_D[v];
        else if (flip == FLIP_EW) v2 = (size_t)P->mirror_EW[v];
        size_t src = (((size_t)iB) * NJB + (size_t)jB) * P->Nv + v2;
        fA[2 * FIDX(gi, gj, v)] = fB[2 * src];
        fA[2 * FIDX(gi, gj, v) + 1] = fB[2 * src + 1];
      }
    }
}

/* edgeExtrapolate (clGhostRoutines.c:544-597) */
void port_edgeExtrapolate(PP, size_t g0, size_t g1, double *Fin, int this_face) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b, ei, ej;
      ghost_cell(P, this_face, &gi, &gj);
      switch (this_face) {
        case GNORTH: ei = gi; ej = P->Nj - P->ghost - 1; break;
        case GEAST: ei = P->Ni - P->ghost - 1; ej = gj; break;
        case GSOUTH: ei = gi; ej = P->ghost; break;
        default: ei = P->ghost; ej = gj; break;
      }
      memcpy(Fin + 2 * FIDX(gi, gj, 0), Fin + 2 * FIDX(ei, ej, 0), sizeof(double) * 2 * P->Nv);
    }
}

/* edgeConstant (clGhostRoutines.c:603-658) */
void port_edgeConstant(PP, size_t g0, size_t g1, double *Fin, int this_face, const double *wall_prop) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b;
      size_t ci = (this_face == GNORTH || this_face == GSOUTH) ? a : b;
      ghost_cell(P, this_face, &gi, &gj);
      d4 prim = ld4(wall_prop, ci * 4 + this_face);
      d2 Q = {0.0, 0.0};
      for (size_t v = 0; v < (size_t)P->Nv; ++v)
        st2(Fin, FIDX(gi, gj, v), shakhov_eq(P, prim, Q, quad_at(P, v), v));
    }
}

/* edgeInflow / edgeOutflow (clGhostRoutines.c:664-839) */
static void inflow_outflow(PP, size_t g0, size_t g1, double *Fin, int this_face, const double *normal,
                           const double *macro, const double *gQ, const double *wall_prop, int outflow) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b, ei, ej, noi, noj, ci;
      int face;
      ghost_cell(P, this_face, &gi, &gj);
      switch (this_face) {
        case GNORTH: ci = a; ei = gi; ej = P->Nj - P->ghost - 1; noi = gi; noj = gj; face = SOUTH; break;
        case GEAST: ci = b; ei = P->Ni - P->ghost - 1; ej = gj; noi = gi; noj = gj; face = WEST; break;
        case GSOUTH: ci = a; ei = gi; ej = P->ghost; noi = ei; noj = ej; face = SOUTH; break;
        default: ci = b; ei = P->ghost; ej = gj; noi = ei; noj = ej; face = WEST; break;
      }
      d4 prim = ld4(wall_prop, ci * 4 + this_face);
      d2 Q = ld2(gQ, MIDX(ei - P->ghost, ej - P->ghost));
      d4 gm = ld4(macro, MIDX(ei - P->ghost, ej - P->ghost));
      d2 n = ld2(normal, FACEIDX(noi, noj, face));
      d2 uv = {gm.s1, gm.s2};
      uv = to_local(uv, n);
      gm.s1 = uv.x;
      gm.s2 = uv.y;
      if (outflow) {
        gm.s3 = gm.s0 / (prim.s0 / prim.s3);
      } else {
        gm.s0 = prim.s0;
        gm.s3 = prim.s3;
      }
      for (size_t v = 0; v < (size_t)P->Nv; ++v)
        st2(Fin, FIDX(gi, gj, v), shakhov_eq(P, gm, Q, quad_at(P, v), v));
    }
}
void port_edgeInflow(PP, size_t g0, size_t g1, double *Fin, int this_face, const double *normal,
                     const double *macro, const double *gQ, const double *wall_prop) {
  inflow_outflow(P, g0, g1, Fin, this_face, normal, macro, gQ, wall_prop, 0);
}
void port_edgeOutflow(PP, size_t g0, size_t g1, double *Fin, int this_face, const double *normal,
                      const double *macro, const double *gQ, const double *wall_prop) {
  inflow_outflow(P, g0, g1, Fin, this_face, normal, macro, gQ, wall_prop, 1);
}

/* edgeMirror / edgeBounceBack (clGhostRoutines.c:845-961) */
static void mirror_edge(PP, size_t g0, size_t g1, double *Fin, int this_face, int bounce) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b, mi, mj;
      ghost_cell(P, this_face, &gi, &gj);
      const int64_t *perm;
      switch (this_face) {
        case GNORTH: mi = gi; mj = 2 * (P->Nj - P->ghost) - gj - 1; perm = P->mirror_NS; break;
        case GEAST: mi = 2 * (P->Ni - P->ghost) - gi - 1; mj = gj; perm = P->mirror_EW; break;
        case GSOUTH: mi = gi; mj = 2 * P->ghost - gj - 1; perm = P->mirror_NS; break;
        default: mi = 2 * P->ghost - gi - 1; mj = gj; perm = P->mirror_EW; break;
      }
      if (bounce) perm = P->mirror_D;
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        size_t src = FIDX(mi, mj, (size_t)perm[v]);
        Fin[2 * FIDX(gi, gj, v)] = Fin[2 * src];
        Fin[2 * FIDX(gi, gj, v) + 1] = Fin[2 * src + 1];
      }
    }
}
void port_edgeMirror(PP, size_t g0, size_t g1, double *Fin, int this_face) {
  mirror_edge(P, g0, g1, Fin, this_face, 0);
}
void port_edgeBounceBack(PP, size_t g0, size_t g1, double *Fin, int this_face) {
  mirror_edge(P, g0, g1, Fin, this_face, 1);
}

/* edgeConstGrad (clGhostRoutines.c:967-1048) */
void port_edgeConstGrad(PP, size_t g0, size_t g1, double *Fin, int this_face) {
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b;
      long ei0, ej0, ei1, ej1;
      double m;
      ghost_cell(P, this_face, &gi, &gj);
      switch (this_face) {
        case GNORTH: ei1 = gi; ej1 = P->Nj - P->ghost - 1; ei0 = ei1; ej0 = ej1 - 1; m = (double)((long)gj - ej1); break;
        case GEAST: ei1 = P->Ni - P->ghost - 1; ej1 = gj; ei0 = ei1 - 1; ej0 = ej1; m = (double)((long)gi - ei1); break;
        case GSOUTH: ei1 = gi; ej1 = P->ghost; ei0 = ei1; ej0 = ej1 + 1; m = (double)(ej1 - (long)gj); break;
        default: ei1 = P->ghost; ej1 = gj; ei0 = ei1 + 1; ej0 = ej1; m = (double)(ei1 - (long)gi); break;
      }
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 f0 = ld2(Fin, FIDX(ei0, ej0, v)), f1 = ld2(Fin, FIDX(ei1, ej1, v));
        d2 out = {f1.x + m * (f1.x - f0.x), f1.y + m * (f1.y - f0.y)};
        st2(Fin, FIDX(gi, gj, v), out);
      }
    }
}

/* stickingProbability (clAdsorb.c:6-16) */
static double sticking(PP, d2 uv, double T, int face) {
  double nrm = 1.0 - P->beta_n[face] * exp(-uv.x * uv.x / T);
  double tan_ = 1.0 - P->beta_t[face] * (1.0 - exp(-uv.y * uv.y / T));
  return nrm * tan_;
}

/* adsorbingWall_P1 (clAdsorb.c:253-482): impinging flux split into adsorbed
   and reflected parts, coverage update, desorption.  Only the constant
   isotherm is restated (vartheta_langmuir, clAdsorb.c:186-191). */
void port_adsorbingWall_P1(PP, size_t g0, size_t g1, const double *normal, int face,
                           const double *wall_prop, double *wall_cover, double *wall_dist,
                           const double *flux_f, const double *macro, double dt, double *flag) {
  (void)wall_prop;
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b, ci;
      int rot, fid;
      double T, D;
      wall_face(P, face, &gi, &gj, &ci, &rot, &fid);
      switch (face) {
        case GNORTH: T = 1.0 / macro[4 * MIDX(ci, gj - P->ghost - 1) + 3]; D = macro[4 * MIDX(ci, gj - P->ghost - 1)]; break;
        case GEAST: T = 1.0 / macro[4 * MIDX(gi - P->ghost - 1, ci) + 3]; D = macro[4 * MIDX(gi - P->ghost - 1, ci)]; break;
        case GSOUTH: T = 1.0 / macro[4 * MIDX(ci, gj - P->ghost) + 3]; D = macro[4 * MIDX(ci, gj - P->ghost)]; break;
        default: T = 1.0 / macro[4 * MIDX(gi - P->ghost, ci) + 3]; D = macro[4 * MIDX(gi - P->ghost, ci)]; break;
      }
      (void)D;
      if (!wall_in_range(P, fid, gi, gj)) continue;
      d2 n = ld2(normal, FACEIDX(gi, gj, fid));
      double *cover = wall_cover + 4 * (ci * 4 + face);
      double vartheta = cover[0];
      double refl_sum = 0.0, ads_sum = 0.0, adj_sum = 0.0;
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 uv = face_velocity(P, v, n);
        d2 fd = ld2(flux_f, FIDX(gi, gj, v));
        int delta = (int)((ocl_sign(uv.x) * rot + 1) / 2);
        double k = -rot * uv.x * (1 - delta);
        d2 total = {k * fd.x, k * fd.y};
        double beta = sticking(P, uv, T, face);
        double g = beta * P->gamma_f[face] * (1.0 - vartheta);
        d2 ads = {beta * total.x * P->gamma_f[face] * (1.0 - vartheta),
                  beta * total.y * P->gamma_f[face] * (1.0 - vartheta)};
        (void)g;
        double fs = ocl_sign(total.x);
        if ((fs * ads.x) > (fs * total.x)) ads = total;
        d2 refl = {total.x - ads.x, total.y - ads.y};
        refl_sum += refl.x;
        ads_sum += ads.x;
        adj_sum += beta * total.x;
        d2 wd = {refl.x / uv.x, refl.y / uv.x};
        st2(wall_dist, ci * P->Nv + v, wd);
      }
      double correct = 1.0;
      double ads_final = ads_sum, dvt, des = 0.0;
      if (P->gamma_f[face] > 0.0) {
        if (P->dynamic[face] == 1) {
          dvt = dt * P->alpha_p[face] * ads_sum;
          if (dvt > (1 - vartheta)) {
            dvt = 1 - vartheta;
            ads_final = dvt / dt * P->alpha_p[face];  /* reference form (clAdsorb.c:420) */
          }
        } else {
          dvt = 0.0;
          ads_final = ads_sum;
        }
        if (P->k_des[face] > 0.0) {
          /* first-order desorption: rate k_des * coverage (no reference counterpart) */
          des = P->k_des[face] * vartheta / P->alpha_p[face];
        } else {
          d2 veq = vartheta_langmuir(P, D, T, face);
          if (veq.y == 1) {
            /* outside the tabulated isotherm (clAdsorb.c:430-434) */
            flag[0] = ERR_CLAMPING_ADSORB_ISOTHERM;
            continue;
          }
          double gamma_b = P->gamma_f[face] * (1.0 / veq.x - 1.0) * adj_sum;
          des = gamma_b * vartheta;
        }
        if (P->dynamic[face] == 1) {
          dvt -= dt * P->alpha_p[face] * des;
          if ((vartheta + dvt) < 0.0) des = vartheta / (dt * P->alpha_p[face]);
        }
      } else {
        dvt = 0.0;
      }
      double refl_final = refl_sum + ads_sum - ads_final;
      correct = refl_final / refl_sum;
      cover[0] += dvt;
      cover[1] = refl_final;
      cover[2] = ads_final;
      cover[3] = des;
      if (correct != 1.0)
        for (size_t v = 0; v < (size_t)P->Nv; ++v) {
          wall_dist[2 * (ci * P->Nv + v)] *= correct;
          wall_dist[2 * (ci * P->Nv + v) + 1] *= correct;
        }
    }
}

/* the second half of adsorbingWall{S,CL,D}_P2 (clAdsorb.c:601-649, 766-814,
   931-973): scale the re-emitted half by `ratio` and add the desorbed
   particles as a wall Maxwellian of density 2 des sqrt(pi lambda_w) */
static void add_desorbed(PP, double *flux_f, size_t gi, size_t gj, d2 n, int rot, d4 wall, const double *cover,
                         double ratio) {
  double refl = cover[1], des = cover[3], ads = cover[2];
  size_t account = ((des == 0.0) && (ads > 0.0) && (refl == 0.0)) ? 1 : 0;
  wall.s0 = 2 * des * sqrt(P->PI * wall.s3);
  for (size_t v = 0; v < (size_t)P->Nv; ++v) {
    d2 uv = face_velocity(P, v, n);
    int delta = (int)((ocl_sign(uv.x) * rot + 1) / 2);
    d2 fd = ld2(flux_f, FIDX(gi, gj, v));
    double sc = 1 - delta * (1 - ratio);
    fd.x *= sc;
    fd.y *= sc;
    d2 M = maxwellian(P, wall, uv, v);
    fd.x += delta * M.x;
    fd.y += delta * M.y;
    fd.x -= account * delta * fd.x;
    fd.y -= account * delta * fd.y;
    st2(flux_f, FIDX(gi, gj, v), fd);
  }
}

/* adsorbingWallS_P2 (clAdsorb.c:656-816): the reflected part of the
   incoming flux is re-emitted specularly, through the velocity mirrored
   about the wall (mirror_EW on WEST/EAST faces, mirror_NS on SOUTH/NORTH;
   axis-aligned walls only, as in the reference) */
void port_adsorbingWallS_P2(PP, size_t g0, size_t g1, const double *normal, int face,
                            const double *wall_prop, const double *wall_cover, const double *wall_dist,
                            double *flux_f, const double *macro, double dt) {
  (void)macro; (void)dt;
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b, ci;
      int rot, fid;
      wall_face(P, face, &gi, &gj, &ci, &rot, &fid);
      if (!wall_in_range(P, fid, gi, gj)) continue;
      d2 n = ld2(normal, FACEIDX(gi, gj, fid));
      d4 wall = ld4(wall_prop, ci * 4 + face);
      d2 wv = {wall.s1, wall.s2};
      wv = to_local(wv, n);
      wall.s1 = wv.x;
      wall.s2 = wv.y;
      const double *cover = wall_cover + 4 * (ci * 4 + face);
      double refl = cover[1];
      double ratio = 1.0;
      if (refl > 0.0) {
        double s = 0.0;
        for (size_t v = 0; v < (size_t)P->Nv; ++v) {
          d2 uv = face_velocity(P, v, n);
          int delta = (int)((ocl_sign(uv.x) * rot + 1) / 2);
          d2 spec = {0.0, 0.0};
          if (delta) {
            size_t mv = (size_t)(fid == WEST ? P->mirror_EW[v] : P->mirror_NS[v]);
            spec = ld2(wall_dist, ci * P->Nv + mv);
          }
          d2 fd = ld2(flux_f, FIDX(gi, gj, v));
          d2 out = {delta * spec.x + (1 - delta) * fd.x, delta * spec.y + (1 - delta) * fd.y};
          st2(flux_f, FIDX(gi, gj, v), out);
          s += rot * uv.x * spec.x;
        }
        ratio = refl / s;
      }
      add_desorbed(P, flux_f, gi, gj, n, rot, wall, cover, ratio);
    }
}

/* modified Bessel function I0 by its power series sum_k ((x/2)^2)^k / (k!)^2
   (all terms positive; the reference evaluates I0 by Blair's rational
   Chebyshev approximation, clFunctions.c:88-145, which agrees to rounding) */
static double bessel_i0(double x) {
  const double y = 0.25 * x * x;
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 1000; ++k) {
    term *= y / ((double)k * (double)k);
    sum += term;
    if (term < 1e-17 * sum) break;
  }
  return sum;
}

/* scatterNormal, scatterTangential, CercignaniLampis (clFunctions.c:146-185) */
static double scatter_normal(PP, double c_in, double c_out, double an, double Tw) {
  (void)P;
  return (2.0 / (an * Tw)) * fabs(c_out) * bessel_i0(((2 * sqrt(1 - an)) / (an * Tw)) * c_in * c_out) *
         exp(-(c_out * c_out + (1 - an) * c_in * c_in) / (an * Tw));
}
static double scatter_tangential(PP, double c_in, double c_out, double at, double Tw) {
  double a = c_out - (1 - at) * c_in;
  return (1.0 / sqrt(P->PI * at * (2 - at) * Tw)) * exp(-(a * a) / (at * (2 - at) * Tw));
}
static d2 cercignani_lampis(PP, d2 uv_in, d2 uv_out, d2 f_in, double an, double at, double Tw) {
  double k = fabs(uv_in.x / uv_out.x) * scatter_normal(P, uv_in.x, uv_out.x, an, Tw) *
             scatter_tangential(P, uv_in.y, uv_out.y, at, Tw);
  d2 r = {k * f_in.x, k * f_in.y};
  r.y *= (1 - at) * (1 - at);
  return r;
}

/* adsorbingWallCL_P2 (clAdsorb.c:488-651): the reflected part of the
   incoming flux is re-emitted through the Cercignani-Lampis kernel, an
   O(Nv^2) sum over incoming velocities per outgoing velocity */
void port_adsorbingWallCL_P2(PP, size_t g0, size_t g1, const double *normal, int face,
                             const double *wall_prop, const double *wall_cover, const double *wall_dist,
                             double *flux_f, const double *macro, double dt) {
  (void)macro; (void)dt;
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b, ci;
      int rot, fid;
      wall_face(P, face, &gi, &gj, &ci, &rot, &fid);
      if (!wall_in_range(P, fid, gi, gj)) continue;
      d2 n = ld2(normal, FACEIDX(gi, gj, fid));
      d4 wall = ld4(wall_prop, ci * 4 + face);
      d2 wv = {wall.s1, wall.s2};
      wv = to_local(wv, n);
      wall.s1 = wv.x;
      wall.s2 = wv.y;
      const double *cover = wall_cover + 4 * (ci * 4 + face);
      double refl = cover[1];
      double ratio = 1.0;
      const double an = P->alpha_n[face], at = P->alpha_t[face];
      if (refl > 0.0) {
        double s = 0.0;
        for (size_t v = 0; v < (size_t)P->Nv; ++v) {
          d2 uv_out = face_velocity(P, v, n);
          int delta = (int)((ocl_sign(uv_out.x) * rot + 1) / 2);
          d2 cl_v = {0.0, 0.0};
          if (delta) {
            for (size_t va = 0; va < (size_t)P->Nv; ++va) {
              d2 uv_in = face_velocity(P, va, n);
              int delta_in = (int)((ocl_sign(uv_in.x) * rot + 1) / 2);
              if ((!delta_in) && (uv_in.x != 0.0)) {
                d2 cl = cercignani_lampis(P, uv_in, uv_out, ld2(wall_dist, ci * P->Nv + va), an, at,
                                          1.0 / wall.s3);
                cl.y += 0.5 * at * (2 - at) / wall.s3 * cl.x;
                cl_v.x += cl.x;
                cl_v.y += cl.y;
              }
            }
            cl_v.x *= P->weight[v];
            cl_v.y *= P->weight[v];
          }
          d2 fd = ld2(flux_f, FIDX(gi, gj, v));
          d2 out = {delta * cl_v.x + (1 - delta) * fd.x, delta * cl_v.y + (1 - delta) * fd.y};
          st2(flux_f, FIDX(gi, gj, v), out);
          s += rot * uv_out.x * cl_v.x;
        }
        ratio = refl / s;
      }
      add_desorbed(P, flux_f, gi, gj, n, rot, wall, cover, ratio);
    }
}

/* adsorbingWallD_P2 (clAdsorb.c:821-975): diffuse re-emission of the
   reflected flux plus the desorbed particles */
void port_adsorbingWallD_P2(PP, size_t g0, size_t g1, const double *normal, int face,
                            const double *wall_prop, const double *wall_cover, const double *wall_dist,
                            double *flux_f, const double *macro, double dt) {
  (void)wall_dist; (void)macro; (void)dt;
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      size_t gi = a, gj = b, ci;
      int rot, fid;
      wall_face(P, face, &gi, &gj, &ci, &rot, &fid);
      if (!wall_in_range(P, fid, gi, gj)) continue;
      d2 n = ld2(normal, FACEIDX(gi, gj, fid));
      d4 wall = ld4(wall_prop, ci * 4 + face);
      d2 wv = {wall.s1, wall.s2};
      wv = to_local(wv, n);
      wall.s1 = wv.x;
      wall.s2 = wv.y;
      const double *cover = wall_cover + 4 * (ci * 4 + face);
      double refl = cover[1];
      double ratio = 1.0;
      if (refl > 0.0) {
        double s = 0.0;
        for (size_t v = 0; v < (size_t)P->Nv; ++v) {
          d2 uv = face_velocity(P, v, n);
          int delta = (int)((ocl_sign(uv.x) * rot + 1) / 2);
          d2 dif = {0.0, 0.0};
          if (delta) dif = maxwellian(P, wall, uv, v);
          d2 fd = ld2(flux_f, FIDX(gi, gj, v));
          d2 out = {delta * dif.x + (1 - delta) * fd.x, delta * dif.y + (1 - delta) * fd.y};
          st2(flux_f, FIDX(gi, gj, v), out);
          s += rot * uv.x * dif.x;
        }
        ratio = refl / s;
      }
      double des = cover[3], ads = cover[2];
      size_t account = ((des == 0.0) && (ads > 0.0) && (refl == 0.0)) ? 1 : 0;
      wall.s0 = 2 * des * sqrt(P->PI * wall.s3);
      for (size_t v = 0; v < (size_t)P->Nv; ++v) {
        d2 uv = face_velocity(P, v, n);
        int delta = (int)((ocl_sign(uv.x) * rot + 1) / 2);
        d2 fd = ld2(flux_f, FIDX(gi, gj, v));
        double sc = 1 - delta * (1 - ratio);
        fd.x *= sc;
        fd.y *= sc;
        d2 M = maxwellian(P, wall, uv, v);
        fd.x += delta * M.x;
        fd.y += delta * M.y;
        fd.x -= account * delta * fd.x;
        fd.y -= account * delta * fd.y;
        st2(flux_f, FIDX(gi, gj, v), fd);
      }
    }
}
