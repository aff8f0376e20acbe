// ugks_geometry.cu -- block geometry set-up: ghost vertices from the
// neighbouring block (xyExchange) or by extrapolation (xyExtrapolate), then
// the cell metrics (cellGeom), as UGKSBlock.updateGeom runs them
// (ugks_block.py:667-760).  Built with -fmad=false: every product and sum is
// rounded on its own, as in the reference's expressions, so the results are
// those of a sequential evaluation of the same formulas.
#include <cuda_runtime.h>
#include <math.h>

#include "ugks_device.cuh"

using namespace ugks;

namespace {

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }
inline int launch_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -(int)e;
}

constexpr int NO_TRANSFORM = 0, MIRROR = 2;

__device__ __forceinline__ V2 xy_at(const double *xy, int NJ, long i, long j) {
  return ld2(xy, (size_t)i * (NJ + 1) + j);
}
__device__ __forceinline__ void xy_set(double *xy, int NJ, long i, long j, V2 p) {
  st2(xy, (size_t)i * (NJ + 1) + j, p);
}

// vertex corners of a block face (xyExchange's A1/A2, B1/B2)
__device__ __forceinline__ void face_corners(int face, int NI, int NJ, int G, int &i1, int &j1, int &i2, int &j2) {
  switch (face) {
    case GNORTH: i1 = G; j1 = NJ - G; i2 = NI - G; j2 = NJ - G; break;
    case GEAST: i1 = NI - G; j1 = G; i2 = NI - G; j2 = NJ - G; break;
    case GSOUTH: i1 = G; j1 = G; i2 = NI - G; j2 = G; break;
    default: i1 = G; j1 = G; i2 = G; j2 = NJ - G; break;
  }
}

// getSwapIndex (clGhostRoutines.c:47-138) for vertex indices
__device__ void swap_vertex_index(int NI, int NJ, int G, int this_face, int &iB, int &jB, int that_face, int NIB,
                                  int NJB) {
  auto rot = [&](int n) {
    int ni = NI + 1, nj = NJ + 1;
    for (int a = 0; a < n; ++a) {
      const int t = iB;
      iB = nj - jB - 1;
      jB = t;
      const int s = ni; ni = nj; nj = s;
    }
  };
  switch (this_face) {
    case GEAST:
      if (that_face == GEAST) { iB = NI - iB; iB += NIB - 2 * G; }
      else if (that_face == GWEST) { iB -= NI - 2 * G; }
      else if (that_face == GNORTH) { rot(3); jB += NJB - 2 * G; }
      else { rot(1); jB -= NI - 2 * G; }
      break;
    case GWEST:
      if (that_face == GWEST) { iB = NI - iB; iB -= NI - 2 * G; }
      else if (that_face == GEAST) { iB += NIB - 2 * G; }
      else if (that_face == GNORTH) { rot(1); jB += NJB - 2 * G; }
      else { rot(3); jB -= NI - 2 * G; }
      break;
    case GNORTH:
      if (that_face == GNORTH) { jB = NJ - jB; jB += NJB - 2 * G; }
      else if (that_face == GSOUTH) { jB -= NJ - 2 * G; }
      else if (that_face == GEAST) { rot(1); iB += NIB - 2 * G; }
      else { rot(3); iB -= NJ - 2 * G; }
      break;
    default:
      if (that_face == GSOUTH) { jB = NJ - jB; jB -= NJ - 2 * G; }
      else if (that_face == GNORTH) { jB += NJB - 2 * G; }
      else if (that_face == GEAST) { rot(3); iB += NIB - 2 * G; }
      else { rot(1); iB -= NJ - 2 * G; }
      break;
  }
}

// transform (clFunctions.c:381-402): the affine map taking a0 -> b0-side,
// a1 -> b1-side corners, applied to n
__device__ V2 corner_transform(V2 a0, V2 a1, V2 b0, V2 b1, V2 n) {
  const double d1 = fabs(a0.x - a1.x) * fabs(a0.x - a1.x) + fabs(a0.y - a1.y) * fabs(a0.y - a1.y);
  const double d2 = ((a0.x - a1.x) * (a0.x - a1.x) + (a0.y - a1.y) * (a0.y - a1.y)) *
                    (fabs(b0.x - b1.x) * fabs(b0.x - b1.x) + fabs(b0.y - b1.y) * fabs(b0.y - b1.y));
  const double q = b0.x * b0.x + b1.x * n.x - b0.x * (b1.x + n.x) + (b0.y - b1.y) * (b0.y - n.y);
  V2 m;
  m.x = a0.x - ((-(a1.x * ((b0.x - b1.x) * (b0.x - n.x) + (b0.y - b1.y) * (b0.y - n.y))) + a0.x * q +
                 (a0.y - a1.y) * (b0.y * b1.x - b0.x * b1.y - b0.y * n.x + b1.y * n.x + b0.x * n.y - b1.x * n.y)) *
                d1) / d2;
  m.y = a0.y - ((a0.y * q - a1.y * q +
                 (a0.x - a1.x) * (b0.x * b1.y - b1.y * n.x + b0.y * (-b1.x + n.x) - b0.x * n.y + b1.x * n.y)) *
                d1) / d2;
  return m;
}

// mirror2D (clFunctions.c:404-428): reflection of p about the line a-b
__device__ V2 mirror_about(V2 a, V2 b, V2 p) {
  const double l2 = (b.x - a.x) * (b.x - a.x) + (b.y - a.y) * (b.y - a.y);
  if (l2 == 0.0) return p;
  const double t = ((p.x - a.x) * (b.x - a.x) + (p.y - a.y) * (b.y - a.y)) / l2;
  const V2 r = v2(a.x + t * (b.x - a.x), a.y + t * (b.y - a.y));
  return v2(r.x + (r.x - p.x), r.y + (r.y - p.y));
}

// xyExchange (clGhostRoutines.c:155-284): one work item per ghost vertex pair
__global__ void k_xyExchange(ugks_block_desc d, size_t g0, size_t g1, double *xyA, int this_face, const double *xyB,
                             int NIB, int NJB, int that_face, int ori, int affine, int flip_normal) {
  const size_t w = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (w >= g0 * g1) return;
  long gi = (long)(w / g1), gj = (long)(w % g1);
  const int G = d.ghost, NI = d.Ni, NJ = d.Nj;
  switch (this_face) {
    case GNORTH: gi += G; gj += NJ - G + 1; break;
    case GEAST: gi += NI - G + 1; gj += G; break;
    case GSOUTH: gi += G; break;
    default: gj += G; break;
  }
  int a1i, a1j, a2i, a2j, b1i, b1j, b2i, b2j;
  face_corners(this_face, NI, NJ, G, a1i, a1j, a2i, a2j);
  if (flip_normal == 1) {
    const int ti = a1i, tj = a1j;
    a1i = a2i; a1j = a2j; a2i = ti; a2j = tj;
  }
  face_corners(that_face, NIB, NJB, G, b1i, b1j, b2i, b2j);
  const V2 A1 = xy_at(xyA, NJ, a1i, a1j), A2 = xy_at(xyA, NJ, a2i, a2j);
  const V2 B1 = xy_at(xyB, NJB, b1i, b1j), B2 = xy_at(xyB, NJB, b2i, b2j);
  const bool misalign = !(fabs(A1.x - B1.x) <= 1e-12) || !(fabs(A1.y - B1.y) <= 1e-12) ||
                        !(fabs(A2.x - B2.x) <= 1e-12) || !(fabs(A2.y - B2.y) <= 1e-12);
  for (int ii = 0; ii < 2; ++ii)
    for (int jj = 0; jj < 2; ++jj) {
      int iB = (int)gi + ii, jB = (int)gj + jj;
      if (misalign && ori == 1) {
        if (this_face == GEAST || this_face == GWEST) jB = NJ - jB;
        else iB = NI - iB;
      }
      swap_vertex_index(NI, NJ, G, this_face, iB, jB, that_face, NIB, NJB);
      if (iB < 0 || iB > NIB || jB < 0 || jB > NJB) continue;  // a connection that does not map
      const V2 p = xy_at(xyB, NJB, iB, jB);
      V2 out;
      if (affine == NO_TRANSFORM) out = p;
      else if (affine == MIRROR) out = mirror_about(A1, A2, p);
      else out = corner_transform(A1, A2, B1, B2, p);
      xy_set(xyA, NJ, gi + ii, gj + jj, out);
    }
}

// xyExtrapolate (clGhostRoutines.c:291-398): ghost vertices continue the
// last interior spacing.  The work items overlap (the first layer rewrites
// the boundary vertices the others read), so one thread walks them in the
// order of a sequential evaluation: the first NDRange index outermost.  It
// is a few hundred vertices per face.
__global__ void k_xyExtrapolate(ugks_block_desc d, size_t g0, size_t g1, double *xy, int this_face) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const int G = d.ghost, NI = d.Ni, NJ = d.Nj;
  auto X = [&](long i, long j) { return xy_at(xy, NJ, i, j); };
  auto add = [](V2 p, V2 q) { return v2(p.x + q.x, p.y + q.y); };
  auto diffm = [](double m, V2 p, V2 q) { return v2(m * (p.x - q.x), m * (p.y - q.y)); };
  for (size_t a = 0; a < g0; ++a)
    for (size_t b = 0; b < g1; ++b) {
      long gi, gj, ei, ej;
      double m;
      V2 d1, d2;
      switch (this_face) {
        case GNORTH:
          gi = (long)a + G; gj = (long)b + NJ - G; ei = gi; ej = NJ - G - 1; m = (double)(gj - ej);
          d1 = diffm(m, X(ei, ej + 1), X(ei, ej));
          d2 = diffm(m, X(ei + 1, ej + 1), X(ei + 1, ej));
          xy_set(xy, NJ, gi, gj, add(X(ei, ej), d1));
          xy_set(xy, NJ, gi + 1, gj, add(X(ei + 1, ej), d2));
          xy_set(xy, NJ, gi + 1, gj + 1, add(X(ei + 1, ej + 1), d2));
          xy_set(xy, NJ, gi, gj + 1, add(X(ei, ej + 1), d1));
          break;
        case GEAST:
          gi = (long)a + NI - G; gj = (long)b + G; ei = NI - G - 1; ej = gj; m = (double)(gi - ei);
          d1 = diffm(m, X(ei + 1, ej), X(ei, ej));
          d2 = diffm(m, X(ei + 1, ej + 1), X(ei, ej + 1));
          xy_set(xy, NJ, gi, gj, add(X(ei, ej), d1));
          xy_set(xy, NJ, gi + 1, gj, add(X(ei + 1, ej), d1));
          xy_set(xy, NJ, gi + 1, gj + 1, add(X(ei + 1, ej + 1), d2));
          xy_set(xy, NJ, gi, gj + 1, add(X(ei, ej + 1), d2));
          break;
        case GSOUTH:
          gi = (long)a + G; gj = (long)b; ei = gi; ej = G; m = (double)(ej - gj);
          d1 = diffm(m, X(ei, ej), X(ei, ej + 1));
          d2 = diffm(m, X(ei + 1, ej), X(ei + 1, ej + 1));
          xy_set(xy, NJ, gi, gj, add(X(ei, ej), d1));
          xy_set(xy, NJ, gi + 1, gj, add(X(ei + 1, ej), d2));
          xy_set(xy, NJ, gi + 1, gj + 1, add(X(ei + 1, ej + 1), d2));
          xy_set(xy, NJ, gi, gj + 1, add(X(ei, ej + 1), d1));
          break;
        default:
          gi = (long)a; gj = (long)b + G; ei = G; ej = gj; m = (double)(ei - gi);
          d1 = diffm(m, X(ei, ej), X(ei + 1, ej));
          d2 = diffm(m, X(ei, ej + 1), X(ei + 1, ej + 1));
          xy_set(xy, NJ, gi, gj, add(X(ei, ej), d1));
          xy_set(xy, NJ, gi + 1, gj, add(X(ei + 1, ej), d1));
          xy_set(xy, NJ, gi + 1, gj + 1, add(X(ei + 1, ej + 1), d2));
          xy_set(xy, NJ, gi, gj + 1, add(X(ei, ej + 1), d2));
          break;
      }
    }
}

// cellGeom (clKernel.c:31-135): normals, area, centroid, mid-sides and side
// lengths of every cell (ghosts included)
__global__ void k_cellGeom(ugks_block_desc d, size_t g0, size_t g1, const double *xy, double *area, double *centre,
                           double *mid_side, double *normal, double *side_length) {
  const size_t w = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (w >= g0 * g1) return;
  const long i = (long)(w / g1), j = (long)(w % g1);
  const int NJ = d.Nj;
  const V2 A = xy_at(xy, NJ, i + 1, j), Bv = xy_at(xy, NJ, i + 1, j + 1), C = xy_at(xy, NJ, i, j + 1),
           Dv = xy_at(xy, NJ, i, j);
  const double xA = A.x, yA = A.y, xB = Bv.x, yB = Bv.y, xC = C.x, yC = C.y, xD = Dv.x, yD = Dv.y;
  const double nSx = -(yA - yD), nSy = xA - xD, nWx = -(yD - yC), nWy = xD - xC;
  const double lS = sqrt(nSx * nSx + nSy * nSy), lW = sqrt(nWx * nWx + nWy * nWy);
  const size_t g = (size_t)i * d.Nj + j;
  st2(normal, 2 * g + SOUTH, v2(nSx / lS, nSy / lS));
  st2(normal, 2 * g + WEST, v2(nWx / lW, nWy / lW));
  const double a = 0.5 * ((xB + xA) * (yB - yA) + (xC + xB) * (yC - yB) + (xD + xC) * (yD - yC) + (xA + xD) * (yA - yD));
  area[g] = a;
  double cx = 1.0 / (a * 6.0) *
              ((yB - yA) * (xA * xA + xA * xB + xB * xB) + (yC - yB) * (xB * xB + xB * xC + xC * xC) +
               (yD - yC) * (xC * xC + xC * xD + xD * xD) + (yA - yD) * (xD * xD + xD * xA + xA * xA));
  if (fabs(cx) > 1.0e6) cx = NAN;
  double cy = -1.0 / (a * 6.0) *
              ((xB - xA) * (yA * yA + yA * yB + yB * yB) + (xC - xB) * (yB * yB + yB * yC + yC * yC) +
               (xD - xC) * (yC * yC + yC * yD + yD * yD) + (xA - xD) * (yD * yD + yD * yA + yA * yA));
  if (fabs(cy) > 1.0e6) cy = NAN;
  st2(centre, g, v2(cx, cy));
  st2(mid_side, 2 * g + SOUTH, v2(0.5 * (xD + xA), 0.5 * (yD + yA)));
  st2(mid_side, 2 * g + WEST, v2(0.5 * (xD + xC), 0.5 * (yD + yC)));
  side_length[2 * g + SOUTH] = sqrt((xD - xA) * (xD - xA) + (yD - yA) * (yD - yA));
  side_length[2 * g + WEST] = sqrt((xC - xD) * (xC - xD) + (yC - yD) * (yC - yD));
}

inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

extern "C" {

int ugks_xyExchange(const ugks_block_desc *d, size_t g0, size_t g1, double *xyA, int this_face, const double *xyB,
                    int NIB, int NJB, int that_face, int ori, int affine, int flip_normal, int this_block_id,
                    int that_block_id, void *stream) {
  (void)this_block_id; (void)that_block_id;
  if (g0 * g1 == 0) return 0;
  k_xyExchange<<<blocks_for(g0 * g1, 128), 128, 0, S(stream)>>>(*d, g0, g1, xyA, this_face, xyB, NIB, NJB,
                                                                  that_face, ori, affine, flip_normal);
  return launch_status();
}

int ugks_xyExtrapolate(const ugks_block_desc *d, size_t g0, size_t g1, double *xy, int this_face, void *stream) {
  if (g0 * g1 == 0) return 0;
  k_xyExtrapolate<<<1, 32, 0, S(stream)>>>(*d, g0, g1, xy, this_face);
  return launch_status();
}

int ugks_cellGeom(const ugks_block_desc *d, size_t g0, size_t g1, const double *xy, double *area, double *centre,
                  double *mid_side, double *normal, double *side_length, void *stream) {
  if (g0 * g1 == 0) return 0;
  k_cellGeom<<<blocks_for(g0 * g1, 128), 128, 0, S(stream)>>>(*d, g0, g1, xy, area, centre, mid_side, normal,
                                                                side_length);
  return launch_status();
}

}  // extern "C"
