// ugks_fused.cu -- the whole UGKS time step in five launches, for every block
// of every solve of a device-resident block table.
//
// Per step (UGKSim.one_step, ugks_sim.py:407-501):
//   face pass   one CTA per face of either direction: reconstruction (iFace),
//               face moments (getFaceCons/getAL/getAR), slopes (getPLR),
//               initMacroFlux, calcFaceQ, macroFlux and distFlux fused, or the
//               wall procedure for wall faces (accommodatingWallDist |
//               adsorbingWall_P1 + adsorbingWallD_P2, then wallFlux and
//               wallMassEnergyFluxes).  The per-velocity interface
//               distribution and slope stay in shared memory between the
//               three velocity sweeps a face needs (moments -> heat flux ->
//               flux), so f is read once per face from HBM/L2.
//   dt check    updateTimeStep inside the dt loop (ugks_sim.py:430-441):
//               device-side, sets the retry flag of a solve whose dt changed.
//   face pass   again, only for solves whose retry flag is set.
//   cell pass   one CTA per cell: calcQ, updateMacro and UGKS_update fused,
//               plus the cell's CFL frequency (clFindDT) and residual terms.
//   dt update   calcTimeStep + updateTimeStep + time advance, device-side.
//   ghost pass  one CTA per ghost cell of every block face (updateBC).
// Nothing reads the host in between, so a step can be captured in a graph.
#include <cuda_runtime.h>
#include <float.h>

#include <algorithm>
#include <mutex>
#include <optional>
#include <type_traits>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "ugks_device.cuh"

using namespace ugks;

namespace {

constexpr int FT = 128;  // threads per face / cell / ghost CTA
// velocities (or pairs) per thread whose loads are in flight together in
// the ghost copies, issued before the first store (a store may alias a later
// load, so the compiler keeps them in program order)
constexpr int GHOST_U = 4;
// face kernels come in two shapes: narrow, FT threads per face at
// FACE_MIN_BLOCKS CTAs per SM (fits while the per-face shared memory allows
// that many), and wide, for larger velocity grids, where shared memory allows
// only 2-3 faces per SM: 384 (FP64) or 256 (FP32) threads per face keep the
// warps per SM up (config-3 batch: face pass 29.6 -> 23.7 ms FP64, 20.1 ->
// 18.1 ms FP32, against 128 threads)
#ifndef FACE_MIN_BLOCKS
#define FACE_MIN_BLOCKS 6
#endif
#ifndef FACE_MIN_BLOCKS_F32
#define FACE_MIN_BLOCKS_F32 5
#endif
#ifndef FACE_MIN_BLOCKS_WIDE
#define FACE_MIN_BLOCKS_WIDE 2
#endif
#ifndef FACE_MIN_BLOCKS_WIDE_F32
#define FACE_MIN_BLOCKS_WIDE_F32 2
#endif
#ifndef FACE_WIDE_THREADS
#define FACE_WIDE_THREADS 384
#endif
#ifndef FACE_WIDE_THREADS_F32
#define FACE_WIDE_THREADS_F32 256
#endif
// per storage type: the narrow and wide register budgets and the largest
// velocity grid of the narrow one (that many face CTAs fit in shared memory:
// FP64 6 x (32 B x 1100 + 3 KB), mixed 5 x (24 B x 1800 + 3 KB) <= 228 KB;
// the mixed kernels' packed-pair arithmetic needs 96 registers to run
// without spilling in its velocity loops)
template <typename T> struct FaceBudget;
template <> struct FaceBudget<double> {
  static constexpr int narrow = FACE_MIN_BLOCKS, wide = FACE_MIN_BLOCKS_WIDE, narrow_max_nv = 1100,
                       wide_threads = FACE_WIDE_THREADS;
};
template <> struct FaceBudget<float> {
  static constexpr int narrow = FACE_MIN_BLOCKS_F32, wide = FACE_MIN_BLOCKS_WIDE_F32, narrow_max_nv = 1800,
                       wide_threads = FACE_WIDE_THREADS_F32;
};
// Launch shapes a face-pass segment can run with (ugks_fused_sizes.seg_variant;
// the tuner in pyugks_b200/tuner.py picks them by timing): variant 0 chooses
// by velocity count (narrow up to FaceBudget::narrow_max_nv, wide above),
// 1..4 force (threads per face CTA, CTAs per SM of the register budget):
//   FP64  1 = 128 x 6 (narrow), 2 = 128 x 5, 3 = 256 x 3, 4 = 384 x 2 (wide)
//   mixed 1 = 128 x 5 (narrow), 2 = 128 x 4, 3 = 256 x 3, 4 = 256 x 2 (wide)
template <typename T, int V> struct FaceShape;
template <> struct FaceShape<double, 1> { static constexpr int nt = 128, minb = 6; };
template <> struct FaceShape<double, 2> { static constexpr int nt = 128, minb = 5; };
template <> struct FaceShape<double, 3> { static constexpr int nt = 256, minb = 3; };
template <> struct FaceShape<double, 4> { static constexpr int nt = 384, minb = 2; };
template <> struct FaceShape<float, 1> { static constexpr int nt = 128, minb = 5; };
template <> struct FaceShape<float, 2> { static constexpr int nt = 128, minb = 4; };
template <> struct FaceShape<float, 3> { static constexpr int nt = 256, minb = 3; };
template <> struct FaceShape<float, 4> { static constexpr int nt = 256, minb = 2; };
// launch shapes of the mixed moments sweep (a face per warp): warps per CTA x
// CTAs per SM
template <int V> struct MomentsShape;
template <> struct MomentsShape<1> { static constexpr int wpc = 4, minb = 5; };
template <> struct MomentsShape<2> { static constexpr int wpc = 4, minb = 4; };
template <> struct MomentsShape<3> { static constexpr int wpc = 8, minb = 3; };
template <> struct MomentsShape<4> { static constexpr int wpc = 4, minb = 6; };
// and of the mixed flux sweep
// 7 CTAs (28 warps) per SM at 72 registers: 0.617 -> 0.598 ms of face pass on
// the 2x2-block cavity, 13.0 -> 12.2 ms on the 64-solve batch, against 5
#ifndef UGKS_FLUX_MINB
#define UGKS_FLUX_MINB 7
#endif
constexpr int FLUX_WPC = 4, FLUX_MINB = UGKS_FLUX_MINB;
// the flux sweep with bulk-copied rows (face_flux_tma) instead of per-lane
// loads: 0.598 -> 0.529 ms of face pass on the 2x2-block cavity (the sweep
// itself 252 -> 169 us under ncu, DRAM 42% -> 62% of peak)
#ifndef UGKS_FLUX_TMA
#define UGKS_FLUX_TMA 1
#endif
#ifndef UGKS_FLUX_TMA_MINB
#define UGKS_FLUX_TMA_MINB 5
#endif
constexpr int FLUX_TMA_MINB = UGKS_FLUX_TMA_MINB;
static_assert(FaceShape<double, 1>::minb == FACE_MIN_BLOCKS && FaceShape<double, 4>::nt == FACE_WIDE_THREADS &&
                  FaceShape<float, 1>::minb == FACE_MIN_BLOCKS_F32 && FaceShape<float, 4>::minb == FACE_MIN_BLOCKS_WIDE_F32,
              "variants 1 and 4 are the narrow and wide default shapes");

// CTAs of 8 cell warps per SM: FP64 at 128 registers (at 80 the update loop
// spills and the pass is 12% slower), mixed at 80 (3 CTAs: 0.215 against
// 0.222 ms at 120 registers on the 2x2-block cavity)
#ifndef CELL_MIN_BLOCKS
#define CELL_MIN_BLOCKS 2
#endif
#ifndef CELL_MIN_BLOCKS_F32
#define CELL_MIN_BLOCKS_F32 3
#endif
// ...and the depth of the per-warp ring of asynchronous copies that stream
// the f and flux rows of the cell update into shared memory
// (FP64 only: with 8-byte FP32 elements the ring was 18% slower than plain loads)
#ifndef CELL_RING_F64
#define CELL_RING_F64 3
#endif
template <typename T> struct CellBudget { static constexpr int minb = CELL_MIN_BLOCKS, ring = CELL_RING_F64; };
template <> struct CellBudget<float> { static constexpr int minb = CELL_MIN_BLOCKS_F32, ring = 0; };
// shared memory of the cell-update ring: per warp, ring stages x 5 rows
// (f, S face j, S face j+1, W face i, W face i+1) x 32 lanes
template <typename T>
constexpr size_t cell_ring_bytes() {
  return (size_t)CellBudget<T>::ring * 5 * 32 * sizeof(typename Store<T>::vec);
}

// cp.async (sm_80+ asynchronous global -> shared copy of 8 or 16 bytes per
// thread; a thread waits only for its own groups)
template <int BYTES>
__device__ __forceinline__ void cp_async(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }
inline int launch_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -(int)e;
}

// block of work item w: the last block whose begin <= w (begins are ascending)
template <int WHICH>
__device__ __forceinline__ int find_block(const ugks_fused_block *B, int nb, int w) {
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    int beg = WHICH == 0 ? B[mid].face_begin
                         : (WHICH == 1 ? B[mid].cell_begin : (WHICH == 2 ? B[mid].ghost_begin : B[mid].wall_begin));
    if (beg <= w) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ bool is_wall(int bc) { return bc == BC_DIFFUSE || bc == BC_ADSORBING; }

// UGKS_CHECKED builds (python -m pyugks_b200.build --checked): every work
// item is checked against the block it was found in -- inside the block's
// range of items, and the block's sizes consistent with its ghost layers and
// its limiter's stencil -- and an item that fails (a table corrupted on the
// device after ugks_fused_layout validated it) flags its solve with status 9
// and is skipped instead of indexing outside the block's arrays.
#ifndef UGKS_CHECKED
#define UGKS_CHECKED 0
#endif
constexpr int STATUS_INDEX_CHECK = 9;
template <int WHICH>
__device__ __forceinline__ bool item_in_block(const ugks_fused_block &b, int w) {
  const ugks_block_desc &d = b.d;
  long begin = 0, count = 0;
  if (WHICH == 0) { begin = b.face_begin; count = 2l * (d.ni + 1) * (d.nj + 1); }
  if (WHICH == 1) { begin = b.cell_begin; count = (long)d.ni * d.nj; }
  if (WHICH == 2) { begin = b.ghost_begin; count = 2l * d.ghost * (d.ni + d.nj); }
  if (WHICH == 3) { begin = b.wall_begin; count = 2l * (d.ni + d.nj); }
  return w >= begin && w < begin + count && d.ghost >= (d.flux_method == 1 ? 3 : 2) &&
         d.Ni == d.ni + 2 * d.ghost && d.Nj == d.nj + 2 * d.ghost;
}
#define UGKS_CHECK_ITEM(WHICH, blk, w, solves, ...)                                                       \
  do {                                                                                                     \
    if (UGKS_CHECKED && !item_in_block<WHICH>((blk), (w))) {                                               \
      atomicExch(const_cast<int *>(&(solves)[(blk).solve].status), STATUS_INDEX_CHECK);                     \
      return __VA_ARGS__;                                                                                  \
    }                                                                                                      \
  } while (0)

// dt update of updateTimeStep (ugks_sim.py:285-311) with limit = True
__device__ __forceinline__ double limited_dt(double dt_old, double dt_new, double delta) {
  if (dt_old != dt_new) {
    if (dt_new > (1.0 + delta) * dt_old) dt_new = (1.0 + delta) * dt_old;
    return dt_new;
  }
  return dt_old;
}

// ---------------------------------------------------------------------------
// face pass
// ---------------------------------------------------------------------------
// The per-face and per-cell coefficient helpers below restate getPrimary,
// microSlope, momentU, relaxTime and the time weights (clUGKS.c:16-80,
// 497-503, clFunctions.c:8-32) with every division by rho, lambda, tau or a
// constant replaced by one Newton-Raphson reciprocal (nr_rcp) and products:
// branch-free, so the independent chains of a face overlap.  Results differ
// from the dividing forms by a few ulp.
struct Rcp {
  double rho, lam;  // 1/rho, 1/lambda
};

__device__ __forceinline__ P4 to_primary_rcp(const ugks_block_desc &d, P4 w, Rcp &r) {
  const double r0 = nr_rcp(w.s0);
  P4 p = w;
  p.s1 = w.s1 * r0;
  p.s2 = w.s2 * r0;
  const double e = w.s3 - 0.5 * (w.s1 * w.s1 + w.s2 * w.s2) * r0;
  p.s3 = (0.5 * w.s0) * nr_rcp((d.gam - 1.0) * e);
  r.rho = r0;
  r.lam = nr_rcp(p.s3);
  return p;
}

__device__ __forceinline__ P4 micro_slope_rcp(double K, P4 prim, Rcp r, P4 sw) {
  const double k2 = 0.5 * (K + 2.0) * r.lam;  // (K + 2) / (2 lambda)
  const double c3 = 4.0 * (prim.s3 * prim.s3) * nr_rcp(K + 2.0) * r.rho;
  const double cl = 2.0 * prim.s3 * r.rho;
  const double uv2 = prim.s1 * prim.s1 + prim.s2 * prim.s2;
  P4 a;
  a.s3 = c3 * (2.0 * sw.s3 - 2.0 * prim.s1 * sw.s1 - 2.0 * prim.s2 * sw.s2 + sw.s0 * (uv2 - k2));
  a.s2 = cl * (sw.s2 - prim.s2 * sw.s0) - prim.s2 * a.s3;
  a.s1 = cl * (sw.s1 - prim.s1 * sw.s0) - prim.s1 * a.s3;
  a.s0 = sw.s0 * r.rho - prim.s1 * a.s1 - prim.s2 * a.s2 - 0.5 * (uv2 + k2) * a.s3;
  return a;
}

// momentU (clUGKS.c:47-80) over one half range: sg = +1 gives the moments
// <u^k> over u > 0 (MuL), sg = -1 those over u < 0 (MuR); Mv and Mxi are the
// full-range moments of v and xi.  The two halves are the same instruction
// stream with the sign flipped, so two lanes compute them side by side.
__device__ __forceinline__ void half_moments_rcp(double PI, double K, P4 prim, Rcp r, double sg,
                                                 double Mh[MNUM], double Mv[MTUM], double Mxi[3]) {
  const double sl = sqrt(prim.s3);
  const double g = 0.5 * exp(-prim.s3 * (prim.s1 * prim.s1)) * nr_rcp(sqrt(PI * prim.s3));
  const double hl = 0.5 * r.lam;
  Mh[0] = 0.5 * erfc((-sg * sl) * prim.s1);
  Mh[1] = prim.s1 * Mh[0] + sg * g;
#pragma unroll
  for (int i = 2; i < MNUM; ++i) Mh[i] = prim.s1 * Mh[i - 1] + ((i - 1) * hl) * Mh[i - 2];
  Mv[0] = 1.0;
  Mv[1] = prim.s2;
#pragma unroll
  for (int i = 2; i < MTUM; ++i) Mv[i] = prim.s2 * Mv[i - 1] + ((i - 1) * hl) * Mv[i - 2];
  Mxi[0] = 1.0;
  Mxi[1] = K * hl;
  Mxi[2] = (K * K + 2.0 * K) * (hl * hl);
}

// named barrier 1 between warp 0 (waits) and warp 1 (arrives): whole warps
__device__ __forceinline__ void pair_wait() {
  __syncwarp();
  asm volatile("bar.sync 1, 64;" ::: "memory");
}
__device__ __forceinline__ void pair_arrive() {
  __syncwarp();
  asm volatile("bar.arrive 1, 64;" ::: "memory");
}

// 1 / relaxTime
__device__ __forceinline__ double inv_relax_time_rcp(const ugks_block_desc &d, P4 prim, Rcp r) {
  const double p = pow(prim.s3, 1.0 - d.omega);
  double c = 1.0;
  switch (d.relax_type) {
    case 0: c = 0.79788456080286541; break;
    case 1: c = (5. / 8.) * sqrt(d.PI); break;
    case 3: c = 2.2567583341910251; break;
    default: break;
  }
  return nr_rcp((d.Kn_eff * r.rho) * c * p);
}

__device__ __forceinline__ void time_weights_rcp(double inv_tau, double dt, double Mt[5]) {
  const double tau = nr_rcp(inv_tau);
  const double e = exp(-dt * inv_tau);
  Mt[3] = tau * (1.0 - e);
  Mt[4] = -tau * dt * e + tau * Mt[3];
  Mt[0] = dt - Mt[3];
  Mt[1] = -tau * Mt[0] + Mt[4];
  Mt[2] = 0.5 * (dt * dt) - tau * Mt[0];
}

template <int NT>
struct FaceShared {
  double scratch[16 * (NT / 32)];
  double bcast[48];
  double nbr[2][5];  // left / right cell: rho, u, v (face frame), lambda, 1/|mid - centre|
  double lr[2][19];  // per side: half-range Mu [7], slope a [4], <a u psi> [4], <a u^2 psi> [4]
  double mt[5];      // time weights
};

// WENO5 (clFunctions.c:266-313) of one component, up to the final division:
// slope * dx = num / den.  Written in the first differences D_k = S_{k+1} - S_k:
//   12 beta_k = 13 (D_{k+1} - D_k)^2 + 3 r_k^2,  r = (3 D1 - D0, D1 + D2, D3 - 3 D2)
//   f_k - S2  = (-D0/3 + 5 D1/6, D1/6 + D2/3, 2 D2/3 - D3/6)
// and the weights c_k / (eps + beta_k)^2 multiplied through by
// prod_j (eps + beta_j)^2 / 0.1 (a common factor of num and den; eps scales
// with beta).
__device__ __forceinline__ void weno5_part(const double (&S)[5], double &num, double &den) {
  const double D0 = S[1] - S[0], D1 = S[2] - S[1], D2 = S[3] - S[2], D3 = S[4] - S[3];
  const double p0 = D1 - D0, p1 = D2 - D1, p2 = D3 - D2;
  const double r0 = fma(3.0, D1, -D0), r1 = D1 + D2, r2 = fma(-3.0, D2, D3);
  const double e0 = 12e-16 + fma(13.0 * p0, p0, (3.0 * r0) * r0);
  const double e1 = 12e-16 + fma(13.0 * p1, p1, (3.0 * r1) * r1);
  const double e2 = 12e-16 + fma(13.0 * p2, p2, (3.0 * r2) * r2);
  const double q0 = e0 * e0, q1 = e1 * e1, q2 = e2 * e2;
  const double a0 = q1 * q2, a1 = 6.0 * (q0 * q2), a2 = 3.0 * (q0 * q1);
  const double f0 = fma(-1.0 / 3.0, D0, (5.0 / 6.0) * D1);
  const double f1 = fma(1.0 / 6.0, D1, (1.0 / 3.0) * D2);
  const double f2 = fma(2.0 / 3.0, D2, (-1.0 / 6.0) * D3);
  num = fma(a0, f0, fma(a1, f1, a2 * f2));
  den = (a0 + a1) + a2;
}

// iFace (clUGKS.c:148-194) for one velocity: face value and slope of (h, b).
// The two components share one reciprocal: 1/x = y * 1/(x y).
// The stencil runs upwind to downwind: cells MID+1 .. 1 before the face and
// 0 .. L-MID-2 after it for u > 0, mirrored for u <= 0; `p` points at stencil
// cell 0 and `st` is the signed cell stride in (h, b) pairs.
template <typename T, int FM>
__device__ __forceinline__ void reconstruct(const typename Store<T>::vec *p, int st, double inv_l,
                                            double ds, double inv_ds, double &fh, double &fb,
                                            double &sh, double &sb) {
  constexpr int L = FM == 1 ? 5 : 3, MID = FM == 1 ? 2 : 1;
  double Sh[L], Sb[L];
#pragma unroll
  for (int s = 0; s < L; ++s) {
    const auto x = p[s * st];
    Sh[s] = (double)x.x;
    Sb[s] = (double)x.y;
  }
  if constexpr (FM == 0) {
    // vanLeer (clFunctions.c:255-261)
    const double h1 = (Sh[1] - Sh[0]) * inv_l, h2 = (Sh[2] - Sh[1]) * inv_l;
    const double b1 = (Sb[1] - Sb[0]) * inv_l, b2 = (Sb[2] - Sb[1]) * inv_l;
    const double dh = fabs(h1) + fabs(h2) + 1e-16, db = fabs(b1) + fabs(b2) + 1e-16;
    const double r = nr_rcp(dh * db);
    sh = (ocl_sign(h1) + ocl_sign(h2)) * (fabs(h1) * fabs(h2)) * (db * r);
    sb = (ocl_sign(b1) + ocl_sign(b2)) * (fabs(b1) * fabs(b2)) * (dh * r);
  } else if constexpr (FM == 1) {
    double nh, dh, nb, db;
    weno5_part(Sh, nh, dh);
    weno5_part(Sb, nb, db);
    const double r = nr_rcp(dh * db) * inv_ds;
    sh = nh * (db * r);
    sb = nb * (dh * r);
  } else {
    sh = (0.5 * minmod(Sh[2] - Sh[1], Sh[1] - Sh[0])) * inv_ds;
    sb = (0.5 * minmod(Sb[2] - Sb[1], Sb[1] - Sb[0])) * inv_ds;
  }
  fh = Sh[MID] + sh * ds;
  fb = Sb[MID] + sb * ds;
}

// The FP32 flux path (FP32 storage of h and b): the same reconstructions in
// single precision.  WENO5 keeps the difference form above, with the three
// smoothness terms e_k (>= 12e-16) divided by their sum before the products:
// the weights only enter as ratios, the largest scaled e_k is >= 1/3 and the
// smallest >= 1e-17, so the weight of the smoothest stencil stays a normal
// FP32 number (>= 1e-35) while only negligible weights can underflow.
// 1 / x by the hardware's approximate reciprocal (rcp.approx.ftz.f32, within
// about an ulp; denormal results flush to zero): the FP32 limiter and WENO5
// weights divide only by sums that are at least 1e-16 or normalised to 1
#ifndef UGKS_FRCP_APPROX
#define UGKS_FRCP_APPROX 1
#endif
__device__ __forceinline__ float frcp(float x) {
#if UGKS_FRCP_APPROX
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
#else
  return __fdividef(1.0f, x);
#endif
}
__device__ __forceinline__ float fsign(float a) {
  return a > 0.0f ? 1.0f : (a < 0.0f ? -1.0f : (a == 0.0f ? a : 0.0f));
}
__device__ __forceinline__ float fminmod(float a, float b) {
  float out = 0.0f;
  if ((fabsf(a) < fabsf(b)) && (a * b > 0.0f)) out = a;
  else if ((fabsf(b) < fabsf(a)) && (a * b > 0.0f)) out = b;
  else if (a == b) out = a;
  return out;
}
__device__ __forceinline__ void weno5_part_f(const float (&S)[5], float &num, float &den) {
  const float D0 = S[1] - S[0], D1 = S[2] - S[1], D2 = S[3] - S[2], D3 = S[4] - S[3];
  const float p0 = D1 - D0, p1 = D2 - D1, p2 = D3 - D2;
  const float r0 = fmaf(3.0f, D1, -D0), r1 = D1 + D2, r2 = fmaf(-3.0f, D2, D3);
  float e0 = 12e-16f + fmaf(13.0f * p0, p0, (3.0f * r0) * r0);
  float e1 = 12e-16f + fmaf(13.0f * p1, p1, (3.0f * r1) * r1);
  float e2 = 12e-16f + fmaf(13.0f * p2, p2, (3.0f * r2) * r2);
  const float sc = frcp((e0 + e1) + e2);
  e0 *= sc;
  e1 *= sc;
  e2 *= sc;
  const float q0 = e0 * e0, q1 = e1 * e1, q2 = e2 * e2;
  const float a0 = q1 * q2, a1 = 6.0f * (q0 * q2), a2 = 3.0f * (q0 * q1);
  const float f0 = fmaf(-1.0f / 3.0f, D0, (5.0f / 6.0f) * D1);
  const float f1 = fmaf(1.0f / 6.0f, D1, (1.0f / 3.0f) * D2);
  const float f2 = fmaf(2.0f / 3.0f, D2, (-1.0f / 6.0f) * D3);
  num = fmaf(a0, f0, fmaf(a1, f1, a2 * f2));
  den = (a0 + a1) + a2;
}
template <int L, typename VEC>
__device__ __forceinline__ void load_stencil(const VEC *p, int st, VEC (&x)[L]) {
#pragma unroll
  for (int s = 0; s < L; ++s) x[s] = p[s * st];
}
template <int FM>
__device__ __forceinline__ void reconstruct_f(const float2 (&xs)[FM == 1 ? 5 : 3], float inv_l, float ds, float inv_ds,
                                              float &fh, float &fb, float &sh, float &sb) {
  constexpr int L = FM == 1 ? 5 : 3, MID = FM == 1 ? 2 : 1;
  float Sh[L], Sb[L];
#pragma unroll
  for (int s = 0; s < L; ++s) {
    const float2 x = xs[s];
    Sh[s] = x.x;
    Sb[s] = x.y;
  }
  if constexpr (FM == 0) {
    const float h1 = (Sh[1] - Sh[0]) * inv_l, h2 = (Sh[2] - Sh[1]) * inv_l;
    const float b1 = (Sb[1] - Sb[0]) * inv_l, b2 = (Sb[2] - Sb[1]) * inv_l;
    sh = (fsign(h1) + fsign(h2)) * (fabsf(h1) * fabsf(h2)) * frcp(fabsf(h1) + fabsf(h2) + 1e-16f);
    sb = (fsign(b1) + fsign(b2)) * (fabsf(b1) * fabsf(b2)) * frcp(fabsf(b1) + fabsf(b2) + 1e-16f);
  } else if constexpr (FM == 1) {
    float nh, dh, nb, db;
    weno5_part_f(Sh, nh, dh);
    weno5_part_f(Sb, nb, db);
    sh = nh * frcp(dh) * inv_ds;
    sb = nb * frcp(db) * inv_ds;
  } else {
    sh = (0.5f * fminmod(Sh[2] - Sh[1], Sh[1] - Sh[0])) * inv_ds;
    sb = (0.5f * fminmod(Sb[2] - Sb[1], Sb[1] - Sb[0])) * inv_ds;
  }
  fh = fmaf(sh, ds, Sh[MID]);
  fb = fmaf(sb, ds, Sb[MID]);
}

// scale * exp(-lambda (x - c)^2) over the nodes of one velocity axis
template <typename R>
__device__ __forceinline__ void axis_exp(R *out, const double *quad, int n, int stride,
                                         int comp, double c, double lambda, int t, int nt,
                                         double scale = 1.0) {
  for (int i = t; i < n; i += nt) {
    const double x = quad[2 * (size_t)i * stride + comp] - c;
    out[i] = (R)(scale * exp(-lambda * (x * x)));
  }
}

// stencil geometry of a face for both upwind directions (iFace,
// clUGKS.c:148-176): |mid - c|, 1/|mid - c| and 1/|c - c'| with c, c' the
// cells MID and MID-1 from the face (u <= 0), then the cells before the face
// (u > 0)
__device__ __forceinline__ void stencil_geometry(const ugks_fused_block &blk, long gi, long gj, int dir, V2 mid,
                                                 double *out) {
  const ugks_block_desc &d = blk.d;
  auto geo = [&](long c0, long c1, double *o) {
    const long c0i = dir == SOUTH ? gi : gi + c0, c0j = dir == SOUTH ? gj + c0 : gj;
    const long c1i = dir == SOUTH ? gi : gi + c1, c1j = dir == SOUTH ? gj + c1 : gj;
    const V2 a = ld2(blk.centre, gidx(d, c0i, c0j)), b = ld2(blk.centre, gidx(d, c1i, c1j));
    o[0] = sqrt((mid.x - a.x) * (mid.x - a.x) + (mid.y - a.y) * (mid.y - a.y));
    o[1] = 1.0 / o[0];
    o[2] = 1.0 / sqrt((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y));
  };
  geo(0, 1, out);        // u <= 0
  geo(-1, -2, out + 3);  // u > 0
}

// the same for every face, once at set-up (read by the FP64 face pass)
__global__ void face_geometry(const ugks_fused_block *__restrict__ B, int nb, int n_faces) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_faces) return;
  const int bi = find_block<0>(B, nb, w);
  const ugks_fused_block &blk = B[bi];
  const ugks_block_desc &d = blk.d;
  int lf = w - blk.face_begin;
  const int dir = lf & 1;
  lf >>= 1;
  const int mi = lf / (d.nj + 1), mj = lf % (d.nj + 1);
  if (dir == SOUTH ? (mi >= d.ni) : (mj >= d.nj)) return;
  const long gi = mi + d.ghost, gj = mj + d.ghost;
  stencil_geometry(blk, gi, gj, dir, ld2(blk.mid_side, faceidx(d, gi, gj, dir)),
                   blk.face_geo + 6 * faceidx(d, gi, gj, dir));
}

// block_sum whose result only thread 0 needs
template <int N>
__device__ __forceinline__ void block_sum_to0(double (&x)[N], double *scratch) {
#pragma unroll
  for (int k = 0; k < N; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x[k] += __shfl_xor_sync(0xffffffffu, x[k], o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) scratch[k * nw + warp] = x[k];
  }
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

// The wall procedure of one wall face (all threads of the CTA take part):
// accommodatingWallDist (clUGKS.c:774-906) or adsorbingWall_P1 (clAdsorb.c:253-482)
// followed by the re-emission stage (adsorbingWallD_P2 / S_P2 / CL_P2,
// clAdsorb.c:488-975), then wallFlux (clUGKS.c:910-1011) and
// wallMassEnergyFluxes (1019-1147).  fw holds the reconstructed face
// distribution (h, b) per velocity in FP64 and is rewritten in place; rin is
// shared scratch of Nv (h, b) pairs (double2, or float2 in the mixed path) for
// the reflected incoming distribution; store_flux(v, h, b) writes the
// face-flux row of velocity v.
template <int NT, typename RIN, typename StoreFlux>
__device__ __forceinline__ void wall_face(const ugks_fused_block &blk, ugks_solve_state &sol, FaceShared<NT> &sh,
                                          double *fw, RIN *rin, const int wall, const int dir, const long gi,
                                          const long gj, const long mi, const long mj, const V2 n, const double len,
                                          const double dt, StoreFlux store_flux) {
  using R = double;
  const ugks_block_desc &d = blk.d;
  const int Nv = d.Nv;
  const double2 *__restrict__ qd = reinterpret_cast<const double2 *>(d.quad);
  const double *__restrict__ wt = d.weight;
  auto fvel = [&](int vv) {
    const double2 e = qd[vv];
    return v2(e.x * n.x + e.y * n.y, e.x * (-n.y) + e.y * n.x);
  };
  const int rot = (wall == GNORTH || wall == GEAST) ? -1 : 1;
  const long ci = dir == SOUTH ? mi : mj;
  P4 wl = ld4(blk.wall_prop, ci * 4 + wall);
  {
    const V2 t = to_local(v2(wl.s1, wl.s2), n);
    wl.s1 = t.x;
    wl.s2 = t.y;
  }
  __syncthreads();
  if (blk.bc_type[wall] == BC_DIFFUSE) {
    // accommodatingWallDist (clUGKS.c:774-906)
    double s[2] = {0.0, 0.0};
    for (int v = threadIdx.x; v < Nv; v += NT) {
      const V2 uv = fvel(v);
      const int delta = upwind_flag(uv.x, rot);
      s[0] += uv.x * (1 - delta) * fw[2 * v];
      s[1] -= uv.x * delta * maxwellian(d, wl, uv, v).x;
    }
    block_sum<2>(s, sh.scratch);
    const double ratio = s[0] / s[1];
    for (int v = threadIdx.x; v < Nv; v += NT) {
      const V2 uv = fvel(v);
      const int delta = upwind_flag(uv.x, rot);
      const V2 M = maxwellian(d, wl, uv, v);
      fw[2 * v] = (R)(ratio * delta * M.x + (1 - delta) * fw[2 * v]);
      fw[2 * v + 1] = (R)(ratio * delta * M.y + (1 - delta) * fw[2 * v + 1]);
    }
  } else {
    // adsorbingWall_P1 (clAdsorb.c:253-482)
    const long ti = dir == SOUTH ? mi : (wall == GEAST ? d.ni - 1 : 0);
    const long tj = dir == SOUTH ? (wall == GNORTH ? d.nj - 1 : 0) : mj;
    const double Tw = 1.0 / blk.macro[4 * midx(d, ti, tj) + 3], Dw = blk.macro[4 * midx(d, ti, tj)];
    double *cover = blk.wall_cover + 4 * (ci * 4 + wall);
    const double theta = cover[0];
    const double gf = d.gamma_f[wall];
    double s[3] = {0.0, 0.0, 0.0};
    for (int v = threadIdx.x; v < Nv; v += NT) {
      const V2 uv = fvel(v);
      const int delta = upwind_flag(uv.x, rot);
      const double k = -rot * uv.x * (1 - delta);
      const V2 total = v2(k * fw[2 * v], k * fw[2 * v + 1]);
      const double beta = sticking(d, uv, Tw, wall);
      V2 ads = v2(beta * total.x * gf * (1.0 - theta), beta * total.y * gf * (1.0 - theta));
      const double fs = ocl_sign(total.x);
      if ((fs * ads.x) > (fs * total.x)) ads = total;
      const V2 refl = v2(total.x - ads.x, total.y - ads.y);
      s[0] += refl.x;
      s[1] += ads.x;
      s[2] += beta * total.x;
      st2(blk.wall_dist, (size_t)ci * Nv + v, v2(refl.x / uv.x, refl.y / uv.x));
    }
    block_sum<3>(s, sh.scratch);
    if (threadIdx.x == 0) {
      double ads_final = s[1], dvt = 0.0, des = 0.0;
      bool ok = true;
      if (gf > 0.0) {
        if (d.dynamic[wall] == 1) {
          dvt = dt * d.alpha_p[wall] * s[1];
          if (dvt > (1 - theta)) {
            dvt = 1 - theta;
            ads_final = dvt / dt * d.alpha_p[wall];  // the reference's form (clAdsorb.c:420)
          }
        }
        if (d.k_des[wall] > 0.0) {
          des = d.k_des[wall] * theta / d.alpha_p[wall];
        } else {
          const V2 veq = vartheta_langmuir(d, Dw, Tw, wall);
          if (veq.y == 1.0) {
            atomicExch(&sol.status, 4);  // outside the tabulated isotherm
            ok = false;
          } else {
            des = gf * (1.0 / veq.x - 1.0) * s[2] * theta;
          }
        }
        if (ok) {
          if (d.dynamic[wall] == 1) {
            dvt -= dt * d.alpha_p[wall] * des;
            if ((theta + dvt) < 0.0) des = theta / (dt * d.alpha_p[wall]);
          }
        }
      }
      double corr = 1.0;
      if (ok) {
        const double refl_final = s[0] + s[1] - ads_final;
        corr = refl_final / s[0];
        cover[0] += dvt;
        cover[1] = refl_final;
        cover[2] = ads_final;
        cover[3] = des;
      }
      sh.bcast[0] = corr;
      sh.bcast[1] = ok ? 1.0 : 0.0;
    }
    __syncthreads();
    const double corr = sh.bcast[0];
    const bool ok = sh.bcast[1] != 0.0;
    if (corr != 1.0)
      for (int v = threadIdx.x; v < Nv; v += NT) {
        const size_t k = (size_t)ci * Nv + v;
        const V2 x = ld2(blk.wall_dist, k);
        st2(blk.wall_dist, k, v2(x.x * corr, x.y * corr));
      }
    if (!ok) {
      // the reference skips the rest of this wall face and carries on
      // (ugks_block.py:949-950, 1084): its flux row keeps what iFace wrote
      // there, the face values of (h, b), and its face macro flux is not
      // written this step
      for (int v = threadIdx.x; v < Nv; v += NT) store_flux(v, fw[2 * v], fw[2 * v + 1]);
      return;
    }
    // re-emission of the reflected flux: adsorbingWallD_P2 (clAdsorb.c:821-975,
    // diffuse), adsorbingWallS_P2 (656-816, specular) or adsorbingWallCL_P2
    // (488-651, Cercignani-Lampis)
    const double refl = cover[1], des = cover[3], ads = cover[2];
    const int kind = d.reflect[wall];
    double ratio = 1.0;
    if (refl > 0.0) {
      // the reflected incoming distribution (wall_dist) of every velocity,
      // staged in the slope buffer, which wall faces do not use
      __syncthreads();
      if (kind != UGKS_REFLECT_DIFFUSE)
        for (int v = threadIdx.x; v < Nv; v += NT) {
          const V2 x = ld2(blk.wall_dist, (size_t)ci * Nv + v);
          rin[v].x = x.x;
          rin[v].y = x.y;
        }
      __syncthreads();
      const double an = d.alpha_n[wall], at = d.alpha_t[wall], Tw = 1.0 / wl.s3;
      double r[1] = {0.0};
      for (int v = threadIdx.x; v < Nv; v += NT) {
        const V2 uv = fvel(v);
        const int delta = upwind_flag(uv.x, rot);
        V2 out = v2(0.0, 0.0);
        if (delta) {
          if (kind == UGKS_REFLECT_DIFFUSE) {
            out = maxwellian(d, wl, uv, v);
          } else if (kind == UGKS_REFLECT_CL) {
            for (int va = 0; va < Nv; ++va) {
              const V2 uv_in = fvel(va);
              if (!upwind_flag(uv_in.x, rot) && uv_in.x != 0.0) {
                const auto fi = rin[va];
                const V2 c = cercignani_lampis(d.PI, uv_in, uv, v2(fi.x, fi.y), an, at, Tw, wl.s3);
                out.x += c.x;
                out.y += c.y;
              }
            }
            out.x *= wt[v];
            out.y *= wt[v];
          } else {
            const auto x = rin[dir == WEST ? d.mirror_EW[v] : d.mirror_NS[v]];
            out = v2(x.x, x.y);
          }
        }
        fw[2 * v] = (R)(delta * out.x + (1 - delta) * fw[2 * v]);
        fw[2 * v + 1] = (R)(delta * out.y + (1 - delta) * fw[2 * v + 1]);
        r[0] += rot * uv.x * out.x;
      }
      block_sum<1>(r, sh.scratch);
      ratio = refl / r[0];
    }
    const int account = ((des == 0.0) && (ads > 0.0) && (refl == 0.0)) ? 1 : 0;
    P4 wd = wl;
    wd.s0 = 2 * des * sqrt(d.PI * wl.s3);
    for (int v = threadIdx.x; v < Nv; v += NT) {
      const V2 uv = fvel(v);
      const int delta = upwind_flag(uv.x, rot);
      const double sc = 1 - delta * (1 - ratio);
      double x = fw[2 * v] * sc, y = fw[2 * v + 1] * sc;
      const V2 M = maxwellian(d, wd, uv, v);
      x += delta * M.x;
      y += delta * M.y;
      x -= account * delta * x;
      y -= account * delta * y;
      fw[2 * v] = (R)x;
      fw[2 * v + 1] = (R)y;
    }
  }
  // wallFlux (clUGKS.c:910-1011) and wallMassEnergyFluxes (1019-1147)
  double s[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) s[k] = 0.0;
  for (int v = threadIdx.x; v < Nv; v += NT) {
    const V2 uv = fvel(v);
    const double wh = fw[2 * v], wb = fw[2 * v + 1];
    const double oh = uv.x * wh * len * dt, ob = uv.x * wb * len * dt;
    store_flux(v, oh, ob);
    const double uu = uv.x * uv.x + uv.y * uv.y;
    s[0] += uv.x * wh;
    s[1] += uv.x * uv.x * wh;
    s[2] += uv.x * uv.y * wh;
    s[3] += 0.5 * uv.x * (uu * wh + wb);
    const int delta = upwind_flag(uv.x, rot);
    const double ix = (1 - delta) * oh, iy = (1 - delta) * ob, ox = delta * oh, oy = delta * ob;
    s[4] += ix; s[5] += uv.x * ix; s[6] += uv.y * ix; s[7] += 0.5 * (uu * ix + iy);
    s[8] += ox; s[9] += uv.x * ox; s[10] += uv.y * ox; s[11] += 0.5 * (uu * ox + oy);
  }
  block_sum<12>(s, sh.scratch);
  if (threadIdx.x == 0) {
    const V2 g = to_global(v2(s[1], s[2]), n);
    st4(dir == SOUTH ? blk.flux_macro_S : blk.flux_macro_W, gidx(d, gi, gj),
        scale(dt * len, p4(s[0], g.x, g.y, s[3])));
    double *wf = blk.wall_fluxes + 8 * (ci * 4 + wall);
    wf[0] = -rot * s[4]; wf[1] = rot * s[8]; wf[2] = -rot * s[5]; wf[3] = rot * s[9];
    wf[4] = -rot * s[6]; wf[5] = rot * s[10]; wf[6] = -rot * s[7]; wf[7] = rot * s[11];
  }
}

// Per-face coefficient block of an interior face, called by every thread of
// the face CTA once W, prim and the neighbour cells (sh.nbr) are in place:
// getPLR slopes (clUGKS.c:424-436) and initMacroFlux (446-518) split over
// lanes 0 / 1 of warp 0 (one per side, the same instructions with one sign
// flipped) while lane 0 of warp 1 computes the time weights and hands them
// over through named barrier 1; the threads from warp 1 on run
// meanwhile(t, nt) (item t of nt) in the meantime.  Leaves in sh.bcast:
//   [0..4] / [5..9] distFlux coefficients of the upwind slope aL / aR,
//   [10..14] those of the time slope aT ([10] includes Mt0),
//   [15] Mt0, [16] Mt3 len, [17] Mt4 len,
//   [18..21] len * g0, the analytic equilibrium part of the macro flux.
template <int NT, typename Meanwhile>
__device__ __forceinline__ void face_coefficients(const ugks_block_desc &d, FaceShared<NT> &sh, const P4 W,
                                                  const P4 prim, const Rcp rc, const double len, const double dt,
                                                  Meanwhile meanwhile) {
  if (threadIdx.x < 32) {
    const double kb = (0.5 * d.K) * rc.lam;
    double Mv[MTUM], Mxi[3];
    P4 a;
    if (threadIdx.x < 2) {
      const int side = threadIdx.x;
      const double sg = side == 0 ? 1.0 : -1.0;
      double Mh[MNUM];
      half_moments_rcp(d.PI, d.K, prim, rc, sg, Mh, Mv, Mxi);
      const double *o = sh.nbr[side];
      // left: (W - W_L) / |mid - c_L|; right: (W_R - W) / |mid - c_R|
      const double id = sg * o[4];
      a = micro_slope_rcp(d.K, prim, rc,
                          p4((W.s0 - o[0]) * id, (W.s1 - o[1]) * id, (W.s2 - o[2]) * id, (W.s3 - o[3]) * id));
      const P4 t1 = moment_au(a, Mh, Mv, Mxi, 1, 0), t2 = moment_au(a, Mh, Mv, Mxi, 2, 0);
      double *x = sh.lr[side];
#pragma unroll
      for (int k = 0; k < MNUM; ++k) x[k] = Mh[k];
      x[7] = a.s0; x[8] = a.s1; x[9] = a.s2; x[10] = a.s3;
      x[11] = t1.s0; x[12] = t1.s1; x[13] = t1.s2; x[14] = t1.s3;
      x[15] = t2.s0; x[16] = t2.s1; x[17] = t2.s2; x[18] = t2.s3;
    }
    pair_wait();
    double Mt[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) Mt[k] = sh.mt[k];
    double *c = sh.bcast;
    if (threadIdx.x < 2) {
      // distFlux coefficients of the upwind slope (derivation at sweep 3)
      const double xk = Mxi[2] - kb * kb;
      double *ck = c + 5 * threadIdx.x;
      ck[0] = Mt[1] * fma(0.5 * a.s3, kb, a.s0);
      ck[1] = Mt[1] * a.s1;
      ck[2] = Mt[1] * a.s2;
      ck[3] = Mt[1] * (0.5 * a.s3);
      ck[4] = Mt[1] * (0.5 * a.s3 * xk);
    }
    if (threadIdx.x == 0) {
      const double *xl = sh.lr[0], *xr = sh.lr[1];
      double Mu[MNUM];
#pragma unroll
      for (int k = 0; k < MNUM; ++k) Mu[k] = xl[k] + xr[k];
      const P4 aT = micro_slope_rcp(d.K, prim, rc,
                                    scale(-prim.s0, add(p4(xl[11], xl[12], xl[13], xl[14]),
                                                        p4(xr[11], xr[12], xr[13], xr[14]))));
      const P4 g0 = scale(prim.s0,
                          add(add(scale(Mt[0], moment_uv(Mu, Mv, Mxi, 1, 0, 0)),
                                  scale(Mt[1], add(p4(xl[15], xl[16], xl[17], xl[18]),
                                                   p4(xr[15], xr[16], xr[17], xr[18])))),
                              scale(Mt[2], moment_au(aT, Mu, Mv, Mxi, 1, 0))));
      const double xk = Mxi[2] - kb * kb;
      c[10] = Mt[2] * fma(0.5 * aT.s3, kb, aT.s0) + Mt[0];
      c[11] = Mt[2] * aT.s1;
      c[12] = Mt[2] * aT.s2;
      c[13] = Mt[2] * (0.5 * aT.s3);
      c[14] = Mt[2] * (0.5 * aT.s3 * xk);
      c[15] = Mt[0];
      c[16] = Mt[3] * len;
      c[17] = Mt[4] * len;
      c[18] = len * g0.s0; c[19] = len * g0.s1; c[20] = len * g0.s2; c[21] = len * g0.s3;
    }
  } else {
    if (threadIdx.x < 64) {
      if (threadIdx.x == 32) {
        double Mt[5];
        time_weights_rcp(inv_relax_time_rcp(d, prim, rc), dt, Mt);
#pragma unroll
        for (int k = 0; k < 5; ++k) sh.mt[k] = Mt[k];
      }
      pair_arrive();
    }
    // warp 1, which computed the time weights, takes the last items
    meanwhile((threadIdx.x + NT - 96) % (NT - 32), NT - 32);
  }
}

// the two cells beside an interior face (the inputs of getAL / getAR and the
// getPLR slopes, clUGKS.c:424-436) into sh.nbr, by two lanes of the last warp
template <int NT>
__device__ __forceinline__ void face_neighbours(const ugks_fused_block &blk, FaceShared<NT> &sh, const long gi,
                                                const long gj, const int dir, const V2 n, const V2 mid) {
  if (threadIdx.x >= NT - 32 && threadIdx.x < NT - 30) {
    const ugks_block_desc &d = blk.d;
    const int side = threadIdx.x - (NT - 32);  // 0: left (u > 0 upwind), 1: right
    const size_t k = side == 0 ? gidx(d, gi - dir, gj - (1 - dir)) : gidx(d, gi, gj);
    const P4 mc = ld4(blk.cell_mom, k);
    const V2 uc = to_local(v2(mc.s1, mc.s2), n);
    const V2 cc = ld2(blk.centre, k);
    double *o = sh.nbr[side];
    o[0] = mc.s0;
    o[1] = uc.x;
    o[2] = uc.y;
    o[3] = mc.s3;
    o[4] = nr_rcp(sqrt((mid.x - cc.x) * (mid.x - cc.x) + (mid.y - cc.y) * (mid.y - cc.y)));
  }
}

// face work item -> (block, i, j, direction, wall face); false when the item
// is skipped (inactive solve, retry pass of a solve without retry, another flux
// method than FM >= 0, or the unused S face of the last column / W face of the last row).
// S and W faces of one corner (i, j) are adjacent work items so that both
// directions read f while it is in L2.
struct FaceWork {
  int bi, dir, mi, mj, wall;
  long gi, gj;
};
template <int FM>
__device__ __forceinline__ bool face_work(const ugks_fused_block *__restrict__ B, int nb,
                                          const ugks_solve_state *__restrict__ solves, const int w, int retry_pass,
                                          FaceWork &fw) {
  fw.bi = find_block<0>(B, nb, w);
  const ugks_fused_block &blk = B[fw.bi];
  const ugks_block_desc &d = blk.d;
  UGKS_CHECK_ITEM(0, blk, w, solves, false);
  const ugks_solve_state &sol = solves[blk.solve];
  if (!sol.active) return false;
  if (retry_pass && !sol.retry) return false;
  if (FM >= 0 && d.flux_method != FM) return false;  // FM < 0: any flux method
  int lf = w - blk.face_begin;
  fw.dir = lf & 1;
  lf >>= 1;
  fw.mi = lf / (d.nj + 1);
  fw.mj = lf % (d.nj + 1);
  if (fw.dir == SOUTH ? (fw.mi >= d.ni) : (fw.mj >= d.nj)) return false;
  fw.gi = fw.mi + d.ghost;
  fw.gj = fw.mj + d.ghost;
  fw.wall = -1;
  if (fw.dir == SOUTH) {
    if (fw.mj == 0 && is_wall(blk.bc_type[GSOUTH])) fw.wall = GSOUTH;
    else if (fw.mj == d.nj && is_wall(blk.bc_type[GNORTH])) fw.wall = GNORTH;
  } else {
    if (fw.mi == 0 && is_wall(blk.bc_type[GWEST])) fw.wall = GWEST;
    else if (fw.mi == d.ni && is_wall(blk.bc_type[GEAST])) fw.wall = GEAST;
  }
  return true;
}

// one FP64 face work item (all threads of the CTA take part)
template <int FM, int NT>
__device__ __forceinline__ void face_item_fp64(const ugks_fused_block *__restrict__ B, int nb,
                                               ugks_solve_state *__restrict__ solves, const int w, int retry_pass) {
  extern __shared__ double dyn[];
  __shared__ FaceShared<NT> sh;
  using St = Store<double>;
  FaceWork fwk;
  if (!face_work<FM>(B, nb, solves, w, retry_pass, fwk)) return;
  const ugks_fused_block &blk = B[fwk.bi];
  const ugks_block_desc &d = blk.d;
  ugks_solve_state &sol = solves[blk.solve];
  const double dt = sol.dt;
  const int dir = fwk.dir, mi = fwk.mi, mj = fwk.mj, wall = fwk.wall;
  const long gi = fwk.gi, gj = fwk.gj;
  const int Nv = d.Nv;

  // per velocity: (h, b) at the face and their slopes, kept for the later
  // sweeps in shared memory
  double2 *fhb = reinterpret_cast<double2 *>(dyn), *sgb = fhb + Nv;
  const V2 n = ld2(blk.normal, faceidx(d, gi, gj, dir));
  const V2 mid = ld2(blk.mid_side, faceidx(d, gi, gj, dir));
  // velocity tables and the face-frame velocity (interfaceVelocity,
  // clFunctions.c:191-209), with the table pointers held in registers
  const double2 *__restrict__ qd = reinterpret_cast<const double2 *>(d.quad);
  const double *__restrict__ wt = d.weight;
  auto fvel = [&](int vv) {
    const double2 e = qd[vv];
    return v2(e.x * n.x + e.y * n.y, e.x * (-n.y) + e.y * n.x);
  };
  // stencil geometry for both upwind directions (iFace, clUGKS.c:148-176),
  // precomputed by face_geometry: index 1 for u > 0 (upwind cell before the
  // face), 0 otherwise
  double g6[6];
  {
    const double *fg = blk.face_geo + 6 * faceidx(d, gi, gj, dir);
#pragma unroll
    for (int k = 0; k < 6; ++k) g6[k] = fg[k];
  }
  const double dist0 = g6[0], idist0 = g6[1], il0 = g6[2], dist1 = g6[3], idist1 = g6[4], il1 = g6[5];
  const int step = dir == SOUTH ? Nv : d.Nj * Nv;
  const size_t base = fidx(d, gi, gj, 0);
  constexpr int MID = FM == 1 ? 2 : 1;
  const double2 *fcell = reinterpret_cast<const double2 *>(blk.f) + base;  // cell (gi, gj), velocity 0
  const double2 *up1 = fcell - (MID + 1) * step, *up0 = fcell + MID * step;

  // ---- sweep 1: reconstruction (+ interior faces: the face moments W of
  // getFaceCons; the 1/2 of the energy moment is applied after the sum)
  double m[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
  for (int v = threadIdx.x; v < Nv; v += NT) {
    const V2 uv = fvel(v);
    const bool up = uv.x > 0.0;
    double ffh, ffb, sx, sy;
    reconstruct<double, FM>((up ? up1 : up0) + v, up ? step : -step, up ? il1 : il0, up ? dist1 : dist0,
                            up ? idist1 : idist0, ffh, ffb, sx, sy);
    fhb[v] = make_double2(ffh, ffb);
    sgb[v] = make_double2(sx, sy);
    if (wall < 0) {
      const double uu = fma(uv.x, uv.x, uv.y * uv.y);
      m[0] += ffh;
      m[1] = fma(uv.x, ffh, m[1]);
      m[2] = fma(uv.y, ffh, m[2]);
      m[3] += fma(uu, ffh, ffb);
    }
  }
  // loaded by the last warp, which has the fewest velocities in sweep 1
  if (wall < 0) face_neighbours<NT>(blk, sh, gi, gj, dir, n, mid);
  const double len = blk.side_length[faceidx(d, gi, gj, dir)];

  if (wall < 0) {
    // ---------------- interior face ----------------
    block_sum_spread<4>(m, sh.scratch);
    const P4 W = p4(m[0], m[1], m[2], 0.5 * m[3]);
    Rcp rc;
    const P4 prim = to_primary_rcp(d, W, rc);  // getPLR (clUGKS.c:421-422), every thread
    const int un = d.u_num, vn = d.v_num;
    const bool sep = un > 0 && un * vn == Nv && un + vn <= 512;
    double *Eu = reinterpret_cast<double *>(sgb + Nv), *Ev = Eu + (sep ? un : 0);
    const V2 Ug = to_global(v2(prim.s1, prim.s2), n);  // face mean velocity, global frame
    // Maxwellian prefactor rho lambda / pi (fM, clFunctions.c:49-58), times the
    // face length: every per-velocity flux below carries the length
    const double chl = (prim.s0 * (prim.s3 / d.PI)) * len;
    double q[2] = {0.0, 0.0};
    face_coefficients<NT>(d, sh, W, prim, rc, len, dt, [&](int t, int nt) {
      // face heat flux (calcFaceQ, clUGKS.c:522-585) and the axis factors of
      // the face Maxwellian
      const double Kinv = 1.0 / d.K;
      for (int v = t; v < Nv; v += nt) {
        const V2 uv = fvel(v);
        const double cx = uv.x - prim.s1, cy = uv.y - prim.s2, c2 = cx * cx + cy * cy;
        const double2 fv = fhb[v];
        const double tq = c2 * fv.x + fv.y * Kinv;
        q[0] += 0.5 * (cx * tq);
        q[1] += 0.5 * (cy * tq);
      }
      if (sep) {
        axis_exp(Eu, d.quad, un, vn, 0, Ug.x, prim.s3, t, nt, chl);
        axis_exp(Ev, d.quad, vn, 1, 1, Ug.y, prim.s3, t, nt);
      }
    });
    block_sum_spread<2>(q, sh.scratch);
    // ---- sweep 3: macroFlux (587-681) and distFlux (683-772).
    // With h0 = weight * fM (times the face length), kb = K / (2 lambda),
    // S = Mt0 s (c . Q) (the Shakhov factor of fS, clFunctions.c:64-77, times
    // Mt0), P4 = 2 lambda c^2 - 4, the upwind slope a (aL for u > 0, else aR),
    //   Ph = a0 + a1 u + a2 v + a3 (|u|^2 + kb) / 2, and Th likewise with aT,
    //   Rh = Mt3 fh - Mt4 u sh,   Rb = Mt3 fb - Mt4 u sb,
    //   Zh = u (S P4 h0 + Rh),    Zb = u (S (P4 + 2) kb h0 + Rb),
    //   B  = Mt0 + Mt1 u Ph + Mt2 Th,
    // distFlux's two components are
    //   hx = Zh + u h0 B,
    //   hy = Zb + u h0 (kb B + Mt1 u a3 X / 2 + Mt2 aT3 X / 2),  X = Mxi2 - kb^2,
    // and macroFlux's discrete part sums (Zh, u Zh, v Zh, (|u|^2 Zh + Zb) / 2).
    const double *c = sh.bcast;
    const V2 Q = v2(q[0], q[1]);
    const double lam = prim.s3, Ux = prim.s1, Uy = prim.s2, lam2 = 2.0 * lam;
    const double kb = (0.5 * d.K) * rc.lam;
    const double s0 = 0.8 * (1 - d.Pr) * (lam * lam) * rc.rho;
    const double Mt0 = c[15], Mt3 = c[16], Mt4 = c[17];
    const double sx = (Mt0 * s0) * Q.x, sy = (Mt0 * s0) * Q.y;
    const double T0 = c[10], T1 = c[11], T2 = c[12], T3 = c[13], CT = c[14];
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    void *flux = dir == SOUTH ? blk.flux_S : blk.flux_W;
    const int qs = sep ? NT / vn : 0, rs = sep ? NT % vn : 0;
    int iu = sep ? threadIdx.x / vn : 0, jv = sep ? threadIdx.x % vn : 0;
    for (int v = threadIdx.x; v < Nv; v += NT) {
      const V2 uv = fvel(v);
      const double u = uv.x, vt = uv.y, uu = fma(u, u, vt * vt);
      const double cx = u - Ux, cy = vt - Uy, c2 = fma(cx, cx, cy * cy);
      double E;
      if (sep) {
        E = Eu[iu] * Ev[jv];
        jv += rs;
        iu += qs;
        if (jv >= vn) { jv -= vn; ++iu; }
      } else {
        E = chl * exp(-lam * c2);
      }
      const double h0 = wt[v] * E;
      const double Sp = fma(cx, sx, cy * sy);
      const double S4 = Sp * fma(lam2, c2, -4.0), S2 = fma(2.0, Sp, S4);
      const double *A = c + (u > 0.0 ? 0 : 5);
      const double MP = fma(A[3], uu, fma(A[2], vt, fma(A[1], u, A[0])));
      const double Bk = fma(u, MP, fma(T3, uu, fma(T2, vt, fma(T1, u, T0))));
      const double2 fd = fhb[v], fs = sgb[v];
      const double mu = Mt4 * u;
      const double Rh = fma(-mu, fs.x, Mt3 * fd.x), Rb = fma(-mu, fs.y, Mt3 * fd.y);
      const double Zh = u * fma(S4, h0, Rh), Zb = u * fma(S2, h0 * kb, Rb);
      const double uh = u * h0;
      const double hx = fma(uh, Bk, Zh);
      const double hy = fma(uh, fma(kb, Bk, fma(A[4], u, CT)), Zb);
      acc[0] += Zh;
      acc[1] = fma(u, Zh, acc[1]);
      acc[2] = fma(vt, Zh, acc[2]);
      acc[3] = fma(uu, Zh, acc[3]);
      acc[4] += Zb;
      St::store(flux, base + v, v2(hx, hy));
    }
    block_sum_spread_to0<5>(acc, sh.scratch);
    if (threadIdx.x == 0) {
      P4 out = p4(acc[0] + c[18], acc[1] + c[19], acc[2] + c[20], 0.5 * (acc[3] + acc[4]) + c[21]);
      const V2 g = to_global(v2(out.s1, out.s2), n);
      out.s1 = g.x;
      out.s2 = g.y;
      st4(dir == SOUTH ? blk.flux_macro_S : blk.flux_macro_W, gidx(d, gi, gj), out);
    }
    return;
  }

  // ---------------- wall face ----------------
  wall_face<NT>(blk, sol, sh, reinterpret_cast<double *>(fhb), sgb, wall, dir, gi, gj, mi, mj, n, len, dt,
                [&](int v, double hx, double hy) { St::store(dir == SOUTH ? blk.flux_S : blk.flux_W, base + v,
                                                               v2(hx, hy)); });
}

// the mixed path's face work item (ugks_delta.cuh, included further down):
// WALLS, the wall faces (main pass: the wall launch; retry pass), else the
// reconstruction and moments of the interior faces
template <int FM, int NT, bool WALLS>
__device__ __forceinline__ void face_item_delta(const ugks_fused_block *__restrict__ B, int nb,
                                                ugks_solve_state *__restrict__ solves, const int w, int retry_pass);

// one face work item: FP64 storage, or the mixed path's FP32 deviations
template <typename T, int FM, int NT, bool RETRY>
__device__ __forceinline__ void face_item(const ugks_fused_block *__restrict__ B, int nb,
                                          ugks_solve_state *__restrict__ solves, const int w) {
  if constexpr (std::is_same<T, float>::value) face_item_delta<FM, NT, RETRY>(B, nb, solves, w, RETRY ? 1 : 0);
  else face_item_fp64<FM, NT>(B, nb, solves, w, RETRY ? 1 : 0);
}

// main face pass: one CTA per face work item of the blocks of one flux method
template <typename T, int FM, int MINB, int NT>
__global__ void __launch_bounds__(NT, MINB) face_pass(const ugks_fused_block *__restrict__ B, int nb,
                                                                 ugks_solve_state *__restrict__ solves,
                                                                 int first) {
  face_item<T, FM, NT, false>(B, nb, solves, first + (int)blockIdx.x);
}

// the flux pass redone after a dt change (ugks_sim.py:432-441): RETRY_CTAS
// CTAs per solve; a solve whose retry flag is clear costs one early exit each
constexpr int RETRY_CTAS = 148;
template <typename T, int FM, int MINB, int NT>
__global__ void __launch_bounds__(NT, MINB) face_retry(const ugks_fused_block *__restrict__ B, int nb,
                                                                  ugks_solve_state *__restrict__ solves,
                                                                  int ns) {
  const int s = blockIdx.x / RETRY_CTAS, r = blockIdx.x % RETRY_CTAS;
  if (s >= ns) return;
  const ugks_solve_state &x = solves[s];
  if (!x.active || !x.retry || x.nblocks <= 0) return;
  const ugks_fused_block &b0 = B[x.first_block], &bl = B[x.first_block + x.nblocks - 1];
  if (b0.d.flux_method != FM) return;
  const int end = bl.face_begin + 2 * (bl.d.ni + 1) * (bl.d.nj + 1);
  for (int w = b0.face_begin + r; w < end; w += RETRY_CTAS) {
    face_item<T, FM, NT, true>(B, nb, solves, w);
    __syncthreads();  // the next item reuses the shared tables
  }
}

// ---------------------------------------------------------------------------
// cell pass: calcQ (clKernel.c:480-543) + updateMacro (clUGKS.c:1158-1187) +
// UGKS_update (clUGKS.c:1189-1257) + clFindDT (clKernel.c:224-308)
// ---------------------------------------------------------------------------
// clFindDT with the descriptor's Kn (the host's unrounded Kn, ugks_block.py:1421)
__device__ __forceinline__ double cfl_freq(const ugks_fused_block &blk, P4 m, long mi, long mj) {
  return cfl_frequency(blk.d, blk.xy, blk.area, m, mi, mj, blk.d.Kn_eff);
}

// one warp per cell, CW cells per CTA: no block-wide barrier, so the serial
// per-cell coefficients of one cell (lane 0) stall only that cell's warp
constexpr int CW = 8;
// per-warp shared memory: the axis tables of the old and new state
// (2 (u_num + v_num) doubles) and CELL_COEF coefficient slots
constexpr int CELL_COEF = 16;

template <int N>
__device__ __forceinline__ void warp_sum(double (&x)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x[k] += __shfl_xor_sync(0xffffffffu, x[k], o);
  }
}

template <typename T, int MINB = CellBudget<T>::minb>
__global__ void __launch_bounds__(CW * 32, MINB) cell_pass(const ugks_fused_block *__restrict__ B, int nb,
                                                        ugks_solve_state *__restrict__ solves, int n_cells,
                                                        int wstride) {
  extern __shared__ double dyn[];
  using St = Store<T>;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int w = blockIdx.x * CW + warp;
  if (w >= n_cells) return;
  const int bi = find_block<1>(B, nb, w);
  const ugks_fused_block &blk = B[bi];
  const ugks_block_desc &d = blk.d;
  UGKS_CHECK_ITEM(1, blk, w, solves);
  ugks_solve_state &sol = solves[blk.solve];
  if (!sol.active) return;
  const int lc = w - blk.cell_begin;
  const long mi = lc / d.nj, mj = lc % d.nj;
  const long gi = mi + d.ghost, gj = mj + d.ghost;
  const int Nv = d.Nv, un = d.u_num, vn = d.v_num;
  const bool sep = un > 0 && un * vn == Nv && un + vn <= 512;
  double *Eou = dyn + (size_t)warp * wstride, *Eov = Eou + un, *Enu = Eov + vn, *Env = Enu + un;
  double *bc = dyn + (size_t)warp * wstride + (wstride - CELL_COEF);
  const size_t base = fidx(d, gi, gj, 0);
  const size_t sj = (size_t)Nv, si = (size_t)d.Nj * Nv;
  const double dt = sol.dt;
  const P4 old = ld4(blk.macro, midx(d, mi, mj));
  // calcQ of f^n with the macro of f^n: accumulated by the previous cell pass
  // (or the initialisation) in Q_next
  const V2 Q = ld2(blk.Q_next, midx(d, mi, mj));
  if (lane == 0) {
    // updateMacro
    const P4 wc = to_conserved(d, old);
    const double iA = 1.0 / blk.area[gidx(d, gi, gj)];
    const P4 s0 = ld4(blk.flux_macro_S, gidx(d, gi, gj)), s1 = ld4(blk.flux_macro_S, gidx(d, gi, gj + 1));
    const P4 w0 = ld4(blk.flux_macro_W, gidx(d, gi, gj)), w1 = ld4(blk.flux_macro_W, gidx(d, gi + 1, gj));
    const P4 nw = p4(wc.s0 + (s0.s0 - s1.s0 + w0.s0 - w1.s0) * iA, wc.s1 + (s0.s1 - s1.s1 + w0.s1 - w1.s1) * iA,
                     wc.s2 + (s0.s2 - s1.s2 + w0.s2 - w1.s2) * iA, wc.s3 + (s0.s3 - s1.s3 + w0.s3 - w1.s3) * iA);
    Rcp rn, ro;
    const P4 prim = to_primary_rcp(d, nw, rn);
    ro.rho = nr_rcp(old.s0);
    ro.lam = nr_rcp(old.s3);
    st4(blk.macro, midx(d, mi, mj), prim);
    st4(blk.prim_old, midx(d, mi, mj), old);
    st2(blk.Q, midx(d, mi, mj), Q);
    // UGKS_update (clUGKS.c:1189-1257) per velocity, regrouped:
    //   f' = f a1 + (sum of face fluxes) a2 + fEQ(new) a3 + fEQ(old) a4,
    //   a1 = (1 - dt/2 /tau_old) / D, a2 = 1 / (A D), a3 = dt/2 / (tau D),
    //   a4 = dt/2 / (tau_old D), D = 1 + dt/2 / tau;
    // a3 and a4 go into the Maxwellian prefactors rho lambda / pi of fEQ
    const double itau_old = inv_relax_time_rcp(d, old, ro), itau = inv_relax_time_rcp(d, prim, rn);
    const double hdt = 0.5 * dt, iden = nr_rcp(1.0 + hdt * itau);
    const double ipi = nr_rcp(d.PI);
    bc[0] = prim.s1;
    bc[1] = prim.s2;
    bc[2] = prim.s3;
    bc[3] = (1.0 - hdt * itau_old) * iden;                         // a1
    bc[4] = iden * iA;                                             // a2
    bc[5] = prim.s0 * (prim.s3 * ipi) * (hdt * itau * iden);       // new prefactor x a3
    bc[6] = old.s0 * (old.s3 * ipi) * (hdt * itau_old * iden);     // old prefactor x a4
    bc[7] = (0.5 * d.K) * rn.lam;                                  // K / (2 lambda) new
    bc[8] = 0.8 * (1 - d.Pr) * (prim.s3 * prim.s3) * rn.rho;       // Shakhov factor new
    const double fq = cfl_freq(blk, prim, mi, mj);
    atomicMax(&sol.max_freq, (unsigned long long)__double_as_longlong(fq));
  } else if (sep) {
    axis_exp(Eou, d.quad, un, vn, 0, old.s1, old.s3, lane - 1, 31);
    axis_exp(Eov, d.quad, vn, 1, 1, old.s2, old.s3, lane - 1, 31);
  }
  __syncwarp();
  const double nU = bc[0], nV = bc[1], nl = bc[2];
  if (sep) {
    axis_exp(Enu, d.quad, un, vn, 0, nU, nl, lane, 32);
    axis_exp(Env, d.quad, vn, 1, 1, nV, nl, lane, 32);
    __syncwarp();
  }
  const double a1 = bc[3], a2 = bc[4], cn = bc[5], co = bc[6], kn = bc[7], sn = bc[8];
  const double ko = (0.5 * d.K) * nr_rcp(old.s3);
  const double so = 0.8 * (1 - d.Pr) * (old.s3 * old.s3) * nr_rcp(old.s0);
  const int qs = sep ? 32 / vn : 0, rs = sep ? 32 % vn : 0;
  int iu = sep ? lane / vn : 0, jv = sep ? lane % vn : 0;
  bool nan = false;
  // FP64: the five rows this lane reads run D velocities (of this lane)
  // ahead through a ring of cp.async stages; a stage is refilled only after
  // the store that consumed its values, whose operands are the stage's loads
  constexpr int D = CellBudget<T>::ring;
  using E = typename St::vec;
  E *ring = reinterpret_cast<E *>(dyn + (size_t)CW * wstride) + (size_t)warp * (D * 5 * 32) + lane;
  const E *gf = reinterpret_cast<const E *>(blk.f), *gS = reinterpret_cast<const E *>(blk.flux_S),
          *gW = reinterpret_cast<const E *>(blk.flux_W);
  auto issue = [&](int vv, int stage) {
    if (D == 0) return;
    if (vv < Nv) {
      const size_t k = base + vv;
      E *r = ring + stage * (5 * 32);
      cp_async<sizeof(E)>(r, gf + k);
      cp_async<sizeof(E)>(r + 32, gS + k);
      cp_async<sizeof(E)>(r + 64, gS + k + sj);
      cp_async<sizeof(E)>(r + 96, gW + k);
      cp_async<sizeof(E)>(r + 128, gW + k + si);
    }
    cp_async_commit();
  };
#pragma unroll
  for (int s = 0; s < D; ++s) issue(lane + 32 * s, s);
  int stage = 0;
#pragma unroll 1
  for (int v = lane; v < Nv; v += 32) {
    const size_t k = base + v;
    V2 f, s0, s1, w0, w1;
    if constexpr (D > 0) {
      cp_async_wait<D - 1>();
      const E *r = ring + stage * (5 * 32);
      const E fe = r[0], s0e = r[32], s1e = r[64], w0e = r[96], w1e = r[128];
      f = v2(fe.x, fe.y);
      s0 = v2(s0e.x, s0e.y);
      s1 = v2(s1e.x, s1e.y);
      w0 = v2(w0e.x, w0e.y);
      w1 = v2(w1e.x, w1e.y);
    } else {
      f = St::load(blk.f, k);
      s0 = St::load(blk.flux_S, k);
      s1 = St::load(blk.flux_S, k + sj);
      w0 = St::load(blk.flux_W, k);
      w1 = St::load(blk.flux_W, k + si);
    }
    const V2 e = quad_at(d, v);
    const double wv = d.weight[v];
    const double ox = e.x - old.s1, oy = e.y - old.s2, o2 = fma(ox, ox, oy * oy);
    const double nx = e.x - nU, ny = e.y - nV, n2 = fma(nx, nx, ny * ny);
    double Eo, En;
    if (sep) {
      Eo = Eou[iu] * Eov[jv];
      En = Enu[iu] * Env[jv];
      jv += rs;
      iu += qs;
      if (jv >= vn) { jv -= vn; ++iu; }
    } else {
      Eo = exp(-old.s3 * o2);
      En = exp(-nl * n2);
    }
    // fEQ (clFunctions.c:79-86) at the old and the new macro state, scaled
    const double ho = wv * co * Eo, hn = wv * cn * En;
    const double So = so * fma(ox, Q.x, oy * Q.y), Sn = sn * fma(nx, Q.x, ny * Q.y);
    const double po = fma(2.0 * old.s3, o2, -4.0), pn = fma(2.0 * nl, n2, -4.0);
    const double eh = fma(So * po, ho, ho) + fma(Sn * pn, hn, hn);
    const double eb = ko * fma(So * (po + 2.0), ho, ho) + kn * fma(Sn * (pn + 2.0), hn, hn);
    const double flh = (s0.x - s1.x) + (w0.x - w1.x), flb = (s0.y - s1.y) + (w0.y - w1.y);
    const V2 out = v2(fma(f.x, a1, fma(flh, a2, eh)), fma(f.y, a1, fma(flb, a2, eb)));
    nan |= isnan(out.x) || isnan(out.y);
    St::store(blk.f, k, out);
    if constexpr (D > 0) {
      issue(v + 32 * D, stage);
      stage = stage + 1 == D ? 0 : stage + 1;
    }
  }
  if constexpr (D > 0) cp_async_wait<0>();
  if (nan) atomicExch(&sol.status, 1);
  // moments of f^{n+1} for the next face pass, and calcQ (clKernel.c:480-543)
  // of f^{n+1} with the new macro for the next cell pass: a second sweep over
  // the values this lane just stored (L2-resident), which keeps the update
  // loop's registers free
  const double Kinv = nr_rcp(d.K);
  double mom[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int v = lane; v < Nv; v += 32) {
    const V2 o = St::load(blk.f, base + v);
    const V2 e = quad_at(d, v);
    const double nx = e.x - nU, ny = e.y - nV, n2 = fma(nx, nx, ny * ny);
    mom[0] += o.x;
    mom[1] = fma(e.x, o.x, mom[1]);
    mom[2] = fma(e.y, o.x, mom[2]);
    mom[3] += fma(fma(e.x, e.x, e.y * e.y), o.x, o.y);
    const double t = fma(n2, o.x, o.y * Kinv);
    mom[4] = fma(nx, t, mom[4]);
    mom[5] = fma(ny, t, mom[5]);
  }
  warp_sum<6>(mom);
  if (lane == 0) {
    st4(blk.cell_mom, gidx(d, gi, gj), p4(mom[0], mom[1], mom[2], 0.5 * mom[3]));
    st2(blk.Q_next, midx(d, mi, mj), v2(0.5 * mom[4], 0.5 * mom[5]));
  }
}

// ---------------------------------------------------------------------------
// ghost pass (UGKSBlock.updateBC, ugks_block.py:621-665): one CTA per ghost
// cell of every block face
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(FT) ghost_pass(const ugks_fused_block *__restrict__ B, int nb,
                                                 const ugks_solve_state *__restrict__ solves) {
  __shared__ double scratch[4 * (FT / 32)];
  using St = Store<T>;
  const int w = blockIdx.x;
  const int bi = find_block<2>(B, nb, w);
  const ugks_fused_block &blk = B[bi];
  const ugks_block_desc &d = blk.d;
  UGKS_CHECK_ITEM(2, blk, w, solves);
  if (!solves[blk.solve].active) return;
  const int G = d.ghost, Nv = d.Nv;
  // strips in face order N, E, S, W: N/S have ni*G cells, E/W G*nj
  int lc = w - blk.ghost_begin;
  int face = 0;
  const int ns_cells = d.ni * G, ew_cells = G * d.nj;
  for (face = 0; face < 4; ++face) {
    const int c = (face == GNORTH || face == GSOUTH) ? ns_cells : ew_cells;
    if (lc < c) break;
    lc -= c;
  }
  long a, b;  // NDRange ids of the reference edge kernels
  if (face == GNORTH || face == GSOUTH) { a = lc / G; b = lc % G; }
  else { a = lc / d.nj; b = lc % d.nj; }
  long gi = a, gj = b;
  switch (face) {
    case GNORTH: gi += G; gj += d.Nj - G; break;
    case GEAST: gi += d.Ni - G; gj += G; break;
    case GSOUTH: gi += G; break;
    default: gj += G; break;
  }
  const size_t dst = fidx(d, gi, gj, 0);
  const int t = blk.bc_type[face];
  // every branch writes the ghost cell through put(), which also sums the
  // cell moments the next face pass reads
  double mom[4] = {0.0, 0.0, 0.0, 0.0};
  auto put = [&](int v, V2 x) {
    St::store(blk.f, dst + v, x);
    const V2 o = St::as_stored(x);
    const V2 e = quad_at(d, v);
    mom[0] += o.x;
    mom[1] = fma(e.x, o.x, mom[1]);
    mom[2] = fma(e.y, o.x, mom[2]);
    mom[3] += fma(fma(e.x, e.x, e.y * e.y), o.x, o.y);
  };
  // load(v) for every velocity, put in the same order as a plain loop
  auto copy = [&](auto load) {
    for (int v0 = threadIdx.x; v0 < Nv; v0 += GHOST_U * FT) {
      V2 x[GHOST_U];
#pragma unroll
      for (int u = 0; u < GHOST_U; ++u)
        if (v0 + u * FT < Nv) x[u] = load(v0 + u * FT);
#pragma unroll
      for (int u = 0; u < GHOST_U; ++u)
        if (v0 + u * FT < Nv) put(v0 + u * FT, x[u]);
    }
  };
  if (t == BC_ADJACENT || t == BC_PERIODIC) {
    // edgeExchange (clGhostRoutines.c:407-538)
    const ugks_fused_block &ob = B[blk.bc_block[face]];
    const int that = blk.bc_face[face], NI = d.Ni, NJ = d.Nj, NIB = ob.d.Ni, NJB = ob.d.Nj;
    int a1i, a1j, a2i, a2j, b1i, b1j, b2i, b2j;
    auto corners = [&](int f, int NI_, int NJ_, int &p, int &q, int &r, int &s) {
      switch (f) {
        case GNORTH: p = G; q = NJ_ - G; r = NI_ - G; s = NJ_ - G; break;
        case GEAST: p = NI_ - G; q = G; r = NI_ - G; s = NJ_ - G; break;
        case GSOUTH: p = G; q = G; r = NI_ - G; s = G; break;
        default: p = G; q = G; r = G; s = NJ_ - G; break;
      }
    };
    corners(face, NI, NJ, a1i, a1j, a2i, a2j);
    corners(that, NIB, NJB, b1i, b1j, b2i, b2j);
    const V2 A1 = ld2(blk.xy, (size_t)a1i * (NJ + 1) + a1j), A2 = ld2(blk.xy, (size_t)a2i * (NJ + 1) + a2j);
    const V2 B1 = ld2(ob.xy, (size_t)b1i * (NJB + 1) + b1j), B2 = ld2(ob.xy, (size_t)b2i * (NJB + 1) + b2j);
    const bool misalign = !(fabs(A1.x - B1.x) <= 1e-6) || !(fabs(A1.y - B1.y) <= 1e-6) ||
                          !(fabs(A2.x - B2.x) <= 1e-6) || !(fabs(A2.y - B2.y) <= 1e-6);
    int iB = (int)gi, jB = (int)gj;
    if (misalign && blk.bc_ori[face]) {
      if (face == GEAST || face == GWEST) jB = (NJ - 1) - jB;
      else iB = (NI - 1) - iB;
    }
    swap_cell_index(NI, NJ, G, face, iB, jB, that, NIB, NJB);
    if (iB < 0 || iB >= NIB || jB < 0 || jB >= NJB || ob.d.Nv != Nv) {
      // connection that does not map onto the neighbour: flag, do not read
      if (threadIdx.x == 0) atomicExch(const_cast<int32_t *>(&solves[blk.solve].status), 6);
      return;
    }
    const size_t src = ((size_t)iB * NJB + jB) * (size_t)Nv;
    const int flip = blk.bc_flip[face];
    const int32_t *perm = flip == FLIP_NS ? d.mirror_NS : (flip == FLIP_D ? d.mirror_D : d.mirror_EW);
    if (flip == NO_FLIP) copy([&](int v) { return St::load(ob.f, src + v); });
    else copy([&](int v) { return St::load(ob.f, src + perm[v]); });
  } else if (t == BC_DIFFUSE || t == BC_ADSORBING) {
    // edgeConstGrad (clGhostRoutines.c:967-1048)
    long ei0, ej0, ei1, ej1;
    double m;
    switch (face) {
      case GNORTH: ei1 = gi; ej1 = d.Nj - G - 1; ei0 = ei1; ej0 = ej1 - 1; m = (double)(gj - ej1); break;
      case GEAST: ei1 = d.Ni - G - 1; ej1 = gj; ei0 = ei1 - 1; ej0 = ej1; m = (double)(gi - ei1); break;
      case GSOUTH: ei1 = gi; ej1 = G; ei0 = ei1; ej0 = ej1 + 1; m = (double)(ej1 - gj); break;
      default: ei1 = G; ej1 = gj; ei0 = ei1 + 1; ej0 = ej1; m = (double)(ei1 - gi); break;
    }
    const size_t k0 = fidx(d, ei0, ej0, 0), k1 = fidx(d, ei1, ej1, 0);
    copy([&](int v) {
      const V2 f0 = St::load(blk.f, k0 + v), f1 = St::load(blk.f, k1 + v);
      return v2(__dadd_rn(f1.x, __dmul_rn(m, __dsub_rn(f1.x, f0.x))),
                __dadd_rn(f1.y, __dmul_rn(m, __dsub_rn(f1.y, f0.y))));
    });
  } else if (t == BC_EXTRAPOLATE_OUT || t == BC_REFLECT || t == BC_BOUNCE_BACK) {
    long si, sj;
    const int32_t *perm = nullptr;
    if (t == BC_EXTRAPOLATE_OUT) {  // edgeExtrapolate (544-597)
      switch (face) {
        case GNORTH: si = gi; sj = d.Nj - G - 1; break;
        case GEAST: si = d.Ni - G - 1; sj = gj; break;
        case GSOUTH: si = gi; sj = G; break;
        default: si = G; sj = gj; break;
      }
    } else {  // edgeMirror / edgeBounceBack (845-961)
      switch (face) {
        case GNORTH: si = gi; sj = 2 * (d.Nj - G) - gj - 1; perm = d.mirror_NS; break;
        case GEAST: si = 2 * (d.Ni - G) - gi - 1; sj = gj; perm = d.mirror_EW; break;
        case GSOUTH: si = gi; sj = 2 * G - gj - 1; perm = d.mirror_NS; break;
        default: si = 2 * G - gi - 1; sj = gj; perm = d.mirror_EW; break;
      }
      if (t == BC_BOUNCE_BACK) perm = d.mirror_D;
    }
    const size_t src = fidx(d, si, sj, 0);
    if (perm) copy([&](int v) { return St::load(blk.f, src + perm[v]); });
    else copy([&](int v) { return St::load(blk.f, src + v); });
  } else if (t == BC_CONSTANT || t == BC_INFLOW || t == BC_OUTFLOW) {
    const long ci = (face == GNORTH || face == GSOUTH) ? a : b;
    const P4 wp = ld4(blk.wall_prop, ci * 4 + face);
    P4 prim = wp;
    V2 Q = v2(0.0, 0.0);
    if (t != BC_CONSTANT) {
      // edgeInflow / edgeOutflow (664-839)
      long ei, ej, noi, noj;
      int fid;
      switch (face) {
        case GNORTH: ei = gi; ej = d.Nj - G - 1; noi = gi; noj = gj; fid = SOUTH; break;
        case GEAST: ei = d.Ni - G - 1; ej = gj; noi = gi; noj = gj; fid = WEST; break;
        case GSOUTH: ei = gi; ej = G; noi = ei; noj = ej; fid = SOUTH; break;
        default: ei = G; ej = gj; noi = ei; noj = ej; fid = WEST; break;
      }
      Q = ld2(blk.Q, midx(d, ei - G, ej - G));
      prim = ld4(blk.macro, midx(d, ei - G, ej - G));
      const V2 uv = to_local(v2(prim.s1, prim.s2), ld2(blk.normal, faceidx(d, noi, noj, fid)));
      prim.s1 = uv.x;
      prim.s2 = uv.y;
      if (t == BC_OUTFLOW) {
        prim.s3 = prim.s0 / (wp.s0 / wp.s3);
      } else {
        prim.s0 = wp.s0;
        prim.s3 = wp.s3;
      }
    }
    for (int v = threadIdx.x; v < Nv; v += FT) put(v, shakhov_eq(d, prim, Q, quad_at(d, v), v));
  }
  block_sum<4>(mom, scratch);
  if (threadIdx.x == 0) st4(blk.cell_mom, gidx(d, gi, gj), p4(mom[0], mom[1], mom[2], 0.5 * mom[3]));
}

// ---------------------------------------------------------------------------
// dt control (ugks_sim.py:285-311, 430-446, 458-460, 491)
// ---------------------------------------------------------------------------
// after a flux pass: updateTimeStep inside the dt loop; phase 0 sets retry
__global__ void dt_check(ugks_solve_state *solves, int ns, int phase) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  ugks_solve_state &x = solves[s];
  if (!x.active) return;
  if (phase == 0) {
    const double dt = limited_dt(x.dt, x.max_dt, x.delta_dt);
    x.retry = dt != x.dt;
    x.dt = dt;
  } else if (x.retry) {
    x.dt = limited_dt(x.dt, x.max_dt, x.delta_dt);
    x.retries += 1;
  }
}

// after the cell pass: calcTimeStep + updateTimeStep, time += dt, residual
__global__ void dt_update(ugks_solve_state *solves, int ns) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  ugks_solve_state &x = solves[s];
  if (!x.active) return;
  const double fq = __longlong_as_double((long long)x.max_freq);
  x.max_dt = x.CFL / fq;
  x.dt = limited_dt(x.dt, x.max_dt, x.delta_dt);
  x.time += x.dt;
  x.steps += 1;
  x.max_freq = 0ull;
  x.retry = 0;
}

// ---------------------------------------------------------------------------
// initial state (ugks_block.py:411-429, ugks_sim.py:88-92)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(FT) init_cells(const ugks_fused_block *__restrict__ B, int nb,
                                                 ugks_solve_state *__restrict__ solves) {
  __shared__ double scratch[4 * (FT / 32)];
  using St = Store<T>;
  const int w = blockIdx.x;
  const int bi = find_block<1>(B, nb, w);
  const ugks_fused_block &blk = B[bi];
  const ugks_block_desc &d = blk.d;
  UGKS_CHECK_ITEM(1, blk, w, solves);
  ugks_solve_state &sol = solves[blk.solve];
  if (!sol.active) return;
  const int lc = w - blk.cell_begin;
  const long mi = lc / d.nj, mj = lc % d.nj;
  const size_t base = fidx(d, mi + d.ghost, mj + d.ghost, 0);
  // initFunctions
  P4 prim = ld4(blk.macro, midx(d, mi, mj));
  V2 Q = ld2(blk.Q, midx(d, mi, mj));
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  for (int v = threadIdx.x; v < d.Nv; v += FT) {
    const V2 e = quad_at(d, v);
    const V2 f = shakhov_eq(d, prim, Q, e, v);
    St::store(blk.f, base + v, f);
    const V2 fs = St::load(blk.f, base + v);  // moments of f as stored
    m[0] += fs.x;
    m[1] += e.x * fs.x;
    m[2] += e.y * fs.x;
    m[3] += 0.5 * ((e.x * e.x + e.y * e.y) * fs.x + fs.y);
  }
  // calcMacro
  block_sum<4>(m, scratch);
  const P4 mom = p4(m[0], m[1], m[2], m[3]);
  prim = to_primary(d, mom);
  // calcQ
  double q[2] = {0.0, 0.0};
  for (int v = threadIdx.x; v < d.Nv; v += FT) {
    const V2 f = St::load(blk.f, base + v);
    const V2 e = quad_at(d, v);
    const double cx = e.x - prim.s1, cy = e.y - prim.s2, c2 = cx * cx + cy * cy;
    const double t = c2 * f.x + f.y / d.K;
    q[0] += 0.5 * (cx * t);
    q[1] += 0.5 * (cy * t);
  }
  block_sum<2>(q, scratch);
  if (threadIdx.x == 0) {
    st4(blk.macro, midx(d, mi, mj), prim);
    st4(blk.cell_mom, gidx(d, mi + d.ghost, mj + d.ghost), mom);
    st2(blk.Q, midx(d, mi, mj), v2(q[0], q[1]));
    st2(blk.Q_next, midx(d, mi, mj), v2(q[0], q[1]));
    const double fq = cfl_freq(blk, prim, mi, mj);
    atomicMax(&sol.max_freq, (unsigned long long)__double_as_longlong(fq));
  }
}

// restart from saved f, macro and Q (initFunctions with a restart file and
// f present, ugks_block.py:274-300, 347-349): f and macro stay as loaded; the
// fused path's own per-cell state is rebuilt from them (the moments of f for
// the face pass, calcQ of f with the macro for the next cell pass) and the CFL
// frequency of every cell is taken as at start-up (calcTimeStep)
template <typename T>
__global__ void __launch_bounds__(FT) restart_cells(const ugks_fused_block *__restrict__ B, int nb,
                                                    ugks_solve_state *__restrict__ solves) {
  __shared__ double scratch[6 * (FT / 32)];
  using St = Store<T>;
  const int w = blockIdx.x;
  const int bi = find_block<1>(B, nb, w);
  const ugks_fused_block &blk = B[bi];
  const ugks_block_desc &d = blk.d;
  UGKS_CHECK_ITEM(1, blk, w, solves);
  ugks_solve_state &sol = solves[blk.solve];
  if (!sol.active) return;
  const int lc = w - blk.cell_begin;
  const long mi = lc / d.nj, mj = lc % d.nj;
  const size_t base = fidx(d, mi + d.ghost, mj + d.ghost, 0);
  const P4 prim = ld4(blk.macro, midx(d, mi, mj));
  const double Kinv = 1.0 / d.K;
  double m[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int v = threadIdx.x; v < d.Nv; v += FT) {
    const V2 f = St::load(blk.f, base + v);
    const V2 e = quad_at(d, v);
    m[0] += f.x;
    m[1] = fma(e.x, f.x, m[1]);
    m[2] = fma(e.y, f.x, m[2]);
    m[3] += fma(fma(e.x, e.x, e.y * e.y), f.x, f.y);
    const double cx = e.x - prim.s1, cy = e.y - prim.s2;
    const double t = fma(fma(cx, cx, cy * cy), f.x, f.y * Kinv);
    m[4] = fma(cx, t, m[4]);
    m[5] = fma(cy, t, m[5]);
  }
  block_sum<6>(m, scratch);
  if (threadIdx.x == 0) {
    st4(blk.cell_mom, gidx(d, mi + d.ghost, mj + d.ghost), p4(m[0], m[1], m[2], 0.5 * m[3]));
    st2(blk.Q_next, midx(d, mi, mj), v2(0.5 * m[4], 0.5 * m[5]));
    const double fq = cfl_freq(blk, prim, mi, mj);
    atomicMax(&sol.max_freq, (unsigned long long)__double_as_longlong(fq));
  }
}

// paraBC (clKernel.c:141-218) for constant wall values, every block
__global__ void init_walls(const ugks_fused_block *B, int nb) {
  const ugks_fused_block &blk = B[blockIdx.x];
  const ugks_block_desc &d = blk.d;
  const int wl = max(d.ni, d.nj);
  for (int ci = threadIdx.x; ci < wl; ci += blockDim.x)
    for (int f = 0; f < 4; ++f) {
      const bool ns = (f == GNORTH || f == GSOUTH);
      if (ns ? !(ci < d.ni) : !(ci < d.nj)) continue;
      const double l = (d.wall_P[f] != -1) ? d.wall_P[f] / d.wall_D[f] : d.wall_T[f];
      st4(blk.wall_prop, ci * 4 + f, p4(d.wall_D[f], d.wall_U[f], d.wall_V[f], l));
    }
}

// calcTimeStep + updateTimeStep(limit=False) at start-up
__global__ void dt_init(ugks_solve_state *solves, int ns) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  ugks_solve_state &x = solves[s];
  if (!x.active) return;
  x.max_dt = x.CFL / __longlong_as_double((long long)x.max_freq);
  if (x.dt != x.max_dt) x.dt = x.max_dt;
  x.max_freq = 0ull;
  x.retry = 0;
}

// the mixed-precision (FP32 deviation) kernels
#include "ugks_delta.cuh"

// the ghost update of every block of the table
template <typename T>
void launch_ghosts(const ugks_fused_block *B, int nb, const ugks_fused_sizes *z, ugks_solve_state *solves,
                   cudaStream_t st) {
  if (!z->n_ghost) return;
  if (std::is_same<T, float>::value) ghost_pass_delta<<<z->n_ghost, FT, 0, st>>>(B, nb, solves);
  else ghost_pass<double><<<z->n_ghost, FT, 0, st>>>(B, nb, solves);
}

template <typename T>
int init_impl(const ugks_fused_block *B, int nb, const ugks_fused_sizes *z, ugks_solve_state *solves,
              int ns, void *stream) {
  cudaStream_t st = S(stream);
  init_walls<<<nb, 128, 0, st>>>(B, nb);
  if (z->n_faces) face_geometry<<<(z->n_faces + 127) / 128, 128, 0, st>>>(B, nb, z->n_faces);
  if (z->n_cells) {
    if (std::is_same<T, float>::value) setup_cells_delta<true><<<z->n_cells, FT, 0, st>>>(B, nb, solves);
    else init_cells<double><<<z->n_cells, FT, 0, st>>>(B, nb, solves);
  }
  dt_init<<<(ns + 127) / 128, 128, 0, st>>>(solves, ns);
  launch_ghosts<T>(B, nb, z, solves, st);
  return launch_status();
}

template <typename T>
int restart_impl(const ugks_fused_block *B, int nb, const ugks_fused_sizes *z, ugks_solve_state *solves,
                 int ns, void *stream) {
  cudaStream_t st = S(stream);
  init_walls<<<nb, 128, 0, st>>>(B, nb);
  if (z->n_faces) face_geometry<<<(z->n_faces + 127) / 128, 128, 0, st>>>(B, nb, z->n_faces);
  if (z->n_cells) {
    if (std::is_same<T, float>::value) setup_cells_delta<false><<<z->n_cells, FT, 0, st>>>(B, nb, solves);
    else restart_cells<double><<<z->n_cells, FT, 0, st>>>(B, nb, solves);
  }
  dt_init<<<(ns + 127) / 128, 128, 0, st>>>(solves, ns);
  launch_ghosts<T>(B, nb, z, solves, st);
  return launch_status();
}

template <typename T, int FM, int MINB, int NT>
cudaError_t set_face_attributes() {
  cudaError_t e = cudaFuncSetAttribute(face_pass<T, FM, MINB, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       200 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(face_retry<T, FM, MINB, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(face_pass<T, FM, MINB, NT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
  return e;
}

template <typename T, int V>
cudaError_t set_face_shape() {
  constexpr int NT = FaceShape<T, V>::nt, MINB = FaceShape<T, V>::minb;
  if constexpr (std::is_same<T, float>::value) {
    return cudaSuccess;  // mixed: no face_pass (set_wall_attributes covers its retry pass)
  } else {
    cudaError_t e = set_face_attributes<T, 0, MINB, NT>();
    if (e == cudaSuccess) e = set_face_attributes<T, 1, MINB, NT>();
    if (e == cudaSuccess) e = set_face_attributes<T, 3, MINB, NT>();
    return e;
  }
}
template <typename T>
cudaError_t set_wall_attributes() {
  if constexpr (std::is_same<T, float>::value) {
    // the wall launch and the retry pass's wall faces (both budgets)
    cudaError_t e =
        cudaFuncSetAttribute(wall_pass_delta<WALL_NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    constexpr int NN = FT, NW = FaceBudget<float>::wide_threads;
    constexpr int MN = FaceBudget<float>::narrow, MW = FaceBudget<float>::wide;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(face_retry<float, 0, MN, NN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(face_retry<float, 1, MN, NN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(face_retry<float, 3, MN, NN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(face_retry<float, 0, MW, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(face_retry<float, 1, MW, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(face_retry<float, 3, MW, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    return e;
  }
  return cudaSuccess;
}
template <typename T>
cudaError_t set_flux_attributes() {
  if constexpr (std::is_same<T, float>::value) {
    cudaError_t e = cudaFuncSetAttribute(face_flux_tma<FLUX_WPC, FLUX_TMA_MINB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(face_flux_tma<FLUX_WPC, FLUX_TMA_MINB>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               cudaSharedmemCarveoutMaxShared);
    return e;
  }
  return cudaSuccess;
}
template <typename T, int MINB>
cudaError_t set_cell_attributes() {
  if (std::is_same<T, float>::value)
    return cudaFuncSetAttribute(cell_pass_delta<MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  return cudaFuncSetAttribute(cell_pass<double, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

// Kernel attributes (the dynamic shared memory above 48 KB that the face and
// cell passes of large velocity grids need) hold per device: they are set
// once for each device a step runs on, with that device current.
constexpr int kMaxDevices = 64;

// The mixed step's wall launch needs only this step's f and writes only wall
// faces, so it runs on a side stream beside the interior moments sweep: a
// fork and a join by events, which stream capture turns into graph edges.
// One side stream per device, created with the device's kernel attributes
// (before any capture: ugks_prepare); `lock` keeps the record-wait pairs of
// concurrent host threads from interleaving.
struct WallStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  std::mutex lock;
};
inline WallStream &wall_stream(int dev) {
  static WallStream ws[kMaxDevices];
  return ws[dev];
}
inline cudaError_t make_wall_stream(int dev) {
  WallStream &w = wall_stream(dev);
  if (w.s) return cudaSuccess;
  cudaError_t e = cudaStreamCreateWithFlags(&w.s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w.fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w.join, cudaEventDisableTiming);
  return e;
}

template <typename T>
cudaError_t set_step_attributes() {
  static std::mutex lock;
  static bool done[kMaxDevices] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> guard(lock);
  if (done[dev]) return cudaSuccess;
  cudaError_t r[8] = {
      set_face_shape<T, 1>(), set_face_shape<T, 2>(), set_face_shape<T, 3>(), set_face_shape<T, 4>(),
      set_cell_attributes<T, 2>(), set_cell_attributes<T, 3>(), set_wall_attributes<T>(), set_flux_attributes<T>()};
  for (cudaError_t x : r)
    if (x != cudaSuccess) return x;
  if (std::is_same<T, float>::value) {
    e = make_wall_stream(dev);
    if (e != cudaSuccess) return e;
  }
  done[dev] = true;
  return cudaSuccess;
}

// shared memory of a face CTA: FP64, (h, b) and slopes per velocity + axis
// tables; mixed, the wall procedure's FP64 face values (retry pass; the
// mixed main pass sizes its warp sweeps itself)
template <typename T>
inline size_t face_smem(int max_nv, int max_axes, bool retry = false) {
  if (std::is_same<T, float>::value) return retry ? delta_wall_smem(max_nv) : 0;
  return 4 * sizeof(double) * (size_t)max_nv + sizeof(double) * (size_t)max_axes;
}

// the main face pass of one segment (one flux method, one register budget)
template <typename T, int MINB, int NT>
void launch_segment(const ugks_fused_block *B, int nb, ugks_solve_state *solves, int method, int first,
                    int count, size_t smem, cudaStream_t st) {
  switch (method) {
    case 0: face_pass<T, 0, MINB, NT><<<count, NT, smem, st>>>(B, nb, solves, first); break;
    case 1: face_pass<T, 1, MINB, NT><<<count, NT, smem, st>>>(B, nb, solves, first); break;
    case 3: face_pass<T, 3, MINB, NT><<<count, NT, smem, st>>>(B, nb, solves, first); break;
    default: break;
  }
}

// the retry pass of every flux method (per solve; rare)
template <typename T, int MINB, int NT>
void launch_retry(const ugks_fused_block *B, int nb, const ugks_fused_sizes *z, ugks_solve_state *solves,
                  int ns, size_t smem, cudaStream_t st) {
  const unsigned rg = (unsigned)ns * RETRY_CTAS;
  if (z->face_count[0]) face_retry<T, 0, MINB, NT><<<rg, NT, smem, st>>>(B, nb, solves, ns);
  if (z->face_count[1]) face_retry<T, 1, MINB, NT><<<rg, NT, smem, st>>>(B, nb, solves, ns);
  if (z->face_count[3]) face_retry<T, 3, MINB, NT><<<rg, NT, smem, st>>>(B, nb, solves, ns);
}

// the mixed moments sweep of one segment, in launch shape v (ugks_fused_sizes.seg_variant)
template <int WPC, int MINB>
void launch_moments_shape(const ugks_fused_block *B, int nb, ugks_solve_state *solves, int method, int first,
                          int count, int axes, cudaStream_t st) {
  const int ws = delta_moments_stride(axes);
  const unsigned g = (unsigned)((count + WPC - 1) / WPC);
  const size_t sm = (size_t)WPC * ws * sizeof(double);
  switch (method) {
    case 0: face_moments_warp<0, WPC, MINB><<<g, WPC * 32, sm, st>>>(B, nb, solves, first, count, ws); break;
    case 1: face_moments_warp<1, WPC, MINB><<<g, WPC * 32, sm, st>>>(B, nb, solves, first, count, ws); break;
    case 3: face_moments_warp<3, WPC, MINB><<<g, WPC * 32, sm, st>>>(B, nb, solves, first, count, ws); break;
    default: break;
  }
}
inline void launch_moments(int v, const ugks_fused_block *B, int nb, ugks_solve_state *solves, int method,
                           int first, int count, int axes, cudaStream_t st) {
  switch (v) {
    case 2: launch_moments_shape<MomentsShape<2>::wpc, MomentsShape<2>::minb>(B, nb, solves, method, first, count, axes, st); break;
    case 3: launch_moments_shape<MomentsShape<3>::wpc, MomentsShape<3>::minb>(B, nb, solves, method, first, count, axes, st); break;
    case 4: launch_moments_shape<MomentsShape<4>::wpc, MomentsShape<4>::minb>(B, nb, solves, method, first, count, axes, st); break;
    default: launch_moments_shape<MomentsShape<1>::wpc, MomentsShape<1>::minb>(B, nb, solves, method, first, count, axes, st); break;
  }
}

// NVTX range over a phase's launches on the host timeline (a profiler shows
// them beside the kernels; without one attached a range costs a few ns)
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

template <typename T>
int step_impl(const ugks_fused_block *B, int nb, const ugks_fused_sizes *z, ugks_solve_state *solves,
              int ns, void *stream, void *const *events = nullptr) {
  cudaStream_t st = S(stream);
  // face pass: (h, b) and slopes per velocity + the two axis factor tables;
  // cell pass: the axis factor tables of the old and new macro state
  const size_t smem = face_smem<T>(z->max_nv, z->max_axes, true);
  constexpr bool mixed = std::is_same<T, float>::value;
  // doubles of shared memory per cell warp
  const int cstride = mixed ? delta_cell_stride(z->max_axes) : 2 * z->max_axes + CELL_COEF;
  const size_t csmem = (size_t)CW * cstride * sizeof(double) + (mixed ? 0 : (size_t)CW * cell_ring_bytes<T>());
  const cudaError_t attr = set_step_attributes<T>();
  if (attr != cudaSuccess) return -(int)attr;
  if (smem > 200 * 1024 || csmem > 200 * 1024) return -(int)cudaErrorInvalidValue;
  const unsigned sg = (unsigned)((ns + 127) / 128);
  auto mark = [&](int k) {
    if (events && events[k]) cudaEventRecord(reinterpret_cast<cudaEvent_t>(events[k]), st);
  };
  // NVTX: the step, and within it the face, cell and ghost phases
  NvtxRange step_range(mixed ? "ugks step (mixed)" : "ugks step (fp64)");
  std::optional<NvtxRange> phase;
  phase.emplace("ugks face pass");
  mark(0);
  // mixed: the wall faces on the device's side stream, beside the segments
  WallStream *ws = nullptr;
  std::unique_lock<std::mutex> ws_guard;
  if (mixed && z->n_wall) {
    int dev = 0;
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return -(int)e;
    ws = &wall_stream(dev);
    ws_guard = std::unique_lock<std::mutex>(ws->lock);
    cudaEventRecord(ws->fork, st);
    cudaStreamWaitEvent(ws->s, ws->fork, 0);
    wall_pass_delta<WALL_NT><<<(unsigned)z->n_wall, WALL_NT, delta_wall_smem(z->max_nv), ws->s>>>(B, nb, solves);
    cudaEventRecord(ws->join, ws->s);
  }
  for (int k = 0; k < z->n_segments && k < UGKS_MAX_FACE_SEGMENTS; ++k) {
    if (z->seg_count[k] <= 0) continue;
    const size_t sm = face_smem<T>(z->seg_max_nv[k], z->seg_max_axes[k]);
    int v = z->seg_variant[k];
    const int m = z->seg_method[k], b0 = z->seg_begin[k], n = z->seg_count[k];
    if constexpr (mixed) {
      if (v <= 0 || v > 4) v = 1;
      launch_moments(v, B, nb, solves, m, b0, n, z->seg_max_axes[k], st);
    } else {
      if (v <= 0 || v > 4) v = z->seg_max_nv[k] <= FaceBudget<T>::narrow_max_nv ? 1 : 4;
      switch (v) {
        case 1: launch_segment<T, FaceShape<T, 1>::minb, FaceShape<T, 1>::nt>(B, nb, solves, m, b0, n, sm, st); break;
        case 2: launch_segment<T, FaceShape<T, 2>::minb, FaceShape<T, 2>::nt>(B, nb, solves, m, b0, n, sm, st); break;
        case 3: launch_segment<T, FaceShape<T, 3>::minb, FaceShape<T, 3>::nt>(B, nb, solves, m, b0, n, sm, st); break;
        default: launch_segment<T, FaceShape<T, 4>::minb, FaceShape<T, 4>::nt>(B, nb, solves, m, b0, n, sm, st); break;
      }
    }
  }
  if (ws) {
    cudaStreamWaitEvent(st, ws->join, 0);
    ws_guard.unlock();
  }
  const bool narrow = z->max_nv <= FaceBudget<T>::narrow_max_nv;
  // mixed: the interior faces' coefficient and flux launches follow the first
  // dt check (they use its dt), and the events bracket all of the face pass
  if (!mixed) mark(1);
  dt_check<<<sg, 128, 0, st>>>(solves, ns, 0);
  if (!mixed) mark(2);
  if (narrow) launch_retry<T, FaceBudget<T>::narrow, FT>(B, nb, z, solves, ns, smem, st);
  else launch_retry<T, FaceBudget<T>::wide, FaceBudget<T>::wide_threads>(B, nb, z, solves, ns, smem, st);
  if (mixed && z->n_faces) {
    face_coef_delta<<<(unsigned)((z->n_faces + 127) / 128), 128, 0, st>>>(B, nb, solves, z->n_faces);
    if (UGKS_FLUX_TMA) {
      const int wb = (int)flux_tma_warp_bytes(z->max_axes);
      face_flux_tma<FLUX_WPC, FLUX_TMA_MINB><<<(unsigned)((z->n_faces + FLUX_WPC - 1) / FLUX_WPC), FLUX_WPC * 32,
                                               (size_t)FLUX_WPC * wb, st>>>(B, nb, solves, z->n_faces, wb);
    } else {
      const int fs = delta_flux_stride(z->max_axes);
      face_flux_warp<FLUX_WPC, FLUX_MINB><<<(unsigned)((z->n_faces + FLUX_WPC - 1) / FLUX_WPC), FLUX_WPC * 32,
                                            (size_t)FLUX_WPC * fs * sizeof(double), st>>>(B, nb, solves, z->n_faces, fs);
    }
  }
  if (mixed) {
    mark(1);
    mark(2);
  }
  mark(3);
  phase.reset();
  dt_check<<<sg, 128, 0, st>>>(solves, ns, 1);
  mark(4);
  phase.emplace("ugks cell pass");
  if (z->n_cells) {
    // cell_variant: 0 the default register budget, 2 or 3 CTAs of 8 warps per SM
    const unsigned cg = (unsigned)((z->n_cells + CW - 1) / CW);
    const int cv = z->cell_variant == 2 || z->cell_variant == 3 ? z->cell_variant : CellBudget<T>::minb;
    if (mixed) {
      if (cv == 3) cell_pass_delta<3><<<cg, CW * 32, csmem, st>>>(B, nb, solves, z->n_cells, cstride);
      else cell_pass_delta<2><<<cg, CW * 32, csmem, st>>>(B, nb, solves, z->n_cells, cstride);
    } else {
      if (cv == 3) cell_pass<double, 3><<<cg, CW * 32, csmem, st>>>(B, nb, solves, z->n_cells, cstride);
      else cell_pass<double, 2><<<cg, CW * 32, csmem, st>>>(B, nb, solves, z->n_cells, cstride);
    }
  }
  mark(5);
  phase.reset();
  dt_update<<<sg, 128, 0, st>>>(solves, ns);
  mark(6);
  phase.emplace("ugks ghost pass");
  launch_ghosts<T>(B, nb, z, solves, st);
  mark(7);
  return launch_status();
}

// residual (getResidual, clUGKS.c:1259-1277, and ugks_block.py:1316-1327):
// one CTA per solve walks its blocks
__global__ void residual_kernel(const ugks_fused_block *B, int nb, ugks_solve_state *solves, int ns) {
  __shared__ double scratch[8 * (FT / 32)];
  const int s = blockIdx.x;
  if (s >= ns || !solves[s].active) return;  // a stopped solve keeps its last residual
  double r[4] = {0.0, 0.0, 0.0, 0.0};
  int n = 0;
  for (int b = 0; b < nb; ++b) {
    if (B[b].solve != s) continue;
    const ugks_fused_block &blk = B[b];
    const int cells = blk.d.ni * blk.d.nj;
    double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = threadIdx.x; c < cells; c += blockDim.x) {
      const P4 p = ld4(blk.macro, c), o = ld4(blk.prim_old, c);
      a[0] += (p.s0 - o.s0) * (p.s0 - o.s0);
      a[1] += (p.s1 - o.s1) * (p.s1 - o.s1);
      a[2] += (p.s2 - o.s2) * (p.s2 - o.s2);
      a[3] += (p.s3 - o.s3) * (p.s3 - o.s3);
      a[4] += fabs(p.s0);
      a[5] += fabs(p.s1);
      a[6] += fabs(p.s2);
      a[7] += fabs(p.s3);
    }
    block_sum<8>(a, scratch);
    for (int k = 0; k < 4; ++k) {
      const double v = sqrt((double)cells * a[k]) / (a[4 + k] + DBL_MIN);
      r[k] += v <= 0.0 ? 1.0 : v;
    }
    ++n;
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) solves[s].residual[k] = n ? r[k] / n : 0.0;
}

// The bounded wait of the face pass's bulk copies, exercised on its own: a
// warp arms an mbarrier for 512 bytes and copies them from `src` (global, 16-
// byte aligned), or, with src null, never does; it then waits at most `polls`
// times and writes 0 when the copy completed, STATUS_COPY_TIMEOUT when the
// wait ran out (what the face pass writes into a solve's status)
__global__ void copy_wait_check(const float4 *src, unsigned polls, int *status) {
  __shared__ __align__(128) float4 buf[32];
  __shared__ __align__(8) uint64_t bar;
  const int lane = threadIdx.x & 31;
  if (lane == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
    mbar_arrive_expect_tx(&bar, 512u);
    if (src) bulk_g2s(buf, src, 512u, &bar);
  }
  __syncwarp();
  const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar, 0u, polls));
  // the copied values read back (a lane's float4 must equal the source's)
  const bool same = ok && src ? __all_sync(0xffffffffu, buf[lane].x == src[lane].x && buf[lane].w == src[lane].w)
                              : true;
  if (lane == 0) *status = !ok ? STATUS_COPY_TIMEOUT : (same ? 0 : -1);
}

// the stop rule of every active solve (ugks_stop_check)
__global__ void stop_check(ugks_solve_state *solves, int ns) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  ugks_solve_state &x = solves[s];
  if (!x.active) return;
  int why = 0;
  if (x.status != 0) why = UGKS_STOP_ERROR;
  else if (x.stop_residual > 0.0 && x.steps >= x.stop_after && x.residual[0] < x.stop_residual)
    why = UGKS_STOP_CONVERGED;
  else if (x.stop_steps > 0 && x.steps >= x.stop_steps) why = UGKS_STOP_STEPS;
  if (why) {
    x.stopped = why;
    x.active = 0;
  }
}

}  // namespace

extern "C" {

int ugks_step_fp64(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                   ugks_solve_state *solves_dev, int nsolves, void *stream) {
  return step_impl<double>(blocks_dev, nblocks, sizes, solves_dev, nsolves, stream);
}
int ugks_step_mixed(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                    ugks_solve_state *solves_dev, int nsolves, void *stream) {
  return step_impl<float>(blocks_dev, nblocks, sizes, solves_dev, nsolves, stream);
}
int ugks_step_profiled(int mixed, const ugks_fused_block *blocks_dev, int nblocks,
                       const ugks_fused_sizes *sizes, ugks_solve_state *solves_dev, int nsolves,
                       void *const *events, void *stream) {
  return mixed ? step_impl<float>(blocks_dev, nblocks, sizes, solves_dev, nsolves, stream, events)
               : step_impl<double>(blocks_dev, nblocks, sizes, solves_dev, nsolves, stream, events);
}
int ugks_step_launches(const ugks_fused_sizes *z, int mixed) {
  int n = 0;
  if (mixed && z->n_faces) n += 2;  // the mixed face pass's coefficient and flux launches
  if (mixed && z->n_wall) n += 1;   // and its wall launch
  for (int k = 0; k < z->n_segments && k < UGKS_MAX_FACE_SEGMENTS; ++k) n += z->seg_count[k] > 0 ? 1 : 0;
  for (int m = 0; m < 4; ++m) n += z->face_count[m] > 0 ? 1 : 0;  // retry passes
  n += 2;                                                          // dt checks
  n += z->n_cells ? 1 : 0;
  n += 1;                                                          // dt update
  n += z->n_ghost ? 1 : 0;
  return n;
}

int ugks_residual(const ugks_fused_block *blocks_dev, int nblocks, ugks_solve_state *solves_dev,
                  int nsolves, void *stream) {
  if (nsolves <= 0) return 0;
  residual_kernel<<<nsolves, FT, 0, S(stream)>>>(blocks_dev, nblocks, solves_dev, nsolves);
  return launch_status();
}

int ugks_stop_check(ugks_solve_state *solves_dev, int nsolves, void *stream) {
  if (nsolves <= 0) return 0;
  stop_check<<<(nsolves + 127) / 128, 128, 0, S(stream)>>>(solves_dev, nsolves);
  return launch_status();
}

int ugks_serve_steps(int mixed, const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                     ugks_solve_state *solves_dev, int nsolves, int nsteps, void *stream) {
  for (int k = 0; k < nsteps; ++k) {
    int rc = mixed ? step_impl<float>(blocks_dev, nblocks, sizes, solves_dev, nsolves, stream)
                   : step_impl<double>(blocks_dev, nblocks, sizes, solves_dev, nsolves, stream);
    if (rc == 0) rc = ugks_residual(blocks_dev, nblocks, solves_dev, nsolves, stream);
    if (rc == 0) rc = ugks_stop_check(solves_dev, nsolves, stream);
    if (rc != 0) return rc;
  }
  return 0;
}

int ugks_check_copy_wait(const void *src_dev, unsigned polls, int *status_dev, void *stream) {
  copy_wait_check<<<1, 32, 0, S(stream)>>>(reinterpret_cast<const float4 *>(src_dev), polls, status_dev);
  return launch_status();
}

int ugks_prepare(int mixed) {
  const cudaError_t e = mixed ? set_step_attributes<float>() : set_step_attributes<double>();
  return e == cudaSuccess ? 0 : -(int)e;
}

// A block the fused kernels can index safely: sizes consistent with the
// ghost layers the flux method's stencil needs, the arrays every pass
// touches present, block connections inside the table and on a face of the
// same extent.  (A corrupted entry would otherwise send a kernel outside its
// arrays: the table is rejected on the host before any launch.)
static bool block_valid(const ugks_fused_block *blocks, int nblocks, int b) {
  const ugks_fused_block &x = blocks[b];
  const ugks_block_desc &d = x.d;
  const int need = d.flux_method == 1 ? 3 : 2;  // stencil half-width of WENO5 / vanLeer, minmod
  if (d.ni <= 0 || d.nj <= 0 || d.Nv <= 0 || d.ghost < need) return false;
  if (d.Ni != d.ni + 2 * d.ghost || d.Nj != d.nj + 2 * d.ghost) return false;
  if (d.u_num < 0 || d.v_num < 0 || (d.u_num > 0 && (int64_t)d.u_num * d.v_num != d.Nv)) return false;
  if (!d.quad || !d.weight || !d.mirror_NS || !d.mirror_EW || !d.mirror_D) return false;
  if (!x.f || !x.flux_S || !x.flux_W || !x.flux_macro_S || !x.flux_macro_W || !x.macro || !x.Q || !x.prim_old ||
      !x.area || !x.centre || !x.mid_side || !x.normal || !x.side_length || !x.xy || !x.cell_mom || !x.Q_next ||
      !x.face_geo || !x.wall_prop || !x.wall_cover || !x.wall_fluxes || !x.wall_dist)
    return false;
  for (int f = 0; f < 4; ++f) {
    if (x.bc_type[f] < BC_ADJACENT || x.bc_type[f] > BC_BOUNCE_BACK) return false;
    if (x.bc_type[f] == BC_ADJACENT || x.bc_type[f] == BC_PERIODIC) {
      const int o = x.bc_block[f], of = x.bc_face[f];
      if (o < 0 || o >= nblocks || of < 0 || of > 3) return false;
      const ugks_block_desc &od = blocks[o].d;
      const int n_here = (f == GNORTH || f == GSOUTH) ? d.ni : d.nj;
      const int n_there = (of == GNORTH || of == GSOUTH) ? od.ni : od.nj;
      if (n_here != n_there || od.Nv != d.Nv || od.ghost != d.ghost || blocks[o].solve != x.solve) return false;
    }
  }
  return true;
}

int ugks_fused_layout(ugks_fused_block *blocks, int nblocks, ugks_fused_sizes *z) {
  if (nblocks < 0 || (nblocks > 0 && !blocks) || !z) return -3;
  for (int b = 0; b < nblocks; ++b)
    if (!block_valid(blocks, nblocks, b)) return -3;
  int64_t f = 0, c = 0, g = 0, wl = 0;
  int32_t max_nv = 0, max_axes = 0;
  int64_t fb[4] = {0, 0, 0, 0}, fc[4] = {0, 0, 0, 0};
  struct Run {
    int method, nv, max_nv, axes;
    int64_t begin, count;
  };
  std::vector<Run> runs;
  int last_method = -1, seen = 0, last_solve = -1;
  for (int b = 0; b < nblocks; ++b) {
    ugks_fused_block &x = blocks[b];
    const int m = x.d.flux_method;
    if (m < 0 || m > 3) return -2;
    if (m != last_method) {
      if (seen & (1 << m)) return -2;  // methods must be contiguous
      seen |= 1 << m;
      fb[m] = f;
      last_method = m;
    }
    if (x.solve != last_solve) {
      if (x.solve != last_solve + 1) return -2;  // solves contiguous and in order
      last_solve = x.solve;
    }
    x.face_begin = (int32_t)f;
    x.cell_begin = (int32_t)c;
    x.ghost_begin = (int32_t)g;
    x.wall_begin = (int32_t)wl;
    wl += 2ll * (x.d.ni + x.d.nj);
    const int64_t nf = 2ll * (x.d.ni + 1) * (x.d.nj + 1);
    const int axes_b = (x.d.u_num > 0 && x.d.u_num * x.d.v_num == x.d.Nv && x.d.u_num + x.d.v_num <= 512)
                           ? x.d.u_num + x.d.v_num : 0;
    if (runs.empty() || runs.back().method != m || runs.back().nv != x.d.Nv)
      runs.push_back(Run{m, x.d.Nv, x.d.Nv, axes_b, f, 0});
    runs.back().count += nf;
    runs.back().axes = std::max(runs.back().axes, axes_b);
    f += nf;
    fc[m] += nf;
    c += (int64_t)x.d.ni * x.d.nj;
    g += 2ll * x.d.ghost * (x.d.ni + x.d.nj);
    if (x.d.Nv > max_nv) max_nv = x.d.Nv;
    const int axes = x.d.u_num + x.d.v_num;
    if (x.d.u_num > 0 && x.d.u_num * x.d.v_num == x.d.Nv && axes <= 512 && axes > max_axes) max_axes = axes;
  }
  if (f > INT32_MAX || c > INT32_MAX || g > INT32_MAX || wl > INT32_MAX) return -1;
  z->n_wall = (int32_t)wl;
  z->n_faces = (int32_t)f;
  z->n_cells = (int32_t)c;
  z->n_ghost = (int32_t)g;
  z->max_nv = max_nv;
  z->max_axes = max_axes;
  // at most UGKS_MAX_FACE_SEGMENTS launches: merge the adjacent pair of one
  // method whose merged Nv is smallest (methods are contiguous, so this ends
  // at one run per method at worst)
  while ((int)runs.size() > UGKS_MAX_FACE_SEGMENTS) {
    int best = -1;
    for (int k = 0; k + 1 < (int)runs.size(); ++k)
      if (runs[k].method == runs[k + 1].method &&
          (best < 0 || std::max(runs[k].max_nv, runs[k + 1].max_nv) <
                           std::max(runs[best].max_nv, runs[best + 1].max_nv)))
        best = k;
    if (best < 0) return -2;
    runs[best].max_nv = std::max(runs[best].max_nv, runs[best + 1].max_nv);
    runs[best].axes = std::max(runs[best].axes, runs[best + 1].axes);
    runs[best].count += runs[best + 1].count;
    runs.erase(runs.begin() + best + 1);
  }
  z->n_segments = (int32_t)runs.size();
  for (int k = 0; k < UGKS_MAX_FACE_SEGMENTS; ++k) {
    const bool on = k < (int)runs.size();
    z->seg_begin[k] = on ? (int32_t)runs[k].begin : 0;
    z->seg_count[k] = on ? (int32_t)runs[k].count : 0;
    z->seg_method[k] = on ? runs[k].method : 0;
    z->seg_max_nv[k] = on ? runs[k].max_nv : 0;
    z->seg_max_axes[k] = on ? runs[k].axes : 0;
  }
  for (int m = 0; m < 4; ++m) {
    z->face_begin[m] = (int32_t)fb[m];
    z->face_count[m] = (int32_t)fc[m];
  }
  for (int k = 0; k < UGKS_MAX_FACE_SEGMENTS; ++k) z->seg_variant[k] = 0;
  z->cell_variant = 0;
  return 0;
}

int ugks_init_fp64(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                   ugks_solve_state *solves_dev, int nsolves, void *stream) {
  return init_impl<double>(blocks_dev, nblocks, sizes, solves_dev, nsolves, stream);
}
int ugks_init_mixed(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                    ugks_solve_state *solves_dev, int nsolves, void *stream) {
  return init_impl<float>(blocks_dev, nblocks, sizes, solves_dev, nsolves, stream);
}
int ugks_restart_fp64(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                      ugks_solve_state *solves_dev, int nsolves, void *stream) {
  return restart_impl<double>(blocks_dev, nblocks, sizes, solves_dev, nsolves, stream);
}
int ugks_restart_mixed(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                       ugks_solve_state *solves_dev, int nsolves, void *stream) {
  return restart_impl<float>(blocks_dev, nblocks, sizes, solves_dev, nsolves, stream);
}

}  // extern "C"
