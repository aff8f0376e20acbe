// ugks_delta.cuh -- the mixed-precision fused step.
//
// Included by ugks_fused.cu inside its anonymous namespace: it uses that
// file's work lists, face coefficient block, wall procedure and dt kernels.
//
// Storage.  f and the two face-flux arrays hold FP32 *deviations* from a
// reference Maxwellian M of the solve (density rho0 and temperature T0 at
// rest, weighted by the quadrature like f):
//   f    = M + df,
//   flux = dt len (u . n) M + dflux,
// so FP32 rounds only the deviations, never the O(1) equilibrium part.  Both
// are exact rewritings of the FP64 scheme:
//   * reconstruction (vanLeer / WENO5 / minmod) works on differences of
//     neighbouring cells, in which M cancels, so the face deviation is the
//     reconstruction of df;
//   * for a uniform equilibrium state the UGKS flux is exactly
//     dt u M (Mt0 + Mt3 = dt), and the dt len (u . n) M parts of a cell's four
//     faces cancel (the edge normals times lengths of a closed quadrilateral
//     sum to zero), so the cell update needs only the deviation fluxes;
//   * the update weights of UGKS_update satisfy a1 + a3 + a4 = 1, so
//     df' = a1 df + a2 sum(dflux) + a3 (fEQ_new - M) + a4 (fEQ_old - M).
// Differences of two Maxwellians, g - M = M ((1 + a)(1 + b) - 1), are formed
// from per-axis tables a = expm1(x_u + ln(P/P0)) and b = expm1(x_v) (x the
// exponent difference along each velocity axis, P the prefactor rho lambda /
// pi), computed in FP64, so that they too are accurate to FP32 relative to
// the difference itself.  Moments of f are the reference's moments (FP64
// constants of the velocity grid) plus the moments of df; the sums over
// velocities of deviation terms run in FP32 within a thread and in FP64
// across threads.  Conserved variables, per-face and per-cell coefficients,
// the relaxation, dt and the residual stay FP64.
//
// Layout: the velocities (iu, jv) of the tensor grid (v = iu v_num + jv) are
// paired along u: pair p = a v_num + jv holds (2a, jv) and (2a + 1, jv), a
// float4 (h, h', b, b'), so that one 16-byte access serves two velocities and
// the arithmetic runs on packed FP32 pairs (f32x2 FMA, sm_100).  The two
// velocities of a pair share v, so on faces whose normal is y they always
// take their upwind stencil from the same side.  NP = ceil(u_num / 2) v_num;
// an odd u_num leaves the second lane of the last pair row as padding, kept at
// 0 (its reference value is 0, so every term of it vanishes).

// ---------------------------------------------------------------------------
// packed FP32 pairs
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 bc2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 lo2(float4 x) { return make_float2(x.x, x.y); }
__device__ __forceinline__ float2 hi2(float4 x) { return make_float2(x.z, x.w); }
__device__ __forceinline__ float4 cat2(float2 a, float2 b) { return make_float4(a.x, a.y, b.x, b.y); }
__device__ __forceinline__ float2 rcp2(float2 x) { return make_float2(frcp(x.x), frcp(x.y)); }

__device__ __forceinline__ int npairs(const ugks_block_desc &d) { return ((d.u_num + 1) >> 1) * d.v_num; }
// pair p of cell (i, j)
__device__ __forceinline__ size_t pidx(const ugks_block_desc &d, long i, long j, int p) {
  return ((size_t)i * d.Nj + (size_t)j) * (size_t)npairs(d) + (size_t)p;
}
// the float of component comp (0 = h, 1 = b) of velocity v (v >= Nv: the
// padding lane) of the cell whose pair 0 is at c
__device__ __forceinline__ float *pair_slot(float4 *c, int v, int vn, int comp) {
  const int iu = v / vn, jv = v - iu * vn;
  return reinterpret_cast<float *>(c + (iu >> 1) * vn + jv) + 2 * comp + (iu & 1);
}
__device__ __forceinline__ float pair_get(const float4 *c, int v, int vn, int comp) {
  return *pair_slot(const_cast<float4 *>(c), v, vn, comp);
}
__device__ __forceinline__ void pair_put(float4 *c, int v, int vn, float h, float b) {
  *pair_slot(c, v, vn, 0) = h;
  *pair_slot(c, v, vn, 1) = b;
}

// ---------------------------------------------------------------------------
// the reference Maxwellian of a solve (ugks_fused_block.ref, UGKS_REF_*)
// ---------------------------------------------------------------------------
enum { RM00, RM10, RM01, RM20, RM11, RM02, RM30, RM21, RM12, RM03, RB00, RB10, RB01, RNMOM };

// Heat flux (calcQ, clKernel.c:480-543) relative to velocity U of a
// distribution given by its raw moments M (the RM* / RB* sums over v of h u^a
// v^b and of b u^a v^b), in the frame of the moments:
//   q = 1/2 sum (c |c|^2 h + c b / K),  c = (u, v) - U.
__device__ __forceinline__ V2 heat_flux_from_moments(const double *M, double K, V2 U) {
  const double Ux = U.x, Uy = U.y;
  const double cx3 = M[RM30] - 3.0 * Ux * M[RM20] + 3.0 * Ux * Ux * M[RM10] - Ux * Ux * Ux * M[RM00] + M[RM12] -
                     2.0 * Uy * M[RM11] + Uy * Uy * M[RM10] - Ux * M[RM02] + 2.0 * Ux * Uy * M[RM01] -
                     Ux * Uy * Uy * M[RM00];
  const double cy3 = M[RM03] - 3.0 * Uy * M[RM02] + 3.0 * Uy * Uy * M[RM01] - Uy * Uy * Uy * M[RM00] + M[RM21] -
                     2.0 * Ux * M[RM11] + Ux * Ux * M[RM01] - Uy * M[RM20] + 2.0 * Ux * Uy * M[RM10] -
                     Uy * Ux * Ux * M[RM00];
  return v2(0.5 * (cx3 + (M[RB10] - Ux * M[RB00]) / K), 0.5 * (cy3 + (M[RB01] - Uy * M[RB00]) / K));
}

struct RefMaxwellian {
  double lam0, P0, kb0;
  const double *mom;  // RNMOM raw moments, global frame
  const double *mh;   // weighted h of M per velocity, FP64
  const double *Au;   // axis factors: mh(iu, jv) ~ Au[iu] Av[jv]
  const double *Av;
};
__device__ __forceinline__ RefMaxwellian ref_of(const ugks_fused_block &blk) {
  const double *r = blk.ref;
  RefMaxwellian m;
  m.lam0 = r[UGKS_REF_LAMBDA];
  m.P0 = r[UGKS_REF_P0];
  m.kb0 = r[UGKS_REF_KB0];
  m.mom = r + UGKS_REF_MOM;
  m.mh = r + UGKS_REF_TAB;
  m.Au = m.mh + blk.d.Nv;
  m.Av = m.Au + blk.d.u_num;
  return m;
}

// ln(g / M) along one velocity axis for a Maxwellian of velocity component c
// and lambda lam against M's lambda0, (lambda0 - lambda) x^2 + 2 lambda x c -
// lambda c^2, plus lnP (the log of the prefactor ratio, on one axis only),
// returned as expm1 of it (FP64)
__device__ __forceinline__ double axis_expm1(double x, double c, double lam, double lam0, double lnP = 0.0) {
  return expm1((lam0 - lam) * (x * x) + 2.0 * lam * x * c - lam * (c * c) + lnP);
}

// (1 + a)(1 + b) - 1 without cancellation (the prefactor ratio P/P0 is folded
// into the u-axis table: a = expm1(x_u + ln(P/P0)))
__device__ __forceinline__ float2 rel_excess(float2 a, float2 b) { return fma2(a, b, add2(a, b)); }

// ---------------------------------------------------------------------------
// reconstruction of a velocity pair (iFace, clUGKS.c:148-194) on the
// deviations: the limiters act on differences, in which M cancels
// ---------------------------------------------------------------------------
// WENO5 (clFunctions.c:266-313) in the difference form of weno5_part with the
// smoothness terms normalised by their sum (the FP32 range), two velocities
// at once; returns the slope times dx as num / den
__device__ __forceinline__ void weno5_pair(const float2 (&S)[5], float2 &num, float2 &den) {
  const float2 D0 = sub2(S[1], S[0]), D1 = sub2(S[2], S[1]), D2 = sub2(S[3], S[2]), D3 = sub2(S[4], S[3]);
  const float2 p0 = sub2(D1, D0), p1 = sub2(D2, D1), p2 = sub2(D3, D2);
  // r0 = 3 D1 - D0 = p0 + 2 D1, r1 = D1 + D2, r2 = D3 - 3 D2 = p2 - 2 D2
  const float2 r0 = fma2(D1, bc2(2.0f), p0), r1 = add2(D1, D2), r2 = fma2(D2, bc2(-2.0f), p2);
  const float2 eps = bc2(12e-16f), c13 = bc2(13.0f), c3 = bc2(3.0f);
  float2 e0 = fma2(mul2(c13, p0), p0, fma2(mul2(c3, r0), r0, eps));
  float2 e1 = fma2(mul2(c13, p1), p1, fma2(mul2(c3, r1), r1, eps));
  float2 e2 = fma2(mul2(c13, p2), p2, fma2(mul2(c3, r2), r2, eps));
  const float2 sc = rcp2(add2(add2(e0, e1), e2));
  e0 = mul2(e0, sc);
  e1 = mul2(e1, sc);
  e2 = mul2(e2, sc);
  const float2 q0 = mul2(e0, e0), q1 = mul2(e1, e1), q2 = mul2(e2, e2);
  const float2 a0 = mul2(q1, q2), a1 = mul2(mul2(bc2(6.0f), q0), q2), a2 = mul2(mul2(c3, q0), q1);
  const float2 f0 = fma2(bc2(-1.0f / 3.0f), D0, mul2(bc2(5.0f / 6.0f), D1));
  const float2 f1 = fma2(bc2(1.0f / 6.0f), D1, mul2(bc2(1.0f / 3.0f), D2));
  const float2 f2 = fma2(bc2(2.0f / 3.0f), D2, mul2(bc2(-1.0f / 6.0f), D3));
  num = fma2(a0, f0, fma2(a1, f1, mul2(a2, f2)));
  den = add2(add2(a0, a1), a2);
}

// slope of one component pair; il / ds / ids: per lane 1 / |c - c'|,
// |mid - c| and 1 / |mid - c|
template <int FM>
__device__ __forceinline__ float2 slope_pair(const float2 (&S)[FM == 1 ? 5 : 3], float2 il, float2 ids) {
  if constexpr (FM == 1) {
    float2 nm, dn;
    weno5_pair(S, nm, dn);
    return mul2(mul2(nm, rcp2(dn)), ids);
  } else if constexpr (FM == 0) {
    // vanLeer (clFunctions.c:255-261) on (S1 - S0) / l and (S2 - S1) / l
    const float2 s1 = mul2(sub2(S[1], S[0]), il), s2 = mul2(sub2(S[2], S[1]), il);
    float2 r;
    r.x = (fsign(s1.x) + fsign(s2.x)) * (fabsf(s1.x) * fabsf(s2.x)) * frcp(fabsf(s1.x) + fabsf(s2.x) + 1e-16f);
    r.y = (fsign(s1.y) + fsign(s2.y)) * (fabsf(s1.y) * fabsf(s2.y)) * frcp(fabsf(s1.y) + fabsf(s2.y) + 1e-16f);
    return r;
  } else {
    // minmod / NND (clFunctions.c:318-353)
    const float2 d2 = sub2(S[2], S[1]), d1 = sub2(S[1], S[0]);
    return mul2(make_float2(0.5f * fminmod(d2.x, d1.x), 0.5f * fminmod(d2.y, d1.y)), ids);
  }
}

// ---------------------------------------------------------------------------
// face pass, in three launches
// ---------------------------------------------------------------------------
// The per-face scalar work (face state, heat flux, half-range moments, slopes,
// time weights: a chain of FP64 transcendentals) would otherwise run on one or
// two lanes of every face CTA while the rest of the CTA waits.  Here it runs
// one face per thread, between two sweeps that take one face per warp:
//   1. face_moments_warp: the reconstruction of every velocity pair, stored
//      as the face deviation in the face's flux row and the slopes in its aux
//      row, and the 13 raw moments of the deviation into the face record;
//   2. face_coef_delta (a thread per face): the face state and every per-face
//      coefficient of the flux into the face record;
//   3. face_flux_warp: the deviation flux of every velocity pair over the
//      stored face deviations, written over them, and the macro flux.
// Wall faces run their whole procedure in a launch of their own
// (wall_pass_delta, a CTA per face).  Interior faces take the dt after the
// first dt check, which is the dt of the reference's final flux pass (its
// first pass is overwritten when dt changes); wall faces run the reference's
// two passes, for the side effects of adsorbing walls.

// layout of a face record (ugks_fused_block.face_rec, UGKS_FACE_REC doubles
// per face): [0, 13) the raw moments of the face deviation (face frame);
// [16, 38) the coefficients of face_coefficients (c[0..21]); then
constexpr int FR_MOM = 0, FR_C = 16, FR_UX = 38, FR_UY = 39, FR_LAM = 40, FR_KB = 41, FR_SX = 42, FR_SY = 43,
              FR_LNP = 44, FR_UGX = 45, FR_UGY = 46;
static_assert(FR_UGY < UGKS_FACE_REC, "face record layout");

// shared memory of a wall CTA: Nv (h, b) FP64 face values plus Nv float2 of
// scratch
inline size_t delta_wall_smem(int max_nv) { return 24 * (size_t)max_nv + 16; }

// a wall face (a CTA per face): its whole procedure, in the main pass's wall
// launch and in the retry pass, where interior faces have nothing to redo
// (their moments do not depend on dt)
template <int FM, int NT, bool WALLS>
__device__ __forceinline__ void face_item_delta(const ugks_fused_block *__restrict__ B, int nb,
                                                ugks_solve_state *__restrict__ solves, const int w, int retry_pass) {
  extern __shared__ double dyn[];
  FaceWork fwk;
  if (!face_work<FM>(B, nb, solves, w, retry_pass, fwk)) return;
  static_assert(WALLS, "interior faces run in face_moments_warp");
  if (fwk.wall < 0) return;
  const ugks_fused_block &blk = B[fwk.bi];
  const ugks_block_desc &d = blk.d;
  ugks_solve_state &sol = solves[blk.solve];
  const double dt = sol.dt;
  const int dir = fwk.dir, mi = fwk.mi, mj = fwk.mj, wall = fwk.wall;
  const long gi = fwk.gi, gj = fwk.gj;
  const int Nv = d.Nv, NP = npairs(d), vn = d.v_num;
  const RefMaxwellian ref = ref_of(blk);
  const V2 n = ld2(blk.normal, faceidx(d, gi, gj, dir));
  const double len = blk.side_length[faceidx(d, gi, gj, dir)];
  double g6[6];
  {
    const double *fg = blk.face_geo + 6 * faceidx(d, gi, gj, dir);
#pragma unroll
    for (int k = 0; k < 6; ++k) g6[k] = fg[k];
  }
  const float dist0 = (float)g6[0], idist0 = (float)g6[1], il0 = (float)g6[2];
  const float dist1 = (float)g6[3], idist1 = (float)g6[4], il1 = (float)g6[5];
  constexpr int L = FM == 1 ? 5 : 3, MID = FM == 1 ? 2 : 1;
  float4 *frow = reinterpret_cast<float4 *>(dir == SOUTH ? blk.flux_S : blk.flux_W) + pidx(d, gi, gj, 0);

  {
    // the FP64 wall procedure on M + df
    __shared__ FaceShared<NT> sh;
    double *fw = dyn;                                          // Nv x (h, b)
    float2 *rin = reinterpret_cast<float2 *>(fw + 2 * (size_t)Nv);  // Nv
    const int step = dir == SOUTH ? 1 : d.Nj;                  // cells
    const float4 *fcell = reinterpret_cast<const float4 *>(blk.f) + pidx(d, gi, gj, 0);
    const double2 *qd = reinterpret_cast<const double2 *>(d.quad);
    for (int v = threadIdx.x; v < Nv; v += NT) {
      const double2 e = qd[v];
      const double u = e.x * n.x + e.y * n.y;
      const bool up = u > 0.0;
      const long st = (up ? step : -step) * (long)NP;
      const float4 *p0 = up ? fcell - (MID + 1) * (long)step * NP : fcell + MID * (long)step * NP;
      float2 xs[L];
#pragma unroll
      for (int s = 0; s < L; ++s) xs[s] = make_float2(pair_get(p0 + s * st, v, vn, 0), pair_get(p0 + s * st, v, vn, 1));
      float fh, fb, sx, sy;
      reconstruct_f<FM>(xs, up ? il1 : il0, up ? dist1 : dist0, up ? idist1 : idist0, fh, fb, sx, sy);
      const double m = ref.mh[v];
      fw[2 * v] = m + (double)fh;
      fw[2 * v + 1] = ref.kb0 * m + (double)fb;
    }
    const double dl = dt * len;
    wall_face<NT>(blk, sol, sh, fw, rin, wall, dir, gi, gj, mi, mj, n, len, dt, [&](int v, double hx, double hy) {
      const double2 e = qd[v];
      const double m = dl * (e.x * n.x + e.y * n.y) * ref.mh[v];
      pair_put(frow, v, vn, (float)(hx - m), (float)(hy - ref.kb0 * m));
    });
  }
}

// wall faces of the main pass: a CTA per wall work item (2 (ni + nj) per
// block: the S faces of rows 0 and nj, then the W faces of columns 0 and ni),
// running the wall procedure when that side of the block is a wall
template <int NT>
__global__ void __launch_bounds__(NT) wall_pass_delta(const ugks_fused_block *__restrict__ B, int nb,
                                                      ugks_solve_state *__restrict__ solves) {
  const int w = (int)blockIdx.x;
  const ugks_fused_block &blk = B[find_block<3>(B, nb, w)];
  const ugks_block_desc &d = blk.d;
  UGKS_CHECK_ITEM(3, blk, w, solves);
  int lw = w - blk.wall_begin, mi, mj, dir;
  if (lw < 2 * d.ni) {
    dir = SOUTH;
    mi = lw % d.ni;
    mj = lw < d.ni ? 0 : d.nj;
  } else {
    lw -= 2 * d.ni;
    dir = WEST;
    mj = lw % d.nj;
    mi = lw < d.nj ? 0 : d.ni;
  }
  const int fw = blk.face_begin + ((mi * (d.nj + 1) + mj) << 1) + dir;
  switch (d.flux_method) {
    case 0: face_item_delta<0, NT, true>(B, nb, solves, fw, 0); break;
    case 1: face_item_delta<1, NT, true>(B, nb, solves, fw, 0); break;
    case 3: face_item_delta<3, NT, true>(B, nb, solves, fw, 0); break;
    default: break;
  }
}
constexpr int WALL_NT = 128;

// raw moments up to third order (RM* / RB*) of a distribution, from the
// global frame (x, y) into a face frame u = nx x + ny y, t = nx y - ny x: the
// moment tensors rotate as the velocities do
__device__ __forceinline__ void rotate_moments(double (&m)[RNMOM], V2 n) {
  const double a = n.x, c = n.y, aa = a * a, cc = c * c, ac = a * c;
  const double m10 = m[RM10], m01 = m[RM01], m20 = m[RM20], m11 = m[RM11], m02 = m[RM02];
  const double m30 = m[RM30], m21 = m[RM21], m12 = m[RM12], m03 = m[RM03], b10 = m[RB10], b01 = m[RB01];
  m[RM10] = a * m10 + c * m01;
  m[RM01] = a * m01 - c * m10;
  m[RM20] = aa * m20 + 2.0 * ac * m11 + cc * m02;
  m[RM11] = ac * (m02 - m20) + (aa - cc) * m11;
  m[RM02] = cc * m20 - 2.0 * ac * m11 + aa * m02;
  // u^3, u^2 t, u t^2, t^3 expanded in x^3, x^2 y, x y^2, y^3
  m[RM30] = a * aa * m30 + 3.0 * aa * c * m21 + 3.0 * a * cc * m12 + c * cc * m03;
  m[RM21] = -aa * c * m30 + a * (aa - 2.0 * cc) * m21 + c * (2.0 * aa - cc) * m12 + a * cc * m03;
  m[RM12] = a * cc * m30 + c * (cc - 2.0 * aa) * m21 + a * (aa - 2.0 * cc) * m12 + aa * c * m03;
  m[RM03] = -c * cc * m30 + 3.0 * a * cc * m21 - 3.0 * aa * c * m12 + a * aa * m03;
  m[RB10] = a * b10 + c * b01;
  m[RB01] = a * b01 - c * b10;
}

// 2. coefficients: the per-face block of face_coefficients, one face per
// thread (the same chain as the lanes of a face CTA run there)
__global__ void __launch_bounds__(128) face_coef_delta(const ugks_fused_block *__restrict__ B, int nb,
                                                       ugks_solve_state *__restrict__ solves, int n_faces) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_faces) return;
  FaceWork fwk;
  if (!face_work<-1>(B, nb, solves, w, 0, fwk) || fwk.wall >= 0) return;
  const ugks_fused_block &blk = B[fwk.bi];
  const ugks_block_desc &d = blk.d;
  const double dt = solves[blk.solve].dt;
  const int dir = fwk.dir;
  const long gi = fwk.gi, gj = fwk.gj;
  const RefMaxwellian ref = ref_of(blk);
  const size_t fk = faceidx(d, gi, gj, dir);
  double *rec = blk.face_rec + (size_t)UGKS_FACE_REC * fk;
  const V2 n = ld2(blk.normal, fk), mid = ld2(blk.mid_side, fk);
  const double len = blk.side_length[fk];
  double dm[RNMOM];
#pragma unroll
  for (int k = 0; k < RNMOM; ++k) dm[k] = rec[FR_MOM + k];
  rotate_moments(dm, n);
  // face state: the reference's moments in the face frame plus the deviation's
  const double *R = ref.mom;
  const V2 rU = to_local(v2(R[RM10], R[RM01]), n);
  const P4 W = p4(R[RM00] + dm[RM00], rU.x + dm[RM10], rU.y + dm[RM01],
                  0.5 * ((R[RM20] + R[RM02] + R[RB00]) + (dm[RM20] + dm[RM02] + dm[RB00])));
  Rcp rc;
  const P4 prim = to_primary_rcp(d, W, rc);
  const V2 Ug = to_global(v2(prim.s1, prim.s2), n);
  // face heat flux (calcFaceQ, clUGKS.c:522-585): M's part from its global
  // moments rotated into the face frame, the deviation's from its raw moments
  V2 Q = to_local(heat_flux_from_moments(R, d.K, Ug), n);
  {
    const V2 qd_ = heat_flux_from_moments(dm, d.K, v2(prim.s1, prim.s2));
    Q.x += qd_.x;
    Q.y += qd_.y;
  }
  // the two cells beside the face (getAL / getAR inputs, getPLR slopes)
  double nbr[2][5];
  for (int side = 0; side < 2; ++side) {
    const size_t k = side == 0 ? gidx(d, gi - dir, gj - (1 - dir)) : gidx(d, gi, gj);
    const P4 mc = ld4(blk.cell_mom, k);
    const V2 uc = to_local(v2(mc.s1, mc.s2), n);
    const V2 cc = ld2(blk.centre, k);
    nbr[side][0] = mc.s0;
    nbr[side][1] = uc.x;
    nbr[side][2] = uc.y;
    nbr[side][3] = mc.s3;
    nbr[side][4] = nr_rcp(sqrt((mid.x - cc.x) * (mid.x - cc.x) + (mid.y - cc.y) * (mid.y - cc.y)));
  }
  // getPLR slopes (clUGKS.c:424-436) and initMacroFlux (446-518)
  const double kb = (0.5 * d.K) * rc.lam;
  double Mh[2][MNUM], Mv[MTUM], Mxi[3];
  P4 a[2], t1[2], t2[2];
  for (int side = 0; side < 2; ++side) {
    const double sg = side == 0 ? 1.0 : -1.0;
    half_moments_rcp(d.PI, d.K, prim, rc, sg, Mh[side], Mv, Mxi);
    const double id = sg * nbr[side][4];
    a[side] = micro_slope_rcp(d.K, prim, rc,
                              p4((W.s0 - nbr[side][0]) * id, (W.s1 - nbr[side][1]) * id,
                                 (W.s2 - nbr[side][2]) * id, (W.s3 - nbr[side][3]) * id));
    t1[side] = moment_au(a[side], Mh[side], Mv, Mxi, 1, 0);
    t2[side] = moment_au(a[side], Mh[side], Mv, Mxi, 2, 0);
  }
  double Mt[5];
  time_weights_rcp(inv_relax_time_rcp(d, prim, rc), dt, Mt);
  double *c = rec + FR_C;
  const double xk = Mxi[2] - kb * kb;
  for (int side = 0; side < 2; ++side) {
    double *ck = c + 5 * side;
    ck[0] = Mt[1] * fma(0.5 * a[side].s3, kb, a[side].s0);
    ck[1] = Mt[1] * a[side].s1;
    ck[2] = Mt[1] * a[side].s2;
    ck[3] = Mt[1] * (0.5 * a[side].s3);
    ck[4] = Mt[1] * (0.5 * a[side].s3 * xk);
  }
  double Mu[MNUM];
#pragma unroll
  for (int k = 0; k < MNUM; ++k) Mu[k] = Mh[0][k] + Mh[1][k];
  const P4 aT = micro_slope_rcp(d.K, prim, rc, scale(-prim.s0, add(t1[0], t1[1])));
  const P4 g0 = scale(prim.s0, add(add(scale(Mt[0], moment_uv(Mu, Mv, Mxi, 1, 0, 0)), scale(Mt[1], add(t2[0], t2[1]))),
                                   scale(Mt[2], moment_au(aT, Mu, Mv, Mxi, 1, 0))));
  c[10] = Mt[2] * fma(0.5 * aT.s3, kb, aT.s0) + Mt[0];
  c[11] = Mt[2] * aT.s1;
  c[12] = Mt[2] * aT.s2;
  c[13] = Mt[2] * (0.5 * aT.s3);
  c[14] = Mt[2] * (0.5 * aT.s3 * xk);
  c[15] = Mt[0];
  c[16] = Mt[3] * len;
  c[17] = Mt[4] * len;
  c[18] = len * g0.s0; c[19] = len * g0.s1; c[20] = len * g0.s2; c[21] = len * g0.s3;
  const double s0 = 0.8 * (1 - d.Pr) * (prim.s3 * prim.s3) * rc.rho;
  rec[FR_UX] = prim.s1;
  rec[FR_UY] = prim.s2;
  rec[FR_LAM] = prim.s3;
  rec[FR_KB] = kb;
  rec[FR_SX] = (Mt[0] * s0) * Q.x;
  rec[FR_SY] = (Mt[0] * s0) * Q.y;
  rec[FR_LNP] = log((prim.s0 * prim.s3) / (ref.P0 * d.PI));  // ln(P / P0), P = rho lambda / pi
  rec[FR_UGX] = Ug.x;
  rec[FR_UGY] = Ug.y;
}

// ---------------------------------------------------------------------------
// warp-per-face forms of kernels 1 and 3: an interior face per warp, whose
// lanes sweep the velocity pairs (p = lane, lane + 32, ...).  The per-face
// sums close with one halving butterfly and no CTA barrier, so that a warp's
// per-face set-up overlaps the other warps' sweeps.
// ---------------------------------------------------------------------------
// doubles of shared memory per warp: moments (the axis velocities as floats,
// in at most max_axes + 2 doubles), flux (the face record, then the axis
// tables)
inline int delta_moments_stride(int max_axes) { return ((max_axes + 2) + 1) & ~1; }
inline int delta_flux_stride(int max_axes) { return 48 + (((12 * (max_axes + 2) + 7) / 8 + 1) & ~1); }

template <int FM, int WPC, int MINB>
__global__ void __launch_bounds__(WPC * 32, MINB) face_moments_warp(const ugks_fused_block *__restrict__ B, int nb,
                                                                    ugks_solve_state *__restrict__ solves,
                                                                    int first, int count, int wstride) {
  extern __shared__ double dyn[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = (int)blockIdx.x * WPC + warp;
  if (item >= count) return;
  FaceWork fwk;
  if (!face_work<FM>(B, nb, solves, first + item, 0, fwk) || fwk.wall >= 0) return;
  const ugks_fused_block &blk = B[fwk.bi];
  const ugks_block_desc &d = blk.d;
  const int dir = fwk.dir;
  const long gi = fwk.gi, gj = fwk.gj;
  const int NP = npairs(d), un = d.u_num, vn = d.v_num;
  const size_t fk = faceidx(d, gi, gj, dir);
  const V2 n = ld2(blk.normal, fk);
  const double *fg = blk.face_geo + 6 * fk;
  const float dist0 = (float)fg[0], idist0 = (float)fg[1], il0 = (float)fg[2];
  const float dist1 = (float)fg[3], idist1 = (float)fg[4], il1 = (float)fg[5];
  constexpr int L = FM == 1 ? 5 : 3, MID = FM == 1 ? 2 : 1;
  // axis velocities as floats (entry u_num: the padding lane's, 0)
  float *QXf = reinterpret_cast<float *>(dyn + (size_t)warp * wstride), *QYf = QXf + (un + 1);
  for (int k = lane; k <= un + vn; k += 32) {
    if (k < un) QXf[k] = (float)d.quad[2 * (size_t)k * vn];
    else if (k == un) QXf[k] = 0.0f;
    else QYf[k - un - 1] = (float)d.quad[2 * (size_t)(k - un - 1) + 1];
  }
  __syncwarp();
  const int pstep = (dir == SOUTH ? 1 : d.Nj) * NP;  // pairs between neighbouring cells along the normal
  const float4 *fcell = reinterpret_cast<const float4 *>(blk.f) + pidx(d, gi, gj, 0);
  const float4 *up1 = fcell - (MID + 1) * pstep, *up0 = fcell + MID * pstep;
  float4 *frow = reinterpret_cast<float4 *>(dir == SOUTH ? blk.flux_S : blk.flux_W) + pidx(d, gi, gj, 0);
  float4 *arow = reinterpret_cast<float4 *>(dir == SOUTH ? blk.aux_S : blk.aux_W) + pidx(d, gi, gj, 0);
  const float2 nx2 = bc2((float)n.x), ny2 = bc2((float)n.y), mny2 = bc2(-(float)n.y);
  // raw moments of the face deviation in the global frame (the coefficient
  // pass rotates the sums into the face frame): products and each lane's sums
  // in packed FP32, the two velocities of a pair in the two halves, about 17
  // terms per half at Nv 1089; the halves and the lanes are combined in FP64
  float2 acc[RNMOM];
#pragma unroll
  for (int k = 0; k < RNMOM; ++k) acc[k] = make_float2(0.0f, 0.0f);
  // pair p = a v_num + jv: velocities (2a, jv) and (2a + 1, jv)
  const int qs = 32 / vn, rs = 32 % vn;
  int ia = lane / vn, jv = lane % vn;
  // reconstruction, stored face values and slopes, and moments of pair p
  // from its stencil rows
  auto pair_work = [&](int p, const float2 (&Sh)[L], const float2 (&Sb)[L], float2 qx, float2 qy, bool ua, bool ub) {
    const float2 il = make_float2(ua ? il1 : il0, ub ? il1 : il0);
    const float2 ds = make_float2(ua ? dist1 : dist0, ub ? dist1 : dist0);
    const float2 ids = make_float2(ua ? idist1 : idist0, ub ? idist1 : idist0);
    const float2 sh2 = slope_pair<FM>(Sh, il, ids), sb2 = slope_pair<FM>(Sb, il, ids);
    const float2 fh = fma2(sh2, ds, Sh[MID]), fb = fma2(sb2, ds, Sb[MID]);
    frow[p] = cat2(fh, fb);
    arow[p] = cat2(sh2, sb2);
    // raw moments (global frame); the padding velocity has df = 0
    const float2 xh = mul2(qx, fh), yh = mul2(qy, fh), xx = mul2(qx, qx), yy = mul2(qy, qy);
    acc[RM00] = add2(acc[RM00], fh);
    acc[RM10] = add2(acc[RM10], xh);
    acc[RM01] = add2(acc[RM01], yh);
    acc[RM20] = fma2(qx, xh, acc[RM20]);
    acc[RM11] = fma2(qy, xh, acc[RM11]);
    acc[RM02] = fma2(qy, yh, acc[RM02]);
    acc[RM30] = fma2(xx, xh, acc[RM30]);
    acc[RM21] = fma2(xx, yh, acc[RM21]);
    acc[RM12] = fma2(yy, xh, acc[RM12]);
    acc[RM03] = fma2(yy, yh, acc[RM03]);
    acc[RB00] = add2(acc[RB00], fb);
    acc[RB10] = fma2(qx, fb, acc[RB10]);
    acc[RB01] = fma2(qy, fb, acc[RB01]);
  };
#pragma unroll 1
  for (int p = lane; p < NP; p += 32) {
    const float2 qx = *reinterpret_cast<const float2 *>(QXf + 2 * ia), qy = bc2(QYf[jv]);
    const float2 U = fma2(qx, nx2, mul2(qy, ny2));
    const bool ua = U.x > 0.0f, ub = U.y > 0.0f;
    float2 Sh[L], Sb[L];
    if (ua == ub) {
      const float4 *s0 = (ua ? up1 : up0) + p;
      const int st = ua ? pstep : -pstep;
#pragma unroll
      for (int s = 0; s < L; ++s) {
        const float4 x = s0[s * st];
        Sh[s] = lo2(x);
        Sb[s] = hi2(x);
      }
    } else {
      // the two velocities of the pair are upwinded from opposite sides
      const float4 *sa = (ua ? up1 : up0) + p, *sb = (ub ? up1 : up0) + p;
      const int ta = ua ? pstep : -pstep, tb = ub ? pstep : -pstep;
#pragma unroll
      for (int s = 0; s < L; ++s) {
        const float4 x = sa[s * ta], y = sb[s * tb];
        Sh[s] = make_float2(x.x, y.y);
        Sb[s] = make_float2(x.z, y.w);
      }
    }
    pair_work(p, Sh, Sb, qx, qy, ua, ub);
    jv += rs;
    ia += qs;
    if (jv >= vn) { jv -= vn; ++ia; }
  }
  double mom[RNMOM];
#pragma unroll
  for (int k = 0; k < RNMOM; ++k) mom[k] = (double)acc[k].x + (double)acc[k].y;
  const double tw = warp_spread_sum<RNMOM>(mom);
  constexpr int S = spread_shift<RNMOM>();
  if ((lane & ((1 << S) - 1)) == 0 && (lane >> S) < RNMOM)
    blk.face_rec[(size_t)UGKS_FACE_REC * fk + FR_MOM + (lane >> S)] = tw;
}

// 3. flux (a warp per face): the FP64 sweep's terms (see face_item_fp64) with
// f = M + df:
//   dflux_h = u Mt0 len M r + Zh + u h0 (B - Mt0),
//   dflux_b = u Mt0 len M ((kb - kb0) + kb r) + Zb + u h0 (kb (B - Mt0) + Mt1 u a3 X/2 + Mt2 aT3 X/2),
//   Zh = u (S P4 h0 + Mt3 len dfh - Mt4 len u sh), Zb likewise,
//   h0 = len M (1 + r), r = g / M - 1,
// and the discrete macro flux is Mt3 len sum(u M (1, u, v, |u|^2; kb0)) (the
// reference's moments) plus the sums of the deviation Z terms
template <int WPC, int MINB>
__global__ void __launch_bounds__(WPC * 32, MINB) face_flux_warp(const ugks_fused_block *__restrict__ B, int nb,
                                                                 ugks_solve_state *__restrict__ solves,
                                                                 int n_faces, int wstride) {
  extern __shared__ double dyn[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = (int)blockIdx.x * WPC + warp;
  if (item >= n_faces) return;
  FaceWork fwk;
  if (!face_work<-1>(B, nb, solves, item, 0, fwk) || fwk.wall >= 0) return;
  const ugks_fused_block &blk = B[fwk.bi];
  const ugks_block_desc &d = blk.d;
  const int dir = fwk.dir;
  const long gi = fwk.gi, gj = fwk.gj;
  const int NP = npairs(d), un = d.u_num, vn = d.v_num;
  const RefMaxwellian ref = ref_of(blk);
  const size_t fk = faceidx(d, gi, gj, dir);
  const double *rec = blk.face_rec + (size_t)UGKS_FACE_REC * fk;
  const V2 n = ld2(blk.normal, fk);
  const double len = blk.side_length[fk];
  double *fc = dyn + (size_t)warp * wstride;
  float2 *EAU = reinterpret_cast<float2 *>(fc + 48), *EAV = EAU + (un + 1);  // (expm1 table, axis factor)
  float *QX = reinterpret_cast<float *>(EAV + vn), *QY = QX + (un + 1);
  const float4 *EAU2 = reinterpret_cast<const float4 *>(EAU);  // the two u-nodes of a pair row
  const float2 *QX2 = reinterpret_cast<const float2 *>(QX);
  fc[lane] = rec[lane];
  if (lane < 16) fc[32 + lane] = rec[32 + lane];
  __syncwarp();
  {
    // expm1 axis tables of the face Maxwellian against M, its axis factors
    // (the face length on the u axis) and the axis velocities; entry un is
    // the padding lane's: 0
    const double lam = fc[FR_LAM], Ugx = fc[FR_UGX], Ugy = fc[FR_UGY], lnP = fc[FR_LNP];
    for (int k = lane; k <= un + vn; k += 32) {
      if (k < un) {
        const double x = d.quad[2 * (size_t)k * vn];
        EAU[k] = make_float2((float)axis_expm1(x, Ugx, lam, ref.lam0, lnP), (float)(ref.Au[k] * len));
        QX[k] = (float)x;
      } else if (k == un) {
        EAU[k] = make_float2(0.0f, 0.0f);
        QX[k] = 0.0f;
      } else {
        const int j = k - un - 1;
        const double y = d.quad[2 * (size_t)j + 1];
        EAV[j] = make_float2((float)axis_expm1(y, Ugy, lam, ref.lam0), (float)ref.Av[j]);
        QY[j] = (float)y;
      }
    }
  }
  __syncwarp();
  const double *c = fc + FR_C;
  const double Mt0 = c[15];
  const float2 nx2 = bc2((float)n.x), ny2 = bc2((float)n.y), mny2 = bc2(-(float)n.y);
  const float2 fUx = bc2((float)fc[FR_UX]), fUy = bc2((float)fc[FR_UY]), flam2 = bc2((float)(2.0 * fc[FR_LAM]));
  const float2 fsx = bc2((float)fc[FR_SX]), fsy = bc2((float)fc[FR_SY]);
  const float2 fkb = bc2((float)fc[FR_KB]), fdkb = bc2((float)(fc[FR_KB] - ref.kb0));
  const float2 fMt0 = bc2((float)Mt0), fMt3L = bc2((float)c[16]), fnMt4L = bc2((float)(-c[17]));
  const float2 fT0 = bc2((float)(c[10] - Mt0)), fT1 = bc2((float)c[11]), fT2 = bc2((float)c[12]);
  const float2 fT3 = bc2((float)c[13]), fCT = bc2((float)c[14]);
  // upwind slope coefficients: aR for u <= 0, aR + dA for u > 0
  const float2 AR0 = bc2((float)c[5]), AR1 = bc2((float)c[6]), AR2 = bc2((float)c[7]), AR3 = bc2((float)c[8]);
  const float2 AR4 = bc2((float)c[9]);
  const float2 dA0 = bc2((float)(c[0] - c[5])), dA1 = bc2((float)(c[1] - c[6])), dA2 = bc2((float)(c[2] - c[7]));
  const float2 dA3 = bc2((float)(c[3] - c[8])), dA4 = bc2((float)(c[4] - c[9]));
  float2 acc[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) acc[k] = make_float2(0.0f, 0.0f);
  float4 *frow = reinterpret_cast<float4 *>(dir == SOUTH ? blk.flux_S : blk.flux_W) + pidx(d, gi, gj, 0);
  const float4 *arow = reinterpret_cast<const float4 *>(dir == SOUTH ? blk.aux_S : blk.aux_W) + pidx(d, gi, gj, 0);
  const int qs = 32 / vn, rs = 32 % vn;
  int ia = lane / vn, jv = lane % vn;
#pragma unroll 1
  for (int p = lane; p < NP; p += 32) {
    const float4 fd = frow[p], sg = arow[p];
    const float4 eu = EAU2[ia];  // (a, len Au) of u-nodes 2ia and 2ia + 1
    const float2 ev = EAV[jv];   // (b, Av), shared by the pair
    const float2 qx = QX2[ia], qy = bc2(QY[jv]);
    const float2 U = fma2(qx, nx2, mul2(qy, ny2)), T = fma2(qy, nx2, mul2(qx, mny2));
    const float2 r = rel_excess(make_float2(eu.x, eu.z), bc2(ev.x));
    const float2 ml = mul2(make_float2(eu.y, eu.w), bc2(ev.y));  // len M
    const float2 h0 = fma2(ml, r, ml);
    const float2 uu = fma2(U, U, mul2(T, T));
    const float2 cx = sub2(U, fUx), cy = sub2(T, fUy), c2 = fma2(cx, cx, mul2(cy, cy));
    const float2 Sp = fma2(cx, fsx, mul2(cy, fsy));
    const float2 S4 = mul2(Sp, fma2(flam2, c2, bc2(-4.0f))), S2 = fma2(bc2(2.0f), Sp, S4);
    const float2 pos = make_float2(U.x > 0.0f ? 1.0f : 0.0f, U.y > 0.0f ? 1.0f : 0.0f);
    const float2 MPR = fma2(AR3, uu, fma2(AR2, T, fma2(AR1, U, AR0)));
    const float2 dMP = fma2(dA3, uu, fma2(dA2, T, fma2(dA1, U, dA0)));
    const float2 MP = fma2(pos, dMP, MPR), A4 = fma2(pos, dA4, AR4);
    const float2 Bk = fma2(U, MP, fma2(fT3, uu, fma2(fT2, T, fma2(fT1, U, fT0))));  // B - Mt0
    const float2 mu = mul2(fnMt4L, U);
    const float2 Rh = fma2(mu, lo2(sg), mul2(fMt3L, lo2(fd))), Rb = fma2(mu, hi2(sg), mul2(fMt3L, hi2(fd)));
    const float2 Zh = mul2(U, fma2(S4, h0, Rh)), Zb = mul2(U, fma2(mul2(S2, fkb), h0, Rb));
    const float2 uh = mul2(U, h0), um0 = mul2(mul2(U, ml), fMt0);
    const float2 hx = fma2(uh, Bk, fma2(um0, r, Zh));
    const float2 hy = fma2(uh, fma2(fkb, Bk, fma2(A4, U, fCT)), fma2(um0, fma2(fkb, r, fdkb), Zb));
    acc[0] = add2(acc[0], Zh);
    acc[1] = fma2(U, Zh, acc[1]);
    acc[2] = fma2(T, Zh, acc[2]);
    acc[3] = fma2(uu, Zh, acc[3]);
    acc[4] = add2(acc[4], Zb);
    frow[p] = cat2(hx, hy);
    jv += rs;
    ia += qs;
    if (jv >= vn) { jv -= vn; ++ia; }
  }
  // the per-lane FP32 sums, added in FP64 across the warp
  double af[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) af[k] = (double)acc[k].x + (double)acc[k].y;
  const double tw = warp_spread_sum<5>(af);
  constexpr int S = spread_shift<5>();
  double da[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) da[k] = __shfl_sync(0xffffffffu, tw, k << S);
  if (lane == 0) {
    // M's part of the discrete macro flux: sums of u_n M (1, u_n, u_t, |u|^2)
    // and u_n M_b from the global moments
    const double *R = ref.mom;
    const double nx = n.x, ny = n.y, Mt3L = c[16];
    const double K0 = nx * R[RM10] + ny * R[RM01];
    const double K1 = nx * nx * R[RM20] + 2.0 * nx * ny * R[RM11] + ny * ny * R[RM02];
    const double K2 = -nx * ny * R[RM20] + (nx * nx - ny * ny) * R[RM11] + nx * ny * R[RM02];
    const double K3 = nx * (R[RM30] + R[RM12]) + ny * (R[RM21] + R[RM03]);
    const double Kb = nx * R[RB10] + ny * R[RB01];
    P4 out = p4(da[0] + Mt3L * K0 + c[18], da[1] + Mt3L * K1 + c[19], da[2] + Mt3L * K2 + c[20],
                0.5 * ((da[3] + Mt3L * K3) + (da[4] + Mt3L * Kb)) + c[21]);
    const V2 g = to_global(v2(out.s1, out.s2), n);
    out.s1 = g.x;
    out.s2 = g.y;
    st4(dir == SOUTH ? blk.flux_macro_S : blk.flux_macro_W, gidx(d, gi, gj), out);
  }
}

// ---------------------------------------------------------------------------
// the flux sweep with its rows staged by the bulk-copy engine: a face per
// warp, its stored face values and slopes copied into shared memory in chunks
// of FLUX_CHUNK pairs, two chunks in flight (the copy of chunk c + 1 runs
// while the lanes work on chunk c; the first overlaps the axis tables)
// ---------------------------------------------------------------------------
#ifndef UGKS_FLUX_CHUNK
#define UGKS_FLUX_CHUNK 128
#endif
constexpr int FLUX_CHUNK = UGKS_FLUX_CHUNK;
static_assert(FLUX_CHUNK % 32 == 0, "whole trips of a warp per chunk");
constexpr uint32_t kCopyWaitPolls = UGKS_MBAR_TRY_WAIT ? 1u << 20 : 1u << 24;  // about 1 s
constexpr int STATUS_COPY_TIMEOUT = 8;
// bytes of shared memory per warp: two barriers, two chunk buffers (values and
// slopes), the face record and the axis tables
inline size_t flux_tma_warp_bytes(int max_axes) {
  return 16 + 2 * 2 * (size_t)FLUX_CHUNK * 16 + 48 * 8 + (((size_t)12 * (max_axes + 2) + 15) & ~(size_t)15);
}

template <int WPC, int MINB>
__global__ void __launch_bounds__(WPC * 32, MINB) face_flux_tma(const ugks_fused_block *__restrict__ B, int nb,
                                                                ugks_solve_state *__restrict__ solves,
                                                                int n_faces, int wbytes) {
  extern __shared__ __align__(128) unsigned char dyn_b[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = (int)blockIdx.x * WPC + warp;
  if (item >= n_faces) return;
  FaceWork fwk;
  if (!face_work<-1>(B, nb, solves, item, 0, fwk) || fwk.wall >= 0) return;
  const ugks_fused_block &blk = B[fwk.bi];
  const ugks_block_desc &d = blk.d;
  const int dir = fwk.dir;
  const long gi = fwk.gi, gj = fwk.gj;
  const int NP = npairs(d), un = d.u_num, vn = d.v_num;
  const RefMaxwellian ref = ref_of(blk);
  const size_t fk = faceidx(d, gi, gj, dir);
  const double *rec = blk.face_rec + (size_t)UGKS_FACE_REC * fk;
  const V2 n = ld2(blk.normal, fk);
  const double len = blk.side_length[fk];
  // this warp's shared memory
  unsigned char *wm = dyn_b + (size_t)warp * wbytes;
  uint64_t *bar = reinterpret_cast<uint64_t *>(wm);
  float4 *buf = reinterpret_cast<float4 *>(wm + 16);  // [2][values | slopes][FLUX_CHUNK]
  double *fc = reinterpret_cast<double *>(buf + 4 * FLUX_CHUNK);
  float2 *EAU = reinterpret_cast<float2 *>(fc + 48), *EAV = EAU + (un + 1);  // (expm1 table, axis factor)
  float *QX = reinterpret_cast<float *>(EAV + vn), *QY = QX + (un + 1);
  const float4 *EAU2 = reinterpret_cast<const float4 *>(EAU);
  const float2 *QX2 = reinterpret_cast<const float2 *>(QX);
  float4 *frow = reinterpret_cast<float4 *>(dir == SOUTH ? blk.flux_S : blk.flux_W) + pidx(d, gi, gj, 0);
  const float4 *arow = reinterpret_cast<const float4 *>(dir == SOUTH ? blk.aux_S : blk.aux_W) + pidx(d, gi, gj, 0);
  const int nchunks = (NP + FLUX_CHUNK - 1) / FLUX_CHUNK;
  auto issue = [&](int c) {  // lane 0: the copies of chunk c into buffer c & 1
    const int p0 = c * FLUX_CHUNK, m = min(FLUX_CHUNK, NP - p0);
    const uint32_t bytes = (uint32_t)m * 16u;
    float4 *dst = buf + (c & 1) * 2 * FLUX_CHUNK;
    mbar_arrive_expect_tx(&bar[c & 1], 2u * bytes);
    bulk_g2s(dst, frow + p0, bytes, &bar[c & 1]);
    bulk_g2s(dst + FLUX_CHUNK, arow + p0, bytes, &bar[c & 1]);
  };
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
    issue(0);
  }
  fc[lane] = rec[lane];
  if (lane < 16) fc[32 + lane] = rec[32 + lane];
  __syncwarp();
  {
    // expm1 axis tables of the face Maxwellian against M, its axis factors
    // (the face length on the u axis) and the axis velocities; entry un is
    // the padding lane's: 0
    const double lam = fc[FR_LAM], Ugx = fc[FR_UGX], Ugy = fc[FR_UGY], lnP = fc[FR_LNP];
    for (int k = lane; k <= un + vn; k += 32) {
      if (k < un) {
        const double x = d.quad[2 * (size_t)k * vn];
        EAU[k] = make_float2((float)axis_expm1(x, Ugx, lam, ref.lam0, lnP), (float)(ref.Au[k] * len));
        QX[k] = (float)x;
      } else if (k == un) {
        EAU[k] = make_float2(0.0f, 0.0f);
        QX[k] = 0.0f;
      } else {
        const int j = k - un - 1;
        const double y = d.quad[2 * (size_t)j + 1];
        EAV[j] = make_float2((float)axis_expm1(y, Ugy, lam, ref.lam0), (float)ref.Av[j]);
        QY[j] = (float)y;
      }
    }
  }
  __syncwarp();
  const double *c = fc + FR_C;
  const double Mt0 = c[15];
  const float2 nx2 = bc2((float)n.x), ny2 = bc2((float)n.y), mny2 = bc2(-(float)n.y);
  const float2 fUx = bc2((float)fc[FR_UX]), fUy = bc2((float)fc[FR_UY]), flam2 = bc2((float)(2.0 * fc[FR_LAM]));
  const float2 fsx = bc2((float)fc[FR_SX]), fsy = bc2((float)fc[FR_SY]);
  const float2 fkb = bc2((float)fc[FR_KB]), fdkb = bc2((float)(fc[FR_KB] - ref.kb0));
  const float2 fMt0 = bc2((float)Mt0), fMt3L = bc2((float)c[16]), fnMt4L = bc2((float)(-c[17]));
  const float2 fT0 = bc2((float)(c[10] - Mt0)), fT1 = bc2((float)c[11]), fT2 = bc2((float)c[12]);
  const float2 fT3 = bc2((float)c[13]), fCT = bc2((float)c[14]);
  const float2 AR0 = bc2((float)c[5]), AR1 = bc2((float)c[6]), AR2 = bc2((float)c[7]), AR3 = bc2((float)c[8]);
  const float2 AR4 = bc2((float)c[9]);
  const float2 dA0 = bc2((float)(c[0] - c[5])), dA1 = bc2((float)(c[1] - c[6])), dA2 = bc2((float)(c[2] - c[7]));
  const float2 dA3 = bc2((float)(c[3] - c[8])), dA4 = bc2((float)(c[4] - c[9]));
  float2 acc[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) acc[k] = make_float2(0.0f, 0.0f);
  bool ok = true;
  for (int ch = 0; ch < nchunks; ++ch) {
    if (lane == 0 && ch + 1 < nchunks) {
      fence_proxy_async_smem();  // the lanes' reads of that buffer (chunk ch - 1) came first
      issue(ch + 1);
    }
    // every lane observes the completion itself (its acquire of the copied
    // rows); a lane that ran out of polls stops the whole warp
    ok = __all_sync(0xffffffffu, mbar_wait(&bar[ch & 1], (uint32_t)((ch >> 1) & 1), kCopyWaitPolls));
    if (!ok) break;
    const float4 *bv = buf + (ch & 1) * 2 * FLUX_CHUNK, *bs = bv + FLUX_CHUNK;
    const int p0 = ch * FLUX_CHUNK, m = min(FLUX_CHUNK, NP - p0);
    int ia = (p0 + lane) / vn, jv = (p0 + lane) % vn;
    const int qs = 32 / vn, rs = 32 % vn;
#pragma unroll 1
    for (int q = lane; q < m; q += 32) {
      const float4 fd = bv[q], sg = bs[q];
      const float4 eu = EAU2[ia];
      const float2 ev = EAV[jv];
      const float2 qx = QX2[ia], qy = bc2(QY[jv]);
      const float2 U = fma2(qx, nx2, mul2(qy, ny2)), T = fma2(qy, nx2, mul2(qx, mny2));
      const float2 r = rel_excess(make_float2(eu.x, eu.z), bc2(ev.x));
      const float2 ml = mul2(make_float2(eu.y, eu.w), bc2(ev.y));  // len M
      const float2 h0 = fma2(ml, r, ml);
      const float2 uu = fma2(U, U, mul2(T, T));
      const float2 cx = sub2(U, fUx), cy = sub2(T, fUy), c2 = fma2(cx, cx, mul2(cy, cy));
      const float2 Sp = fma2(cx, fsx, mul2(cy, fsy));
      const float2 S4 = mul2(Sp, fma2(flam2, c2, bc2(-4.0f))), S2 = fma2(bc2(2.0f), Sp, S4);
      const float2 pos = make_float2(U.x > 0.0f ? 1.0f : 0.0f, U.y > 0.0f ? 1.0f : 0.0f);
      const float2 MPR = fma2(AR3, uu, fma2(AR2, T, fma2(AR1, U, AR0)));
      const float2 dMP = fma2(dA3, uu, fma2(dA2, T, fma2(dA1, U, dA0)));
      const float2 MP = fma2(pos, dMP, MPR), A4 = fma2(pos, dA4, AR4);
      const float2 Bk = fma2(U, MP, fma2(fT3, uu, fma2(fT2, T, fma2(fT1, U, fT0))));  // B - Mt0
      const float2 mu = mul2(fnMt4L, U);
      const float2 Rh = fma2(mu, lo2(sg), mul2(fMt3L, lo2(fd))), Rb = fma2(mu, hi2(sg), mul2(fMt3L, hi2(fd)));
      const float2 Zh = mul2(U, fma2(S4, h0, Rh)), Zb = mul2(U, fma2(mul2(S2, fkb), h0, Rb));
      const float2 uh = mul2(U, h0), um0 = mul2(mul2(U, ml), fMt0);
      const float2 hx = fma2(uh, Bk, fma2(um0, r, Zh));
      const float2 hy = fma2(uh, fma2(fkb, Bk, fma2(A4, U, fCT)), fma2(um0, fma2(fkb, r, fdkb), Zb));
      acc[0] = add2(acc[0], Zh);
      acc[1] = fma2(U, Zh, acc[1]);
      acc[2] = fma2(T, Zh, acc[2]);
      acc[3] = fma2(uu, Zh, acc[3]);
      acc[4] = add2(acc[4], Zb);
      frow[p0 + q] = cat2(hx, hy);
      jv += rs;
      ia += qs;
      if (jv >= vn) { jv -= vn; ++ia; }
    }
    __syncwarp();
  }
  if (!ok) {
    // a copy outlived its bound: flag the solve, give the copies in flight
    // one more bound, and leave the face
    if (lane == 0) {
      atomicExch(&solves[blk.solve].status, STATUS_COPY_TIMEOUT);
      mbar_wait(&bar[0], 0u, kCopyWaitPolls);
      mbar_wait(&bar[1], 0u, kCopyWaitPolls);
    }
    __syncwarp();
    return;
  }
  double af[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) af[k] = (double)acc[k].x + (double)acc[k].y;
  const double tw = warp_spread_sum<5>(af);
  constexpr int S = spread_shift<5>();
  double da[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) da[k] = __shfl_sync(0xffffffffu, tw, k << S);
  if (lane == 0) {
    const double *R = ref.mom;
    const double nx = n.x, ny = n.y, Mt3L = c[16];
    const double K0 = nx * R[RM10] + ny * R[RM01];
    const double K1 = nx * nx * R[RM20] + 2.0 * nx * ny * R[RM11] + ny * ny * R[RM02];
    const double K2 = -nx * ny * R[RM20] + (nx * nx - ny * ny) * R[RM11] + nx * ny * R[RM02];
    const double K3 = nx * (R[RM30] + R[RM12]) + ny * (R[RM21] + R[RM03]);
    const double Kb = nx * R[RB10] + ny * R[RB01];
    P4 out = p4(da[0] + Mt3L * K0 + c[18], da[1] + Mt3L * K1 + c[19], da[2] + Mt3L * K2 + c[20],
                0.5 * ((da[3] + Mt3L * K3) + (da[4] + Mt3L * Kb)) + c[21]);
    const V2 g = to_global(v2(out.s1, out.s2), n);
    out.s1 = g.x;
    out.s2 = g.y;
    st4(dir == SOUTH ? blk.flux_macro_S : blk.flux_macro_W, gidx(d, gi, gj), out);
  }
}

// The cell pass stores the new deviation with stochastic rounding: round to
// nearest is biased where a slowly relaxing solve changes df by less than
// half an FP32 ulp per step (the stored value stays put while the FP64 one
// drifts), and that bias carried the heat flux of high-Kn cavities to
// 1.1e-5 relative after 2000 steps; unbiased rounding gives 3.9e-6.  The
// random bits hash (step, block within its solve, velocity pair), so a solve
// gets the same bits alone and in any batch.
#ifndef UGKS_SR_STORE
#define UGKS_SR_STORE 1
#endif
// integer hash (a 32-bit xorshift-multiply mixer) for stochastic rounding
__device__ __forceinline__ uint32_t sr_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
// x = f a1 + inc for two velocities as float pairs hi + lo, hi = RN(x),
// |lo| <= ulp(hi) / 2, in FP32 arithmetic only: a1 = a1h + a1l (two floats,
// given as -a1h and -a1l), the product's rounding error by FMA (Dekker's
// product) and the sums' by Knuth's two-sum.  hi + lo is x to within about
// 2^-24 of lo (2^-48 of f where f a1 and inc cancel), far below what the
// rounding probability needs.
__device__ __forceinline__ void sr_parts(float2 f, float2 inc, float2 a1h, float2 na1h, float2 na1l, float2 &hi,
                                         float2 &lo) {
  const float2 p = mul2(f, a1h);      // RN(f a1h)
  const float2 q = fma2(f, na1h, p);  // p - f a1h, exact
  const float2 cn = fma2(f, na1l, q); // -(f a1h - p + f a1l): x = p + inc - cn
  const float2 s = add2(p, inc);
  const float2 bp = sub2(s, p);
  const float2 e = add2(sub2(p, sub2(s, bp)), sub2(inc, bp));  // s + e = p + inc exactly
  const float2 r = sub2(e, cn);                                 // x - s
  hi = add2(s, r);
  const float2 bq = sub2(hi, s);
  lo = add2(sub2(s, sub2(hi, bq)), sub2(r, bq));                // hi + lo = s + r exactly
}
// hi + lo rounded to hi or to hi's neighbour on lo's side, the neighbour
// with probability |lo| / (the gap between them), u16 / 65536 uniform.  A
// zero, infinite or NaN hi comes back unchanged (the comparison is false).
__device__ __forceinline__ float sr_pick(float hi, float lo, uint32_t u16) {
  const uint32_t hb = __float_as_uint(hi);
  const float nb = __uint_as_float(((hb ^ __float_as_uint(lo)) >> 31) ? hb - 1u : hb + 1u);
  const float u = __uint_as_float(0x3f800000u | (u16 << 7)) - 1.0f;  // u16 / 65536, exact
  return fabsf(lo) > u * fabsf(nb - hi) ? nb : hi;
}

// ---------------------------------------------------------------------------
// cell pass: updateMacro + UGKS_update + clFindDT + calcQ of the next step on
// the deviations, one warp per cell (as cell_pass)
// ---------------------------------------------------------------------------
// per-warp shared memory (doubles): per velocity-axis node a float4 (the old
// and new states' expm1 tables, the axis factor, the axis velocity) for the
// u_num + 1 and v_num nodes, then CELL_COEF coefficient slots
inline int delta_cell_stride(int max_axes) { return 2 * (max_axes + 1) + CELL_COEF; }

template <int MINB>
__global__ void __launch_bounds__(CW * 32, MINB) cell_pass_delta(const ugks_fused_block *__restrict__ B, int nb,
                                                                   ugks_solve_state *__restrict__ solves,
                                                                   int n_cells, int wstride) {
  extern __shared__ double dyn[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int w = blockIdx.x * CW + warp;
  if (w >= n_cells) return;
  const int bi = find_block<1>(B, nb, w);
  const ugks_fused_block &blk = B[bi];
  const ugks_block_desc &d = blk.d;
  UGKS_CHECK_ITEM(1, blk, w, solves);
  ugks_solve_state &sol = solves[blk.solve];
  if (!sol.active) return;
  const RefMaxwellian ref = ref_of(blk);
  const int lc = w - blk.cell_begin;
  const long mi = lc / d.nj, mj = lc % d.nj;
  const long gi = mi + d.ghost, gj = mj + d.ghost;
  const int NP = npairs(d), un = d.u_num, vn = d.v_num;
  float4 *TU = reinterpret_cast<float4 *>(dyn + (size_t)warp * wstride), *TV = TU + (un + 1);
  double *bc = dyn + (size_t)warp * wstride + (wstride - CELL_COEF);
  const double dt = sol.dt;
  const P4 old = ld4(blk.macro, midx(d, mi, mj));
  // calcQ of f^n with the macro of f^n (accumulated by the previous cell pass)
  const V2 Q = ld2(blk.Q_next, midx(d, mi, mj));
  const double *R = ref.mom;
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
    // UGKS_update (clUGKS.c:1189-1257):
    //   df' = a1 df + a2 sum(dflux) + a4 (fEQ(old) - M) + a3 (fEQ(new) - M),
    //   a1 = (1 - dt/2 /tau_old) / D, a2 = 1 / (A D), a3 = dt/2 / (tau D),
    //   a4 = dt/2 / (tau_old D), D = 1 + dt/2 / tau (a1 + a3 + a4 = 1)
    const double itau_old = inv_relax_time_rcp(d, old, ro), itau = inv_relax_time_rcp(d, prim, rn);
    const double hdt = 0.5 * dt, iden = nr_rcp(1.0 + hdt * itau);
    const double P0pi = ref.P0 * d.PI;
    bc[0] = prim.s1;
    bc[1] = prim.s2;
    bc[2] = prim.s3;
    bc[3] = (1.0 - hdt * itau_old) * iden;                            // a1
    bc[4] = iden * iA;                                                // a2
    bc[5] = hdt * itau * iden;                                        // a3
    bc[6] = hdt * itau_old * iden;                                    // a4
    bc[7] = log((prim.s0 * prim.s3) / P0pi);                          // ln(P / P0) new
    bc[8] = log((old.s0 * old.s3) / P0pi);                            // ln(P / P0) old
    bc[9] = (0.5 * d.K) * rn.lam;                                     // K / (2 lambda) new
    bc[10] = 0.8 * (1 - d.Pr) * (prim.s3 * prim.s3) * rn.rho;         // Shakhov factor new
    const double fq = cfl_freq(blk, prim, mi, mj);
    atomicMax(&sol.max_freq, (unsigned long long)__double_as_longlong(fq));
  } else {
    // the old state's tables, axis factors and velocities
    const double lnPo = log((old.s0 * old.s3) / (ref.P0 * d.PI));
    for (int k = lane - 1; k <= un + vn; k += 31) {
      if (k < un) {
        const double x = d.quad[2 * (size_t)k * vn];
        TU[k] = make_float4((float)axis_expm1(x, old.s1, old.s3, ref.lam0, lnPo), 0.0f, (float)ref.Au[k], (float)x);
      } else if (k == un) {
        TU[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      } else {
        const int j = k - un - 1;
        const double y = d.quad[2 * (size_t)j + 1];
        TV[j] = make_float4((float)axis_expm1(y, old.s2, old.s3, ref.lam0), 0.0f, (float)ref.Av[j], (float)y);
      }
    }
  }
  __syncwarp();
  const double nU = bc[0], nV = bc[1], nl = bc[2], lnPn = bc[7];
  for (int k = lane; k < un + vn; k += 32) {
    if (k < un) TU[k].y = (float)axis_expm1(d.quad[2 * (size_t)k * vn], nU, nl, ref.lam0, lnPn);
    else TV[k - un].y = (float)axis_expm1(d.quad[2 * (size_t)(k - un) + 1], nV, nl, ref.lam0);
  }
  __syncwarp();
  const double a3 = bc[5], a4 = bc[6], kn = bc[9], sn = bc[10];
  const double ko = (0.5 * d.K) * nr_rcp(old.s3);
  const double so = 0.8 * (1 - d.Pr) * (old.s3 * old.s3) * nr_rcp(old.s0);
  const float2 fa1 = bc2((float)bc[3]), fa2 = bc2((float)bc[4]), fa3 = bc2((float)a3), fa4 = bc2((float)a4);
#if UGKS_SR_STORE
  const float a1h = (float)bc[3];
  const float2 fa1h = bc2(a1h), fna1h = bc2(-a1h), fna1l = bc2(-(float)(bc[3] - (double)a1h));
  const uint32_t srseed =
      sr_hash((uint32_t)sol.steps * 0x9e3779b9u + (uint32_t)(bi - sol.first_block) * 0x85ebca6bu);
#endif
  const float2 fkbn = bc2((float)kn), fkbo = bc2((float)ko);
  const float2 fdkn = bc2((float)(kn - ref.kb0)), fdko = bc2((float)(ko - ref.kb0));
  // the Shakhov factors weighted by a4 / a3, times the heat flux
  const float2 fSoQx = bc2((float)(a4 * so * Q.x)), fSoQy = bc2((float)(a4 * so * Q.y));
  const float2 fSnQx = bc2((float)(a3 * sn * Q.x)), fSnQy = bc2((float)(a3 * sn * Q.y));
  const float2 fUox = bc2((float)old.s1), fUoy = bc2((float)old.s2), fUnx = bc2((float)nU), fUny = bc2((float)nV);
  const float2 flo2 = bc2((float)(2.0 * old.s3)), fln2 = bc2((float)(2.0 * nl));
  const size_t base = pidx(d, gi, gj, 0);
  const size_t sj = (size_t)NP, si = (size_t)d.Nj * NP;
  float4 *gf = reinterpret_cast<float4 *>(blk.f);
  const float4 *gS = reinterpret_cast<const float4 *>(blk.flux_S), *gW = reinterpret_cast<const float4 *>(blk.flux_W);
  // moments of df' in FP64, products included: the deviation's heat flux
  // nearly cancels the reference's (q is a small difference of large
  // moments), so FP32 sums would dominate its error
  double mom[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) mom[k] = 0.0;
  const double *__restrict__ qd = d.quad;
  const double dUx = nU, dUy = nV, Kinv = nr_rcp(d.K);
  // pair p = a v_num + jv: velocities (2a, jv) and (2a + 1, jv)
  const int qs = 32 / vn, rs = 32 % vn;
  int ia = lane / vn, jv = lane % vn;
#pragma unroll 1
  for (int p = lane; p < NP; p += 32) {
    const size_t k = base + p;
    const float4 f = gf[k], s0 = gS[k], s1 = gS[k + sj], w0 = gW[k], w1 = gW[k + si];
    const float4 ta = TU[2 * ia], tb = TU[2 * ia + 1], tv = TV[jv];
    const float2 qx = make_float2(ta.w, tb.w), qy = bc2(tv.w);
    const float2 m = mul2(make_float2(ta.z, tb.z), bc2(tv.z));  // M of the pair
    const float2 ro = rel_excess(make_float2(ta.x, tb.x), bc2(tv.x));
    const float2 rn = rel_excess(make_float2(ta.y, tb.y), bc2(tv.y));
    const float2 Mo = fma2(m, ro, m), Mn = fma2(m, rn, m);
    const float2 ox = sub2(qx, fUox), oy = sub2(qy, fUoy), o2 = fma2(ox, ox, mul2(oy, oy));
    const float2 nx = sub2(qx, fUnx), ny = sub2(qy, fUny), n2 = fma2(nx, nx, mul2(ny, ny));
    // a4 S and a3 S of the old and new states' Shakhov terms
    const float2 So = fma2(ox, fSoQx, mul2(oy, fSoQy)), Sn = fma2(nx, fSnQx, mul2(ny, fSnQy));
    const float2 po = fma2(flo2, o2, bc2(-4.0f)), pn = fma2(fln2, n2, bc2(-4.0f));
    // fEQ - M of both states, weighted by a4 / a3 (fEQ, clFunctions.c:79-86)
    const float2 eh = fma2(mul2(So, po), Mo, fma2(mul2(Sn, pn), Mn, mul2(m, fma2(fa4, ro, mul2(fa3, rn)))));
    const float2 So_b = fma2(So, po, add2(So, So)), Sn_b = fma2(Sn, pn, add2(Sn, Sn));  // S (P4 + 2)
    const float2 eb = fma2(mul2(fkbo, So_b), Mo,
                           fma2(mul2(fkbn, Sn_b), Mn,
                                mul2(m, fma2(fa4, fma2(fkbo, ro, fdko), mul2(fa3, fma2(fkbn, rn, fdkn))))));
    const float2 flh = add2(sub2(lo2(s0), lo2(s1)), sub2(lo2(w0), lo2(w1)));
    const float2 flb = add2(sub2(hi2(s0), hi2(s1)), sub2(hi2(w0), hi2(w1)));
#if UGKS_SR_STORE
    // stochastic rounding of the new deviation: f a1 + increment as a float
    // pair, rounded to a neighbouring float with probability given by its
    // distance
    const float2 ih = fma2(flh, fa2, eh), ib = fma2(flb, fa2, eb);
    uint32_t h1 = sr_hash((uint32_t)k * 2654435761u ^ srseed), h2 = sr_hash(h1 ^ 0x68e31da4u);
    float2 hh, hl, bh, bl;
    sr_parts(lo2(f), ih, fa1h, fna1h, fna1l, hh, hl);
    sr_parts(hi2(f), ib, fa1h, fna1h, fna1l, bh, bl);
    const float2 oh = make_float2(sr_pick(hh.x, hl.x, h1 & 0xffffu), sr_pick(hh.y, hl.y, h1 >> 16));
    const float2 ob = make_float2(sr_pick(bh.x, bl.x, h2 & 0xffffu), sr_pick(bh.y, bl.y, h2 >> 16));
#else
    const float2 oh = fma2(lo2(f), fa1, fma2(flh, fa2, eh)), ob = fma2(hi2(f), fa1, fma2(flb, fa2, eb));
#endif
    gf[k] = cat2(oh, ob);
    // moments of df' for the next face pass and calcQ of f^{n+1} with the new
    // macro (the deviation's part); a NaN anywhere reaches mom[0] or mom[3].
    // The padding velocity of an odd u_num has df' = 0 and reads velocity 0.
    {
      const double y = qd[2 * (size_t)jv + 1];
      const int ua = 2 * ia, ub = 2 * ia + 1 < un ? 2 * ia + 1 : 0;
      const double xa = qd[2 * (size_t)ua * vn], xb = qd[2 * (size_t)ub * vn];
      const double ha = oh.x, hb = oh.y, ba = ob.x, bb = ob.y;
      const double cy = y - dUy, cxa = xa - dUx, cxb = xb - dUx;
      mom[0] += ha + hb;
      mom[1] = fma(xa, ha, fma(xb, hb, mom[1]));
      mom[2] = fma(y, ha + hb, mom[2]);
      mom[3] += fma(fma(xa, xa, y * y), ha, fma(fma(xb, xb, y * y), hb, ba + bb));
      const double ta = fma(fma(cxa, cxa, cy * cy), ha, ba * Kinv);
      const double tb = fma(fma(cxb, cxb, cy * cy), hb, bb * Kinv);
      mom[4] = fma(cxa, ta, fma(cxb, tb, mom[4]));
      mom[5] = fma(cy, ta + tb, mom[5]);
    }
    jv += rs;
    ia += qs;
    if (jv >= vn) { jv -= vn; ++ia; }
  }
  double dm[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) dm[k] = mom[k];
  warp_sum<6>(dm);
  if (lane == 0) {
    if (isnan(dm[0]) || isnan(dm[3])) atomicExch(&sol.status, 1);
    st4(blk.cell_mom, gidx(d, gi, gj),
        p4(R[RM00] + dm[0], R[RM10] + dm[1], R[RM01] + dm[2], 0.5 * ((R[RM20] + R[RM02] + R[RB00]) + dm[3])));
    const V2 qr = heat_flux_from_moments(R, d.K, v2(nU, nV));
    st2(blk.Q_next, midx(d, mi, mj), v2(qr.x + 0.5 * dm[4], qr.y + 0.5 * dm[5]));
  }
}

// ---------------------------------------------------------------------------
// ghost pass on the deviations (ghost_pass's branches): copies, permutations
// and the constant-gradient extrapolation act on df unchanged (M is the same
// in every cell and symmetric under the mirror permutations); equilibrium
// ghosts are fEQ - M in FP64, rounded once
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(FT) ghost_pass_delta(const ugks_fused_block *__restrict__ B, int nb,
                                                       const ugks_solve_state *__restrict__ solves) {
  __shared__ double scratch[4 * (FT / 32)];
  const int w = blockIdx.x;
  const int bi = find_block<2>(B, nb, w);
  const ugks_fused_block &blk = B[bi];
  const ugks_block_desc &d = blk.d;
  UGKS_CHECK_ITEM(2, blk, w, solves);
  if (!solves[blk.solve].active) return;
  const RefMaxwellian ref = ref_of(blk);
  const int G = d.ghost, Nv = d.Nv, NP = npairs(d), vn = d.v_num;
  int lc = w - blk.ghost_begin;
  int face = 0;
  const int ns_cells = d.ni * G, ew_cells = G * d.nj;
  for (face = 0; face < 4; ++face) {
    const int c = (face == GNORTH || face == GSOUTH) ? ns_cells : ew_cells;
    if (lc < c) break;
    lc -= c;
  }
  long a, b;
  if (face == GNORTH || face == GSOUTH) { a = lc / G; b = lc % G; }
  else { a = lc / d.nj; b = lc % d.nj; }
  long gi = a, gj = b;
  switch (face) {
    case GNORTH: gi += G; gj += d.Nj - G; break;
    case GEAST: gi += d.Ni - G; gj += G; break;
    case GSOUTH: gi += G; break;
    default: gj += G; break;
  }
  float4 *dst = reinterpret_cast<float4 *>(blk.f) + pidx(d, gi, gj, 0);
  const int t = blk.bc_type[face];
  // deviation moments of the ghost cell (velocity by velocity)
  double mom[4] = {0.0, 0.0, 0.0, 0.0};
  auto tally = [&](int v, float h, float bb) {
    const V2 e = quad_at(d, v);
    mom[0] += h;
    mom[1] = fma(e.x, (double)h, mom[1]);
    mom[2] = fma(e.y, (double)h, mom[2]);
    mom[3] += fma(fma(e.x, e.x, e.y * e.y), (double)h, (double)bb);
  };
  // a gather of velocities perm[v] (or v) from another cell, pair by pair
  // the velocities of pair p: (2a, jv) and (2a + 1, jv), p = a v_num + jv
  auto lanes = [&](int p, int &va, int &vb) {
    const int a = p / vn, jv = p - a * vn;
    va = 2 * a * vn + jv;
    vb = va + vn;
  };
  auto gather = [&](const float4 *src, const int32_t *perm) {
    if (perm == nullptr) {
      // a plain copy: GHOST_U loads per thread in flight before the first
      // store (a store may alias a later load, so the compiler keeps them in
      // program order)
      for (int p0 = threadIdx.x; p0 < NP; p0 += GHOST_U * FT) {
        float4 o[GHOST_U];
#pragma unroll
        for (int u = 0; u < GHOST_U; ++u)
          if (p0 + u * FT < NP) o[u] = src[p0 + u * FT];
#pragma unroll
        for (int u = 0; u < GHOST_U; ++u) {
          const int p = p0 + u * FT;
          if (p < NP) {
            dst[p] = o[u];
            int va, vb;
            lanes(p, va, vb);
            tally(va, o[u].x, o[u].z);
            if (vb < Nv) tally(vb, o[u].y, o[u].w);
          }
        }
      }
      return;
    }
    for (int p = threadIdx.x; p < NP; p += FT) {
      int va, vb;
      lanes(p, va, vb);
      float4 o;
      if (perm == nullptr) {
        o = src[p];
      } else {
        const int sa = perm[va];
        o.x = pair_get(src, sa, vn, 0);
        o.z = pair_get(src, sa, vn, 1);
        if (vb < Nv) {
          const int sb = perm[vb];
          o.y = pair_get(src, sb, vn, 0);
          o.w = pair_get(src, sb, vn, 1);
        } else {
          o.y = o.w = 0.0f;
        }
      }
      dst[p] = o;
      tally(va, o.x, o.z);
      if (vb < Nv) tally(vb, o.y, o.w);
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
    if (iB < 0 || iB >= NIB || jB < 0 || jB >= NJB || ob.d.Nv != Nv || ob.ref != blk.ref) {
      // connection that does not map onto the neighbour: flag, do not read
      if (threadIdx.x == 0) atomicExch(const_cast<int32_t *>(&solves[blk.solve].status), 6);
      return;
    }
    const float4 *src = reinterpret_cast<const float4 *>(ob.f) + ((size_t)iB * NJB + jB) * (size_t)NP;
    const int flip = blk.bc_flip[face];
    gather(src, flip == NO_FLIP ? nullptr : (flip == FLIP_NS ? d.mirror_NS : (flip == FLIP_D ? d.mirror_D : d.mirror_EW)));
  } else if (t == BC_DIFFUSE || t == BC_ADSORBING) {
    // edgeConstGrad (clGhostRoutines.c:967-1048): f1 + m (f1 - f0), linear
    // with weights summing to one, so the same on df
    long ei0, ej0, ei1, ej1;
    float m;
    switch (face) {
      case GNORTH: ei1 = gi; ej1 = d.Nj - G - 1; ei0 = ei1; ej0 = ej1 - 1; m = (float)(gj - ej1); break;
      case GEAST: ei1 = d.Ni - G - 1; ej1 = gj; ei0 = ei1 - 1; ej0 = ej1; m = (float)(gi - ei1); break;
      case GSOUTH: ei1 = gi; ej1 = G; ei0 = ei1; ej0 = ej1 + 1; m = (float)(ej1 - gj); break;
      default: ei1 = G; ej1 = gj; ei0 = ei1 + 1; ej0 = ej1; m = (float)(ei1 - gi); break;
    }
    const float4 *c0 = reinterpret_cast<const float4 *>(blk.f) + pidx(d, ei0, ej0, 0);
    const float4 *c1 = reinterpret_cast<const float4 *>(blk.f) + pidx(d, ei1, ej1, 0);
    const float2 fm = bc2(m);
    for (int p0 = threadIdx.x; p0 < NP; p0 += GHOST_U * FT) {
      float4 x0[GHOST_U], x1[GHOST_U];
#pragma unroll
      for (int u = 0; u < GHOST_U; ++u)
        if (p0 + u * FT < NP) {
          x0[u] = c0[p0 + u * FT];
          x1[u] = c1[p0 + u * FT];
        }
#pragma unroll
      for (int u = 0; u < GHOST_U; ++u) {
        const int p = p0 + u * FT;
        if (p < NP) {
          const float2 h = fma2(fm, sub2(lo2(x1[u]), lo2(x0[u])), lo2(x1[u]));
          const float2 bb = fma2(fm, sub2(hi2(x1[u]), hi2(x0[u])), hi2(x1[u]));
          dst[p] = cat2(h, bb);
          int va, vb;
          lanes(p, va, vb);
          tally(va, h.x, bb.x);
          if (vb < Nv) tally(vb, h.y, bb.y);
        }
      }
    }
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
    gather(reinterpret_cast<const float4 *>(blk.f) + pidx(d, si, sj, 0), perm);
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
    for (int v = threadIdx.x; v < Nv; v += FT) {
      const V2 e = shakhov_eq(d, prim, Q, quad_at(d, v), v);
      const double mh = ref.mh[v];
      const float h = (float)(e.x - mh), bb = (float)(e.y - ref.kb0 * mh);
      pair_put(dst, v, vn, h, bb);
      tally(v, h, bb);
    }
    for (int v = Nv + threadIdx.x; v < 2 * NP; v += FT) pair_put(dst, v, vn, 0.0f, 0.0f);  // padding lanes
  }
  block_sum<4>(mom, scratch);
  if (threadIdx.x == 0) {
    const double *R = ref.mom;
    st4(blk.cell_mom, gidx(d, gi, gj),
        p4(R[RM00] + mom[0], R[RM10] + mom[1], R[RM01] + mom[2], 0.5 * ((R[RM20] + R[RM02] + R[RB00]) + mom[3])));
  }
}

// ---------------------------------------------------------------------------
// start-up (initFunctions + calcMacro + calcQ, ugks_block.py:411-429) and
// restart from saved distributions, on the deviations
// ---------------------------------------------------------------------------
// macro := moments of the stored f; Q and Q_next := calcQ with that macro
// (restart: the loaded macro); cell_mom := the moments; CFL frequency
template <bool FRESH>
__global__ void __launch_bounds__(FT) setup_cells_delta(const ugks_fused_block *__restrict__ B, int nb,
                                                        ugks_solve_state *__restrict__ solves) {
  __shared__ double scratch[RNMOM * (FT / 32)];
  const int w = blockIdx.x;
  const int bi = find_block<1>(B, nb, w);
  const ugks_fused_block &blk = B[bi];
  const ugks_block_desc &d = blk.d;
  UGKS_CHECK_ITEM(1, blk, w, solves);
  ugks_solve_state &sol = solves[blk.solve];
  if (!sol.active) return;
  const RefMaxwellian ref = ref_of(blk);
  const int lc = w - blk.cell_begin;
  const long mi = lc / d.nj, mj = lc % d.nj;
  float4 *cell = reinterpret_cast<float4 *>(blk.f) + pidx(d, mi + d.ghost, mj + d.ghost, 0);
  P4 prim = ld4(blk.macro, midx(d, mi, mj));
  const V2 Q0 = ld2(blk.Q, midx(d, mi, mj));
  double m[RNMOM];
#pragma unroll
  for (int k = 0; k < RNMOM; ++k) m[k] = 0.0;
  for (int v = threadIdx.x; v < d.Nv; v += FT) {
    const V2 e = quad_at(d, v);
    float h, bb;
    if (FRESH) {
      // initFunctions: f := fEQ(macro, Q), stored as its deviation from M
      const V2 f = shakhov_eq(d, prim, Q0, e, v);
      h = (float)(f.x - ref.mh[v]);
      bb = (float)(f.y - ref.kb0 * ref.mh[v]);
      pair_put(cell, v, d.v_num, h, bb);
    } else {
      h = pair_get(cell, v, d.v_num, 0);
      bb = pair_get(cell, v, d.v_num, 1);
    }
    // raw moments of the stored deviation (global frame)
    const double x = e.x, y = e.y, dh = h, db = bb;
    m[RM00] += dh; m[RM10] += x * dh; m[RM01] += y * dh;
    m[RM20] += x * x * dh; m[RM11] += x * y * dh; m[RM02] += y * y * dh;
    m[RM30] += x * x * x * dh; m[RM21] += x * x * y * dh; m[RM12] += x * y * y * dh; m[RM03] += y * y * y * dh;
    m[RB00] += db; m[RB10] += x * db; m[RB01] += y * db;
  }
  block_sum<RNMOM>(m, scratch);
  if (threadIdx.x == 0) {
    const double *R = ref.mom;
    double T[RNMOM];
#pragma unroll
    for (int k = 0; k < RNMOM; ++k) T[k] = R[k] + m[k];
    const P4 mom = p4(T[RM00], T[RM10], T[RM01], 0.5 * (T[RM20] + T[RM02] + T[RB00]));
    if (FRESH) {
      prim = to_primary(d, mom);  // calcMacro
      st4(blk.macro, midx(d, mi, mj), prim);
    }
    st4(blk.cell_mom, gidx(d, mi + d.ghost, mj + d.ghost), mom);
    const V2 q = heat_flux_from_moments(T, d.K, v2(prim.s1, prim.s2));  // calcQ
    if (FRESH) st2(blk.Q, midx(d, mi, mj), q);
    st2(blk.Q_next, midx(d, mi, mj), q);
    const double fq = cfl_freq(blk, prim, mi, mj);
    atomicMax(&sol.max_freq, (unsigned long long)__double_as_longlong(fq));
  }
}
