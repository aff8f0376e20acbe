/* ugks_b200.h -- C ABI of libugks_b200.so, the B200 (sm_100a) UGKS time step.
 *
 * Two layers, both plain pointers and sizes:
 *
 *  1. Drop-in kernels.  One entry point per pyUGKS OpenCL kernel on the
 *     time-step path, with the reference kernel's name, argument order and
 *     meaning.  A pyUGKS-style driver that called
 *         self.prg.<name>(queue, global_size, local_size, *args)
 *     calls ugks_<name>(desc, g0, g1, *args, stream) instead: `desc` replaces
 *     the per-block #define header that ugks_CL.py:20-400 generated, (g0, g1)
 *     is the reference NDRange (work-group size is irrelevant here), every
 *     buffer is a device pointer in the reference layout (source/clKernel.c:4-26):
 *         f-like     [(i*Nj + j)*Nv + v] x (h, b)         (double2)
 *         macro      [i*nj + j] x (rho, U, V, 1/T)        (double4, no ghosts)
 *         per face   [(i*Nj + j)*2 + face]                (face 0 = SOUTH, 1 = WEST)
 *     Each returns 0 on success or a negative cudaError_t on a launch error.
 *     Nothing is synchronised; work is queued on `stream` (a cudaStream_t,
 *     NULL = legacy default stream).
 *
 *  2. Fused step.  ugks_step_* run a whole UGKS step (both face directions,
 *     walls, cell update, dt control, ghost exchange) for every block of every
 *     solve listed in a device-resident block table, with no host
 *     synchronisation, so that a caller can capture steps in a CUDA graph.
 *
 * The library never allocates, frees or keeps device memory: every buffer
 * belongs to the caller and is borrowed for the duration of the call.
 */
#ifndef UGKS_B200_H
#define UGKS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------
 * Per-block constants: what the reference baked into each block's OpenCL
 * header (ugks_CL.py:58-96, 102-156, 270-395).
 * --------------------------------------------------------------------- */
typedef struct ugks_block_desc {
  int32_t ni, nj;        /* interior cells                                  */
  int32_t Ni, Nj;        /* with ghosts: ni + 2*ghost, nj + 2*ghost         */
  int32_t ghost;         /* 2 (vanLeer/minmod) or 3 (WENO5)                 */
  int32_t Nv;            /* discrete velocities                             */
  int32_t flux_method;   /* 0 vanLeer, 1 WENO5, 3 minmod                    */
  int32_t relax_type;    /* relaxTime variant 0..3 (clFunctions.c:8-32)     */
  double PI, Pr, umax, vmax, Kn_eff, gam, K, omega;
  const double *quad;         /* device [Nv][2] global velocities          */
  const double *weight;       /* device [Nv] quadrature weights            */
  const int32_t *mirror_NS;   /* device [Nv] velocity permutations         */
  const int32_t *mirror_EW;
  const int32_t *mirror_D;
  /* wall values of faces N, E, S, W (WALL_<f>_{D,U,V,T,P}; T holds 1/T) */
  double wall_D[4], wall_U[4], wall_V[4], wall_T[4], wall_P[4];
  /* adsorbing walls (BETA_N, BETA_T, GAMMA_F, ALPHA_P, ADSORB_<face>)      */
  double beta_n[4], beta_t[4], gamma_f[4], alpha_p[4], adsorb[4];
  /* first-order desorption rate (0 = the reference's Langmuir desorption) */
  double k_des[4];
  int32_t dynamic[4];          /* DYNAMIC_VARTHETA                         */
  int32_t constant_adsorb[4];  /* CONSTANT_ADSORB_<face>                   */
  /* tensor velocity grid: v = iu * v_num + jv with quad[v] = (u_iu, v_jv)
     (ugks_data.py:287-292); u_num * v_num == Nv lets the fused kernels
     factor the Maxwellian exponential; 0 for an unstructured set */
  int32_t u_num, v_num;
  /* adsorbing-wall re-emission per face: UGKS_REFLECT_SPECULAR (the
     reference's default 'S'), _DIFFUSE ('D') or _CL (Cercignani-Lampis with
     accommodation ALPHA_N, ALPHA_T; ugks_CL.py:134-148, 255-273) */
  double alpha_n[4], alpha_t[4];
  int32_t reflect[4];
  /* tabulated isotherms (constant_adsorb[f] == 0; ISO_, TRI_, NBR_<face>,
     N_TRI, ugks_CL.py:158-252): device [n][4] points (P, T, theta, 0), the
     [n_tri][4] Delaunay triangles of (P, T) and their [n_tri][4] neighbours
     (-1: none) */
  const double *iso[4];
  const int32_t *tri[4];
  const int32_t *nbr[4];
  int32_t n_tri[4];
  double B;              /* degrees of freedom b (getInternal's T divisor)  */
} ugks_block_desc;

#define UGKS_REFLECT_SPECULAR 0
#define UGKS_REFLECT_DIFFUSE 1
#define UGKS_REFLECT_CL 2

/* ------------------------------------------------------------------------
 * 1. Drop-in kernels (reference: source/clUGKS.c, clKernel.c,
 *    clGhostRoutines.c, clAdsorb.c).  Arguments follow the __kernel
 *    signatures; double2/double4/double8 buffers are double* here.
 * --------------------------------------------------------------------- */
#define UGKS_STREAM void *stream

/* clUGKS.c:110-199 */
int ugks_iFace(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin, double *iface_f,
               double *fsigma, const double *centre, const double *mid_side, const double *normal,
               int face, UGKS_STREAM);
/* clUGKS.c:209-271 */
int ugks_getFaceCons(const ugks_block_desc *d, size_t g0, size_t g1, const double *iface_f,
                     const double *normal, int face, double *primary, int offset_bottom,
                     int offset_top, UGKS_STREAM);
/* clUGKS.c:273-335 */
int ugks_getAL(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin,
               const double *normal, int face, double *gaL, int offset_bottom, int offset_top,
               UGKS_STREAM);
/* clUGKS.c:337-399 */
int ugks_getAR(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin,
               const double *normal, int face, double *gaR, int offset_bottom, int offset_top,
               UGKS_STREAM);
/* clUGKS.c:401-442 */
int ugks_getPLR(const ugks_block_desc *d, size_t g0, size_t g1, const double *centre,
                const double *mid_side, int face, double *primary, double *gaL, double *gaR,
                int offset_bottom, int offset_top, UGKS_STREAM);
/* clUGKS.c:446-518 */
int ugks_initMacroFlux(const ugks_block_desc *d, size_t g0, size_t g1, double *flux_macro,
                       int face, double dt, const double *primary, const double *gaL,
                       const double *gaR, double *gaT, double *gMxi, int offset_bottom,
                       int offset_top, UGKS_STREAM);
/* clUGKS.c:522-585 */
int ugks_calcFaceQ(const ugks_block_desc *d, size_t g0, size_t g1, const double *iface_f,
                   const double *primary, const double *normal, double *faceQ, int face,
                   int offset_bottom, int offset_top, UGKS_STREAM);
/* clUGKS.c:587-681 */
int ugks_macroFlux(const ugks_block_desc *d, size_t g0, size_t g1, const double *flux_f,
                   const double *fsigma, double *flux_macro, const double *normal,
                   const double *side_length, int face, double dt, const double *primary,
                   const double *faceQ, int offset_bottom, int offset_top, UGKS_STREAM);
/* clUGKS.c:683-772 */
int ugks_distFlux(const ugks_block_desc *d, size_t g0, size_t g1, double *flux_f,
                  const double *fsigma, const double *normal, const double *side_length, int face,
                  double dt, const double *primary, const double *gaL, const double *gaR,
                  const double *gaT, const double *gMxi, const double *faceQ, int offset_bottom,
                  int offset_top, UGKS_STREAM);
/* clUGKS.c:774-906 */
int ugks_accommodatingWallDist(const ugks_block_desc *d, size_t g0, size_t g1,
                               const double *normal, int face, const double *wall_prop,
                               double *flux_f, double dt, UGKS_STREAM);
/* clUGKS.c:910-1011 */
int ugks_wallFlux(const ugks_block_desc *d, size_t g0, size_t g1, const double *normal,
                  const double *side_length, int face, double *flux_f, double *flux_macro,
                  double dt, UGKS_STREAM);
/* clUGKS.c:1019-1147 */
int ugks_wallMassEnergyFluxes(const ugks_block_desc *d, size_t g0, size_t g1,
                              const double *normal, const double *side_length, const double *area,
                              int face, const double *flux_f, double *wall_flux, double dt,
                              UGKS_STREAM);
/* clUGKS.c:1158-1187 */
int ugks_updateMacro(const ugks_block_desc *d, size_t g0, size_t g1, const double *flux_macro_S,
                     const double *flux_macro_W, const double *area, double *macro,
                     double *residual, UGKS_STREAM);
/* clUGKS.c:1189-1257; flag[0] becomes 1.0 if any new f is NaN */
int ugks_UGKS_update(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin,
                     const double *flux_f_S, const double *flux_f_W, const double *area,
                     const double *macro, const double *gQ, const double *residual, double dt,
                     double *flag, UGKS_STREAM);
/* clUGKS.c:1259-1277 */
int ugks_getResidual(const ugks_block_desc *d, size_t g0, size_t g1, const double *macro,
                     double *residual, UGKS_STREAM);
/* clUGKS.c:1282-1337 */
int ugks_edgeMassFlow(const ugks_block_desc *d, size_t g0, size_t g1, const double *macro,
                      const double *normal, const double *side_length, double *mdot,
                      int this_face, UGKS_STREAM);
/* clKernel.c:480-543 */
int ugks_calcQ(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin,
               const double *macro, double *gQ, UGKS_STREAM);
/* clKernel.c:414-478 */
int ugks_calcMacro(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin,
                   double *macro, UGKS_STREAM);
/* clKernel.c:382-412 */
int ugks_initFunctions(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin,
                       const double *macro, const double *gQ, UGKS_STREAM);
/* clKernel.c:224-308 */
int ugks_clFindDT(const ugks_block_desc *d, size_t g0, size_t g1, const double *xy,
                  const double *area, const double *macro, double *time_step, double Kn,
                  UGKS_STREAM);
/* pyopencl.array.max of ugks_block.py:1426: out[0] = max(x[0..n)) */
int ugks_array_max(const double *x, size_t n, double *out, UGKS_STREAM);
/* clKernel.c:141-218 (constant wall values; para_def and t are unused there) */
int ugks_paraBC(const ugks_block_desc *d, size_t g0, size_t g1, const double *para_def,
                double *wall_prop, double t, UGKS_STREAM);
/* clGhostRoutines.c:407-538; fB, xyB belong to the neighbour block */
int ugks_edgeExchange(const ugks_block_desc *d, size_t g0, size_t g1, double *fA,
                      const double *xyA, int this_face, const double *fB, const double *xyB,
                      int NIB, int NJB, int that_face, int ori, int flip, UGKS_STREAM);
/* clGhostRoutines.c:544-597 */
int ugks_edgeExtrapolate(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin,
                         int this_face, UGKS_STREAM);
/* clGhostRoutines.c:603-658 */
int ugks_edgeConstant(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin,
                      int this_face, const double *wall_prop, UGKS_STREAM);
/* clGhostRoutines.c:664-749 */
int ugks_edgeInflow(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin, int this_face,
                    const double *normal, const double *macro, const double *gQ,
                    const double *wall_prop, UGKS_STREAM);
/* clGhostRoutines.c:755-839 */
int ugks_edgeOutflow(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin,
                     int this_face, const double *normal, const double *macro, const double *gQ,
                     const double *wall_prop, UGKS_STREAM);
/* clGhostRoutines.c:845-905 */
int ugks_edgeMirror(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin, int this_face,
                    UGKS_STREAM);
/* clGhostRoutines.c:911-961 */
int ugks_edgeBounceBack(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin,
                        int this_face, UGKS_STREAM);
/* clGhostRoutines.c:967-1048 */
int ugks_edgeConstGrad(const ugks_block_desc *d, size_t g0, size_t g1, double *Fin,
                       int this_face, UGKS_STREAM);
/* clAdsorb.c:253-482; flag[0] becomes 4.0 for a tabulated isotherm (not supported) */
int ugks_adsorbingWall_P1(const ugks_block_desc *d, size_t g0, size_t g1, const double *normal,
                          int face, const double *wall_prop, double *wall_cover,
                          double *wall_dist, const double *flux_f, const double *macro,
                          double dt, double *flag, UGKS_STREAM);
/* clAdsorb.c:821-975 */
int ugks_adsorbingWallD_P2(const ugks_block_desc *d, size_t g0, size_t g1, const double *normal,
                           int face, const double *wall_prop, const double *wall_cover,
                           const double *wall_dist, double *flux_f, const double *macro,
                           double dt, UGKS_STREAM);
/* clKernel.c:314-375: per interior cell the directional temperatures
   Txyz = (Tx, Ty, Tz, T) and the stress (tau_xx, tau_xy, tau_yy, 0) */
int ugks_getInternal(const ugks_block_desc *d, size_t g0, size_t g1, const double *Fin, double *Txyz,
                     double *Stress, UGKS_STREAM);

/* Geometry set-up (UGKSBlock.updateGeom, ugks_block.py:667-760).
   clGhostRoutines.c:155-284: ghost vertices from the neighbouring block */
int ugks_xyExchange(const ugks_block_desc *d, size_t g0, size_t g1, double *xyA, int this_face,
                    const double *xyB, int NIB, int NJB, int that_face, int ori, int affine,
                    int flip_normal, int this_block_id, int that_block_id, UGKS_STREAM);
/* clGhostRoutines.c:291-398: ghost vertices by extrapolation */
int ugks_xyExtrapolate(const ugks_block_desc *d, size_t g0, size_t g1, double *xy, int this_face,
                       UGKS_STREAM);
/* clKernel.c:31-135: normals, areas, centroids, mid-sides, side lengths */
int ugks_cellGeom(const ugks_block_desc *d, size_t g0, size_t g1, const double *xy, double *area,
                  double *centre, double *mid_side, double *normal, double *side_length, UGKS_STREAM);

/* clAdsorb.c:656-816: specular re-emission of the reflected flux */
int ugks_adsorbingWallS_P2(const ugks_block_desc *d, size_t g0, size_t g1, const double *normal,
                           int face, const double *wall_prop, const double *wall_cover,
                           const double *wall_dist, double *flux_f, const double *macro,
                           double dt, UGKS_STREAM);
/* clAdsorb.c:488-651: Cercignani-Lampis re-emission of the reflected flux */
int ugks_adsorbingWallCL_P2(const ugks_block_desc *d, size_t g0, size_t g1, const double *normal,
                            int face, const double *wall_prop, const double *wall_cover,
                            const double *wall_dist, double *flux_f, const double *macro,
                            double dt, UGKS_STREAM);

/* ------------------------------------------------------------------------
 * 2. Fused step.
 *
 * A solve is one pyUGKS simulation (UGKSim); it owns one or more blocks.
 * The caller keeps, in device memory, an array of ugks_fused_block (one per
 * block of every solve) and an array of ugks_solve_state (one per solve).
 *
 * *_fp64: f and the two face-flux arrays of a block are FP64 in the reference
 * layout [Ni][Nj][Nv] x (h, b).
 *
 * *_mixed: they are FP32 *deviations* from a reference Maxwellian M of the
 * solve (ugks_fused_block.ref): f = M + df and
 * flux = dt len (u . n) M + dflux, in a velocity-pair layout
 * [Ni][Nj][(Nv + 1) / 2] x (h_2p, h_2p+1, b_2p, b_2p+1); an odd Nv pads the
 * last pair with a velocity whose entries stay 0.  The tensor velocity grid
 * (u_num * v_num == Nv) is required.  Moments, the conserved update, the
 * relaxation, dt and the residual stay FP64 in both.
 * --------------------------------------------------------------------- */

/* Reference Maxwellian of a mixed-precision solve: a device array of doubles
 * shared by the solve's blocks, written once by the caller:
 *   [UGKS_REF_LAMBDA] lambda0 = 1/T0, [UGKS_REF_P0] rho0 lambda0 / pi,
 *   [UGKS_REF_KB0] K / (2 lambda0),
 *   [UGKS_REF_MOM + k] the 13 sums over v of mh (1, u, v, u^2, u v, v^2,
 *     u^3, u^2 v, u v^2, v^3) and of kb0 mh (1, u, v), (u, v) = quad[v],
 *   [UGKS_REF_TAB + v] mh[v] = weight[v] rho0 lambda0 / pi exp(-lambda0 |quad[v]|^2),
 *   then Au[u_num], Av[v_num] with mh(iu, jv) = Au[iu] Av[jv] (to rounding). */
#define UGKS_REF_LAMBDA 0
#define UGKS_REF_P0 1
#define UGKS_REF_KB0 2
#define UGKS_REF_MOM 4
#define UGKS_REF_TAB 32
/* doubles per face of ugks_fused_block.face_rec (the mixed face pass's
 * per-face record: the deviation's moments, the flux coefficients and the
 * face state, handed from one launch of the pass to the next) */
#define UGKS_FACE_REC 48
typedef struct ugks_fused_block {
  ugks_block_desc d;           /* sizes, constants, tables, wall values    */
  int32_t solve;               /* index of the owning ugks_solve_state     */
  int32_t bc_type[4];          /* per face N,E,S,W: geom_bc_defs.py codes  */
  int32_t bc_block[4];         /* ADJACENT: index (in this table) of the neighbour */
  int32_t bc_face[4];          /* ADJACENT: neighbour face                 */
  int32_t bc_ori[4];           /* ADJACENT: orientation flag               */
  int32_t bc_flip[4];          /* ADJACENT: velocity permutation code      */
  int32_t face_begin;          /* first face work item of this block       */
  int32_t cell_begin;          /* first cell work item                     */
  int32_t ghost_begin;         /* first ghost-cell work item               */
  int32_t wall_begin;          /* first wall-face work item (2 (ni + nj) per block:
                                  S faces of rows 0 and nj, W faces of columns 0 and ni) */
  void *f;                     /* [Ni][Nj][Nv] x (h, b), double or float    */
  void *flux_S;                /* [Ni][Nj][Nv] x (h, b), SOUTH-face fluxes  */
  void *flux_W;                /* WEST-face fluxes                          */
  double *flux_macro_S;        /* [Ni][Nj] x 4                              */
  double *flux_macro_W;
  double *macro;               /* [ni][nj] x (rho, U, V, 1/T)               */
  double *Q;                   /* [ni][nj] x 2 heat flux                    */
  double *prim_old;            /* [ni][nj] x 4 (the reference's residual buffer) */
  const double *area;          /* [Ni][Nj]                                  */
  const double *centre;        /* [Ni][Nj] x 2                              */
  const double *mid_side;      /* [Ni][Nj][2] x 2                           */
  const double *normal;        /* [Ni][Nj][2] x 2                           */
  const double *side_length;   /* [Ni][Nj][2]                               */
  const double *xy;            /* [Ni+1][Nj+1] x 2                          */
  double *wall_prop;           /* [max(ni,nj)][4] x 4                       */
  double *wall_cover;          /* [max(ni,nj)][4] x 4                       */
  double *wall_fluxes;         /* [max(ni,nj)][4] x 8                       */
  double *wall_dist;           /* [max(ni,nj)][Nv] x 2                      */
  double *cell_mom;            /* [Ni][Nj] x 4: sum over v of f (1, u, v,
                                  (u^2+v^2)/2 | 1/2) per cell, global frame;
                                  written by the init, cell and ghost passes,
                                  read by the face pass (getAL/getAR)       */
  double *Q_next;              /* [ni][nj] x 2: calcQ of f^{n+1} with the macro of
                                  step n+1, accumulated by the cell pass of step n
                                  and moved to Q by the cell pass of step n+1 */
  double *face_geo;            /* [Ni][Nj][2] x 6: reconstruction geometry of every
                                  face (iFace, clUGKS.c:148-176): |mid - c|, its
                                  reciprocal and 1/|c - c'| for the u <= 0 stencil,
                                  then the same for u > 0; written by ugks_init_* and
                                  ugks_restart_* from centre and mid_side */
  const double *ref;           /* *_mixed only: the solve's reference Maxwellian
                                  (UGKS_REF_* layout above), the same array for
                                  every block of the solve; unused by *_fp64 */
  void *aux_S;                 /* *_mixed only: scratch of the face pass, shaped like
                                  flux_S: the slopes of the SOUTH-face deviations */
  void *aux_W;                 /* *_mixed only: the same for the WEST faces */
  double *face_rec;            /* *_mixed only: [Ni][Nj][2] x UGKS_FACE_REC scratch */
} ugks_fused_block;

typedef struct ugks_solve_state {
  double dt;                   /* current time step                         */
  double time;                 /* simulated time                            */
  double CFL;
  double delta_dt;             /* dt growth limit (ugks_sim.py:306)         */
  double max_dt;               /* CFL / max frequency of the last dt update */
  unsigned long long max_freq; /* bits of the running max CFL frequency (atomicMax) */
  int32_t retry;               /* 1 while this step's flux pass is redone   */
  int32_t status;              /* 0 ok, 1 NaN in f, 4 isotherm, 6 bad block
                                  connection (clError.c codes otherwise), 8 a bulk
                                  copy of the face pass outlived its wait bound */
  int32_t steps;               /* completed steps                           */
  int32_t retries;             /* flux passes redone so far                 */
  int32_t active;              /* 0: skipped by every fused kernel          */
  int32_t nblocks;             /* blocks of this solve                      */
  int32_t first_block;         /* index of its first block in the table     */
  int32_t stopped;             /* set by ugks_stop_check: 0 running, UGKS_STOP_* */
  double residual[4];          /* written by ugks_residual: mean over blocks
                                  of sqrt(ni nj sum (dprim)^2) / sum |prim|
                                  (ugks_block.py:1319-1327, ugks_sim.py:463-468) */
  double stop_residual;        /* stop rule: density residual below this (0: none) */
  int32_t stop_steps;          /* stop rule: this many completed steps (0: none)   */
  int32_t stop_after;          /* the residual rule applies from this many completed
                                  steps on (the reference's residual_start, 10) */
} ugks_solve_state;

#define UGKS_STOP_CONVERGED 1
#define UGKS_STOP_STEPS 2
#define UGKS_STOP_ERROR 3

#define UGKS_MAX_FACE_SEGMENTS 16

/* Work sizes of a block table, computed on the host by ugks_fused_layout. */
typedef struct ugks_fused_sizes {
  int32_t n_faces;        /* face work items (2 per cell corner of every block) */
  int32_t n_cells;        /* interior cells                                    */
  int32_t n_ghost;        /* ghost cells of the four strips of every block     */
  int32_t max_nv;         /* largest Nv (sizes the face pass's shared memory)  */
  int32_t face_begin[4];  /* first face work item of the blocks of flux_method k */
  int32_t face_count[4];  /* their number (0 when no block uses method k)      */
  int32_t max_axes;       /* largest u_num + v_num of a tensor velocity grid   */
  /* face-pass launches: runs of consecutive blocks with one flux method and
     one Nv (merged within a method when there are more than
     UGKS_MAX_FACE_SEGMENTS), each launched with shared memory for its own Nv */
  int32_t n_segments;
  int32_t seg_begin[UGKS_MAX_FACE_SEGMENTS];
  int32_t seg_count[UGKS_MAX_FACE_SEGMENTS];
  int32_t seg_method[UGKS_MAX_FACE_SEGMENTS];
  int32_t seg_max_nv[UGKS_MAX_FACE_SEGMENTS];
  int32_t seg_max_axes[UGKS_MAX_FACE_SEGMENTS];
  /* launch shape per face-pass segment (0 by velocity count; 1..4 force one
     of the compiled shapes, ugks_fused.cu FaceShape) and of the cell pass
     (0 default; 2 or 3 CTAs of 8 warps per SM); ugks_fused_layout sets 0, a
     caller (the autotuner) may change them before stepping.  The shape
     changes the order of the per-face sums, not the arithmetic: results agree
     to round-off across shapes and are reproducible for a fixed shape. */
  int32_t seg_variant[UGKS_MAX_FACE_SEGMENTS];
  int32_t cell_variant;
  int32_t n_wall;         /* wall-face work items (2 (ni + nj) per block)          */
} ugks_fused_sizes;

#define UGKS_FACE_VARIANTS 5

/* Fills face_begin/cell_begin/ghost_begin of the host copy `blocks` and the
   sizes.  The blocks of one solve must be contiguous and in the order of
   their solve index, and the blocks of one flux method contiguous (group the
   solves by flux method).  Returns 0, -1 when a count exceeds INT32_MAX, -2
   when the ordering rule is broken, -3 when a block fails validation (sizes
   inconsistent with its ghost layers or its flux method's stencil, a missing
   array or table, a connection outside the table or to a face of another
   extent, velocity count or solve): a corrupted table is rejected here,
   before any kernel could index outside its arrays. */
int ugks_fused_layout(ugks_fused_block *blocks, int nblocks, ugks_fused_sizes *sizes);

/* Initial state (ugks_block.py:411-429, ugks_sim.py:88-92): f := fEQ(macro,
   Q) on interior cells, macro := moments(f), Q := heat flux(f), wall_prop
   from the wall values, ghosts filled, dt := CFL / max frequency. */
int ugks_init_fp64(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                   ugks_solve_state *solves_dev, int nsolves, UGKS_STREAM);
int ugks_init_mixed(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                    ugks_solve_state *solves_dev, int nsolves, UGKS_STREAM);

/* Restart with saved distributions (UGKSBlock.initFunctions with a restart
   file that holds f, ugks_block.py:274-300, 347-349, then ugks_sim.py:85-92):
   f, macro and Q are the caller's (loaded into the block arrays beforehand;
   for *_mixed, f as its deviation from the reference Maxwellian);
   wall_prop from the wall values, the fused path's per-cell moments and next
   heat flux from f, ghosts filled, dt := CFL / max frequency of the loaded
   macro.  `time` and `steps` of each solve record are left as the caller set
   them.  (A restart without saved f is ugks_init_*: f := fEQ(macro, Q).) */
int ugks_restart_fp64(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                      ugks_solve_state *solves_dev, int nsolves, UGKS_STREAM);
int ugks_restart_mixed(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                       ugks_solve_state *solves_dev, int nsolves, UGKS_STREAM);

/* One UGKSim.one_step (ugks_sim.py:407-501) of every active solve: flux
   pass, dt check with the reference's single retry, cell update, new dt,
   time advance, ghost update. */
int ugks_step_fp64(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                   ugks_solve_state *solves_dev, int nsolves, UGKS_STREAM);
int ugks_step_mixed(const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                    ugks_solve_state *solves_dev, int nsolves, UGKS_STREAM);

/* The same step with cudaEventRecord of events[0..7] (cudaEvent_t) on the
   stream around the phases: [0] start, [1] after the face pass, [2] after the
   dt check, [3] after the retry face pass, [4] after the second dt check,
   [5] after the cell pass, [6] after the dt update, [7] after the ghost pass.
   mixed != 0 selects FP32 storage.  A null entry records nothing (each
   record costs the stream a few microseconds).  Used to time each kernel
   live. */
int ugks_step_profiled(int mixed, const ugks_fused_block *blocks_dev, int nblocks,
                       const ugks_fused_sizes *sizes, ugks_solve_state *solves_dev, int nsolves,
                       void *const *events, UGKS_STREAM);

/* Residual of the last step (getResidual + the host reduction of
   ugks_block.py:1303-1327, averaged over a solve's blocks as
   ugks_sim.py:463-468 does) into ugks_solve_state.residual. */
int ugks_residual(const ugks_fused_block *blocks_dev, int nblocks, ugks_solve_state *solves_dev,
                  int nsolves, UGKS_STREAM);

/* The stop rule of ugks_solve_state for every active solve, after
   ugks_residual of the same step: a solve with a non-zero status, a density
   residual below stop_residual after at least stop_after completed steps, or
   stop_steps completed steps gets stopped =
   UGKS_STOP_ERROR / _CONVERGED / _STEPS and active = 0, so that later fused
   launches skip it (the run loop's exits, ugks_sim.py:587-645, decided on the
   device). */
int ugks_stop_check(ugks_solve_state *solves_dev, int nsolves, UGKS_STREAM);

/* nsteps times: ugks_step_fp64 (mixed = 0) or ugks_step_mixed (mixed = 1),
   ugks_residual and ugks_stop_check -- a serving tick, with no host
   synchronisation, suitable for capture in one CUDA graph. */
int ugks_serve_steps(int mixed, const ugks_fused_block *blocks_dev, int nblocks, const ugks_fused_sizes *sizes,
                     ugks_solve_state *solves_dev, int nsolves, int nsteps, UGKS_STREAM);

/* Sets the kernel attributes the fused step needs (dynamic shared memory
   above 48 KB) on the current device; the first ugks_step_* call on a device
   does the same.  Call it before capturing steps in a CUDA graph. */
int ugks_prepare(int mixed);

/* The bounded wait the mixed face pass puts on its bulk copies
   (cp.async.bulk on an mbarrier), checked on its own: one warp expects 512
   bytes and copies them from src_dev (device, 16-byte aligned) or, with
   src_dev NULL, never does, then waits at most `polls` times (each at most
   about a microsecond).  *status_dev (device int) becomes 0 when the copy
   completed and matched, 8 (the solve status of a copy that outlived its
   bound) when the wait ran out, -1 on a mismatch. */
int ugks_check_copy_wait(const void *src_dev, unsigned polls, int *status_dev, UGKS_STREAM);

/* ------------------------------------------------------------------------
 * 3. Time-step frequency without device allocation.  No counterpart in the
 *    reference.  For callers that cannot allocate device memory (a host
 *    runtime that forbids cudaMalloc while it drives the solver, or one that
 *    runs from a fixed memory plan): the same maximum CFL frequency that
 *    ugks_clFindDT followed by ugks_array_max yields (the quantity
 *    UGKSBlock.getDT turns into max_dt = CFL / max_freq), with the per-cell
 *    frequencies kept in a static array inside the library instead of a
 *    caller buffer.  The caller passes the inputs and max_freq (one double,
 *    device memory) only.
 *
 *    - At most UGKS_NOALLOC_MAX_CELLS interior cells (ni * nj) per call;
 *      larger blocks return UGKS_ERR_TOO_LARGE without launching anything.
 *    - The array (8 MiB) is held on every GPU that loads the library until
 *      the process exits.
 *    - The first call on a device looks up the array's device address
 *      (cudaGetSymbolAddress) with that device current; make that first call
 *      before any stream capture.
 *    - All calls share the array and it keeps the last call's contents:
 *      calls that overlap on the GPU (different streams, no ordering) race.
 *    Returns 0, UGKS_ERR_TOO_LARGE, UGKS_ERR_BAD_SIZE or a negative cudaError_t.
 * --------------------------------------------------------------------- */
#define UGKS_NOALLOC_MAX_CELLS (1 << 20)
#define UGKS_ERR_TOO_LARGE (-10001)
#define UGKS_ERR_BAD_SIZE (-10002)
int ugks_getDT_noalloc(const ugks_block_desc *d, const double *xy, const double *area,
                       const double *macro, double Kn, double *max_freq, UGKS_STREAM);

/* Kernel launches one ugks_step_fp64 (mixed = 0) or ugks_step_mixed
   (mixed = 1) call makes for a block table of these sizes. */
int ugks_step_launches(const ugks_fused_sizes *sizes, int mixed);

/* Library identification: returns a static version string. */
const char *ugks_version(void);
/* sizeof(ugks_block_desc), sizeof(ugks_fused_block), sizeof(ugks_solve_state),
   offsetof(ugks_fused_block, f), offsetof(ugks_solve_state, residual),
   offsetof(ugks_block_desc, wall_D), sizeof(ugks_fused_sizes): the first n
   into out; returns 7.  Lets a
   binding check its struct layout against the library's. */
int ugks_abi_sizes(int64_t *out, int n);

#ifdef __cplusplus
}
#endif
#endif /* UGKS_B200_H */
