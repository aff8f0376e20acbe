/* ugks_port.h -- TEST INFRASTRUCTURE ONLY (oracle).
 *
 * Plain-C restatement of the pyUGKS OpenCL kernels on the time-step path,
 * executed sequentially on the CPU.  Each port_<name> function restates the
 * reference __kernel <name> (file:line given at each definition in
 * ugks_port.c) over the NDRange g0 x g1 with one work-item per work-group, and
 * takes the reference kernel's arguments in the reference order.  The
 * compile-time header of the reference (ugks_CL.py:20-400) becomes the runtime
 * struct below.
 *
 * Array layouts are the reference's (source/clKernel.c:4-26): a "double2"
 * array is interleaved pairs of doubles, "double4" is quadruples, etc.
 */
#ifndef UGKS_PORT_H
#define UGKS_PORT_H
#include <stddef.h>
#include <stdint.h>

typedef struct {
  int ni, nj, Ni, Nj, ghost, Nv;
  int flux_method;  /* 0 vanLeer, 1 WENO5, 3 minmod (NND) */
  int relax_type;
  double PI, Pr, umax, vmax, Kn_eff, gam, B, K, omega;
  const double *quad;        /* [Nv][2] */
  const double *weight;      /* [Nv]    */
  const int64_t *mirror_NS, *mirror_EW, *mirror_D;
  /* WALL_<f>_{D,U,V,T,P} values per face N,E,S,W (T holds the lambda macro) */
  double wall_D[4], wall_U[4], wall_V[4], wall_T[4], wall_P[4];
  /* adsorbing-wall tables (ugks_CL.py:102-185) */
  double beta_n[4], beta_t[4], gamma_f[4], alpha_p[4];
  int dynamic[4];
  int constant_adsorb[4];
  double adsorb[4];
  /* first-order desorption rate per face; 0 selects the reference's
     Langmuir-driven desorption (clAdsorb.c:436-438) */
  double k_des[4];
  /* Cercignani-Lampis accommodation (ALPHA_N, ALPHA_T, ugks_CL.py:134-148) */
  double alpha_n[4], alpha_t[4];
  /* tabulated isotherms (ISO_, TRI_, NBR_<face>, N_TRI; ugks_CL.py:158-252):
     points (P, T, theta, 0), Delaunay triangles and their neighbours */
  const double *iso[4];
  const int32_t *tri[4], *nbr[4];
  int n_tri[4];
} ugks_port_params;

#endif
