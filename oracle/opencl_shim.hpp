// opencl_shim.hpp -- TEST INFRASTRUCTURE ONLY (oracle), never linked into the product.
//
// Lets the reference's OpenCL C kernels (pyUGKS source/*.c) compile as host C++
// so that the reference itself can be run on the CPU as an oracle.  The kernels
// are executed with one work-item per work-group (LOCAL_SIZE = 1): every
// __local tree reduction in the reference (e.g. source/clUGKS.c:251-261)
// degenerates to a sequential sum over the velocity loop and every barrier()
// is trivially satisfied.
//
// Provides: the OpenCL vector types used by the reference (double2/4/8,
// int2/3/4) with the swizzles it uses (.x .y .z .w .s0-.s7 .s01 .s12 .s012),
// component-wise arithmetic with scalar broadcast, the OpenCL built-ins it
// calls (dot, length, normalize, sign, fabs, isnan, any, min, max), the
// address-space qualifiers and the work-item functions.
#pragma once
#include <math.h>
#include <stddef.h>
#include <stdint.h>

#define __kernel static
#define __global
#define __constant const
#define __local static thread_local
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
static inline void barrier(int) {}

// work-item ids of the work-group being executed by this host thread
static thread_local size_t ocl_gid[3];
static inline size_t get_global_id(int d) { return ocl_gid[d]; }
static inline size_t get_local_id(int) { return 0; }

#define OCL_VEC_OPS(T, S, N)                                                        \
  static inline T operator+(T a, T b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] + b.v[i]; return r; } \
  static inline T operator-(T a, T b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] - b.v[i]; return r; } \
  static inline T operator*(T a, T b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] * b.v[i]; return r; } \
  static inline T operator/(T a, T b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] / b.v[i]; return r; } \
  static inline T operator+(T a, S b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] + b; return r; }      \
  static inline T operator-(T a, S b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] - b; return r; }      \
  static inline T operator*(T a, S b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] * b; return r; }      \
  static inline T operator/(T a, S b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] / b; return r; }      \
  static inline T operator+(S a, T b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a + b.v[i]; return r; }      \
  static inline T operator-(S a, T b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a - b.v[i]; return r; }      \
  static inline T operator*(S a, T b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a * b.v[i]; return r; }      \
  static inline T operator/(S a, T b) { T r; for (int i = 0; i < N; ++i) r.v[i] = a / b.v[i]; return r; }      \
  static inline T operator-(T a) { T r; for (int i = 0; i < N; ++i) r.v[i] = -a.v[i]; return r; }              \
  static inline T& operator+=(T& a, T b) { a = a + b; return a; }                                             \
  static inline T& operator-=(T& a, T b) { a = a - b; return a; }                                             \
  static inline T& operator*=(T& a, T b) { a = a * b; return a; }                                             \
  static inline T& operator/=(T& a, T b) { a = a / b; return a; }                                             \
  static inline T& operator+=(T& a, S b) { a = a + b; return a; }                                             \
  static inline T& operator-=(T& a, S b) { a = a - b; return a; }                                             \
  static inline T& operator*=(T& a, S b) { a = a * b; return a; }                                             \
  static inline T& operator/=(T& a, S b) { a = a / b; return a; }

// Vector types: plain unions so that they stay trivially copyable (they are
// members of other unions and of __local arrays).  Scalar broadcast assignment
// (`v = 0.0;`) goes through operator=(scalar).
struct double2 {
  union {
    struct { double x, y; };
    struct { double s0, s1; };
    double v[2];
  };
  double2& operator=(double s) { x = s; y = s; return *this; }
};
struct double4 {
  union {
    struct { double x, y, z, w; };
    struct { double s0, s1, s2, s3; };
    struct { double2 s01, s23; };
    struct { double pad0_; double2 s12; double pad3_; };
    double v[4];
  };
  double4& operator=(double s) { for (int i = 0; i < 4; ++i) v[i] = s; return *this; }
};
struct double8 {
  union {
    struct { double s0, s1, s2, s3, s4, s5, s6, s7; };
    double v[8];
  };
  double8& operator=(double s) { for (int i = 0; i < 8; ++i) v[i] = s; return *this; }
};
struct int2 {
  union {
    struct { int x, y; };
    struct { int s0, s1; };
    int v[2];
  };
  int2& operator=(int s) { x = s; y = s; return *this; }
};
struct int3 {
  union {
    struct { int x, y, z; };
    struct { int s0, s1, s2; };
    int v[3];
  };
  int3& operator=(int s) { x = s; y = s; z = s; return *this; }
};
struct int4 {
  union {
    struct { int x, y, z, w; };
    struct { int s0, s1, s2, s3; };
    struct { int3 s012; int pad3_; };
    int v[4];
  };
  int4& operator=(int s) { for (int i = 0; i < 4; ++i) v[i] = s; return *this; }
};

OCL_VEC_OPS(double2, double, 2)
OCL_VEC_OPS(double4, double, 4)
OCL_VEC_OPS(double8, double, 8)

static inline double2 make_double2(double a, double b) { double2 r; r.x = a; r.y = b; return r; }
static inline double4 make_double4(double a, double b, double c, double d) {
  double4 r; r.x = a; r.y = b; r.z = c; r.w = d; return r;
}
static inline double8 make_double8(double a, double b, double c, double d, double e, double f,
                                   double g, double h) {
  double8 r; r.s0 = a; r.s1 = b; r.s2 = c; r.s3 = d; r.s4 = e; r.s5 = f; r.s6 = g; r.s7 = h; return r;
}
static inline int4 make_int4(int a, int b, int c, int d) {
  int4 r; r.x = a; r.y = b; r.z = c; r.w = d; return r;
}

// OpenCL built-ins used by the reference kernels
static inline double sign(double a) {
  if (a > 0.0) return 1.0;
  if (a < 0.0) return -1.0;
  if (a == 0.0) return a;  // keeps the sign of zero
  return 0.0;              // NaN
}
static inline double2 sign(double2 a) { return make_double2(sign(a.x), sign(a.y)); }
static inline double2 fabs(double2 a) { return make_double2(fabs(a.x), fabs(a.y)); }
static inline double dot(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }
static inline double length(double2 a) { return sqrt(a.x * a.x + a.y * a.y); }
static inline double2 normalize(double2 a) { return a / length(a); }
static inline int2 isnan(double2 a) {
  int2 r; r.x = isnan(a.x) ? -1 : 0; r.y = isnan(a.y) ? -1 : 0; return r;
}
static inline int any(int2 a) { return (a.x < 0) || (a.y < 0); }
static inline double min(double a, double b) { return fmin(a, b); }
static inline double max(double a, double b) { return fmax(a, b); }
