// common.cuh -- device-side configuration, grid indexing and the forward
// tangent (dual number) scalar used by the Newton kernels.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/grim_b200.h"

#define GRIM_HD __host__ __device__ __forceinline__
#define GRIM_D __device__ __forceinline__

namespace grim {

enum { RHO = 0, UU = 1, U1 = 2, U2 = 3, U3 = 4 };

// Everything a kernel needs from grim_config, in one by-value argument.
struct DevCfg {
  int N1, N2, N3, dim, ng;
  int g1, g2, g3;
  int N1T, N2T, N3T;
  // rows of faces the interior needs (its own faces and the corner EMFs one
  // row beyond it): j in [fj0, fj0 + nfj), k in [fk0, fk0 + nfk)
  int fj0, nfj, fk0, nfk;
  long long Z, Zint;
  long long GZ;  // zones of one (i, j) plane: the stride of the stored geometry
  int nf, dof, Q, DP, B1;
  int conduction, viscosity, hoCond, hoVisc;
  int metric, reconstruction, riemann, closure, problem;
  int maxIter, maxLS;
  int bc[6];  // left, right, bottom, top, back, front
  double dX[3], invdX[3];
  double X1Start, X2Start, X3Start, X2End;
  double Gam;
  double rhoFloor, uFloor, bSqrFloor, TFloor;
  double CondAlpha, ViscAlpha, CondClosure, ViscClosure;
  double theta;
  double atol, rtol, jacEps, lsFloor;
  double tolUlps;  // rounding floor of the Newton test in ulps of the residual's largest term (0: none)
  double tau0, tau1;
  // torus floors (problem hook)
  double maxLF, rhoFloorAmpl, uFloorAmpl, rhoFloorSlope, uFloorSlope, bsqOverRhoMax, bsqOverUMax;
  // debug setting (grim_set_debug): the TMA-staged face kernels issue no
  // copies, so their bounded waits run out
  int dbgSkipCopies;
};

GRIM_HD long long zidx(const DevCfg& c, int i, int j, int k) {
  return (long long)i + (long long)c.N1T * ((long long)j + (long long)c.N2T * k);
}
// Index decompositions in 32-bit unsigned arithmetic (grids are limited to
// fewer than 2^31 zones at creation): a fraction of the instructions of
// 64-bit division.
GRIM_HD void zijk(const DevCfg& c, long long z, int& i, int& j, int& k) {
  const unsigned zz = (unsigned)z, n1 = (unsigned)c.N1T, n2 = (unsigned)c.N2T;
  const unsigned r = zz / n1;
  i = (int)(zz - r * n1);
  const unsigned q = r / n2;
  j = (int)(r - q * n2);
  k = (int)q;
}
// n-th interior zone -> full-grid index
GRIM_HD long long interior_to_z(const DevCfg& c, long long n) {
  const unsigned nn = (unsigned)n, n1 = (unsigned)c.N1, n2 = (unsigned)c.N2;
  const unsigned r = nn / n1;
  const unsigned q = r / n2;
  return zidx(c, (int)(nn - r * n1) + c.g1, (int)(r - q * n2) + c.g2, (int)q + c.g3);
}
// The metrics (Minkowski, modified Kerr-Schild with derefine / cylindrify)
// do not depend on X3, so the geometry is stored for one (i, j) plane.
GRIM_HD long long gidx(const DevCfg& c, int i, int j) { return (long long)i + (long long)c.N1T * j; }
GRIM_HD long long gidx(const DevCfg& c, long long z) { return z % c.GZ; }
GRIM_HD long long stride_of(const DevCfg& c, int dir) {
  return dir == 0 ? 1LL : (dir == 1 ? (long long)c.N1T : (long long)c.N1T * c.N2T);
}

// ---------------------------------------------------------------------------
// Forward tangent scalar: value + N directional derivatives.  Arithmetic with
// plain doubles treats them as constants.  Used to get all Jacobian columns
// of the zone residual in one pass (the product's replacement for the
// reference's nf+1 residual finite-difference assembly, solve.cpp:82-109).
// ---------------------------------------------------------------------------
template <class T, int N>
struct Dual {
  T v;
  T d[N];
  GRIM_HD Dual() {}
  GRIM_HD Dual(T x) : v(x) {
#pragma unroll
    for (int k = 0; k < N; k++) d[k] = T(0);
  }
  GRIM_HD static Dual var(T x, int dir) {
    Dual r(x);
    r.d[dir] = T(1);
    return r;
  }
};

template <class T, int N>
GRIM_HD Dual<T, N> operator+(const Dual<T, N>& a, const Dual<T, N>& b) {
  Dual<T, N> r; r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <class T, int N>
GRIM_HD Dual<T, N> operator-(const Dual<T, N>& a, const Dual<T, N>& b) {
  Dual<T, N> r; r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <class T, int N>
GRIM_HD Dual<T, N> operator-(const Dual<T, N>& a) {
  Dual<T, N> r; r.v = -a.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = -a.d[k];
  return r;
}
template <class T, int N>
GRIM_HD Dual<T, N> operator*(const Dual<T, N>& a, const Dual<T, N>& b) {
  Dual<T, N> r; r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <class T, int N>
GRIM_HD Dual<T, N> operator/(const Dual<T, N>& a, const Dual<T, N>& b) {
  Dual<T, N> r; r.v = a.v / b.v;
  T ib = T(1) / b.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
// mixed with constants (type T)
template <class T, int N>
GRIM_HD Dual<T, N> operator+(const Dual<T, N>& a, T b) { Dual<T, N> r = a; r.v = a.v + b; return r; }
template <class T, int N>
GRIM_HD Dual<T, N> operator+(T b, const Dual<T, N>& a) { Dual<T, N> r = a; r.v = b + a.v; return r; }
template <class T, int N>
GRIM_HD Dual<T, N> operator-(const Dual<T, N>& a, T b) { Dual<T, N> r = a; r.v = a.v - b; return r; }
template <class T, int N>
GRIM_HD Dual<T, N> operator-(T b, const Dual<T, N>& a) {
  Dual<T, N> r; r.v = b - a.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = -a.d[k];
  return r;
}
template <class T, int N>
GRIM_HD Dual<T, N> operator*(const Dual<T, N>& a, T b) {
  Dual<T, N> r; r.v = a.v * b;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * b;
  return r;
}
template <class T, int N>
GRIM_HD Dual<T, N> operator*(T b, const Dual<T, N>& a) {
  Dual<T, N> r; r.v = b * a.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = b * a.d[k];
  return r;
}
template <class T, int N>
GRIM_HD Dual<T, N> operator/(const Dual<T, N>& a, T b) {
  Dual<T, N> r; r.v = a.v / b;
  T ib = T(1) / b;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * ib;
  return r;
}
template <class T, int N>
GRIM_HD Dual<T, N> operator/(T a, const Dual<T, N>& b) {
  Dual<T, N> r; r.v = a / b.v;
  T ib = T(1) / b.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = -r.v * b.d[k] * ib;
  return r;
}
template <class T, int N>
GRIM_HD Dual<T, N>& operator+=(Dual<T, N>& a, const Dual<T, N>& b) { a = a + b; return a; }
template <class T, int N>
GRIM_HD Dual<T, N>& operator-=(Dual<T, N>& a, const Dual<T, N>& b) { a = a - b; return a; }
template <class T, int N>
GRIM_HD Dual<T, N>& operator*=(Dual<T, N>& a, const Dual<T, N>& b) { a = a * b; return a; }

// scalar helpers usable for double, float and Dual
GRIM_HD double val(double x) { return x; }
GRIM_HD float val(float x) { return x; }
template <class T, int N>
GRIM_HD T val(const Dual<T, N>& x) { return x.v; }

// the value of a scalar: a double, or the value part of a tangent scalar
GRIM_HD double val_of(double x) { return x; }
template <class T, int N>
GRIM_HD T val_of(const Dual<T, N>& x) { return x.v; }

GRIM_HD double dsqrt(double x) { return sqrt(x); }
GRIM_HD float dsqrt(float x) { return sqrtf(x); }
// 1 / sqrt(x) (the fast path forms gamma and 1 / gamma from one call)
GRIM_HD double drsqrt(double x) { return rsqrt(x); }
GRIM_HD float drsqrt(float x) { return rsqrtf(x); }
template <class T, int N>
GRIM_HD Dual<T, N> drsqrt(const Dual<T, N>& a) {
  Dual<T, N> r; r.v = drsqrt(a.v);
  const T h = T(-0.5) * r.v * r.v * r.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * h;
  return r;
}
template <class T, int N>
GRIM_HD Dual<T, N> dsqrt(const Dual<T, N>& a) {
  Dual<T, N> r; r.v = dsqrt(a.v);
  T h = T(0.5) / r.v;
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * h;
  return r;
}
// max(a, const): the reference's af::max(x, floor) -- derivative follows
// the selected branch
GRIM_HD double dmaxc(double a, double b) { return fmax(a, b); }
GRIM_HD float dmaxc(float a, float b) { return fmaxf(a, b); }
template <class T, int N>
GRIM_HD Dual<T, N> dmaxc(const Dual<T, N>& a, T b) {
  if (a.v >= b) return a;
  return Dual<T, N>(b);
}

// Conversion of a double constant into the scalar type S.
template <class S> struct Lift;
template <> struct Lift<double> { GRIM_HD static double of(double x) { return x; } };
template <> struct Lift<float> { GRIM_HD static float of(double x) { return (float)x; } };
template <class T, int N> struct Lift<Dual<T, N>> {
  GRIM_HD static Dual<T, N> of(double x) { return Dual<T, N>((T)x); }
};
// base real type of S
template <class S> struct Real { typedef S type; };
template <class T, int N> struct Real<Dual<T, N>> { typedef T type; };

}  // namespace grim
