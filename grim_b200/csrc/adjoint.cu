// adjoint.cu -- reverse (adjoint) sweep of whole implicit timesteps.
//
// The forward step (timestep.cpp:3-334) is, per stage with dt' = dt/2 then
// dt, the implicit system R(P) = (U(P; B) - U(P0)) / dt' + divF(Ps) +
// S(Ps) = 0 for the fluid unknowns (S: the geometric source, zero in
// Minkowski), with the field advanced explicitly, sqrt(-g) B = sqrt(-g) B0
// - dt' divF_B(Ps), and Ps = P0 (half stage) or Ph (full stage).  Given
// lambda = dL/dP1 at the end of a step, the adjoint of the step is
// (implicit-function theorem, so the Newton iterations are not
// differentiated; they are converged):
//
//   full stage at P1:  mu = (dU/dPf / dt)^-T lambda_f
//                      beta = lambda_B - (dU/dB / dt)^T mu
//                      g_h = [-mu ; -dt / sqrt(-g) beta]   (= dL/d divF(Ph))
//   lambda_h = D(Ph)^T g_h + dS/dP(Ph)^T g_h,fluid   (stencil VJP, ghosts folded)
//   half stage at Ph:  mu_h, beta_h likewise with dt/2, g_0 = [-mu_h ; -dt/2 / sqrt(-g) beta_h]
//   lambda_0 = D(P0)^T g_0 + dS/dP(P0)^T g_0,fluid
//              + dU(P0)/dP^T (mu/dt + mu_h/(dt/2)) + [0 ; beta + beta_h]
//
// D^T is the transpose of the stencil: divergence (fvmfluxes.cpp:36-45),
// flux-CT / EMF (constrainedtransport.cpp:3-83), Riemann solver
// (riemannsolver.cpp:202-328) with the face metric, reconstruction, and the
// ghost fill (boundary.cpp:5-241 and grid::communicate: every ghost zone
// copies the interior zone that the periodic / outflow / mirror map of each
// direction selects, so its adjoint goes back to that zone); the Riemann
// solver, the reconstruction, the conserved variables and the geometric
// source (physics.cpp:360-420) through local Jacobians taken with the
// forward-tangent scalar on the same templated physics the kernels run.
// Scope: ideal or extended MHD (conduction and / or viscosity: the EMHD
// residual's tangents, its source's gradient gathers), Minkowski or
// modified Kerr-Schild, 2D or 3D, periodic / outflow / mirror boundaries,
// without problem hooks or with the torus problem's (floors, inflow check,
// pole fix, flux filter), dt held fixed over the run; the runtime rejects
// anything else.  Every accumulation is a gather in a fixed order (no
// atomics), so a gradient is the same bits run to run.
#include <cuda_runtime.h>

#include "launch.h"
#include "physics.cuh"
#include "recon.cuh"

namespace grim {

// ---- the forward-tangent scalar in the reconstruction's expressions:
// comparisons on values, min / max / |.| / copysign on the selected branch
template <class T, int N>
GRIM_D bool operator<(const Dual<T, N>& a, const Dual<T, N>& b) { return a.v < b.v; }
template <class T, int N>
GRIM_D bool operator>(const Dual<T, N>& a, const Dual<T, N>& b) { return a.v > b.v; }
template <class T, int N>
GRIM_D bool operator<=(const Dual<T, N>& a, const Dual<T, N>& b) { return a.v <= b.v; }
template <class T, int N>
GRIM_D bool operator>=(const Dual<T, N>& a, const Dual<T, N>& b) { return a.v >= b.v; }
template <class T, int N>
GRIM_D bool operator<(const Dual<T, N>& a, T b) { return a.v < b; }
template <class T, int N>
GRIM_D bool operator>(const Dual<T, N>& a, T b) { return a.v > b; }
template <class T, int N>
GRIM_D bool operator<=(const Dual<T, N>& a, T b) { return a.v <= b; }
template <class T, int N>
GRIM_D bool operator>=(const Dual<T, N>& a, T b) { return a.v >= b; }
template <class T, int N>
GRIM_D Dual<T, N> fabs(const Dual<T, N>& a) { return a.v < T(0) ? -a : a; }
// IEEE fmin / fmax: a NaN argument yields the other one, as on doubles
// (the reconstruction's limiters then discard a NaN neighbour, and so does
// its derivative)
template <class T, int N>
GRIM_D Dual<T, N> fmin(const Dual<T, N>& a, const Dual<T, N>& b) {
  if (isnan(a.v)) return b;
  if (isnan(b.v)) return a;
  return (b.v < a.v) ? b : a;
}
template <class T, int N>
GRIM_D Dual<T, N> fmax(const Dual<T, N>& a, const Dual<T, N>& b) {
  if (isnan(a.v)) return b;
  if (isnan(b.v)) return a;
  return (b.v > a.v) ? b : a;
}
template <class T, int N>
GRIM_D Dual<T, N> copysign(T a, const Dual<T, N>& b) { return Dual<T, N>(::copysign(a, b.v)); }

// minmod of three slopes (minmod.cpp:3-19) on the tangent scalar: where the
// smallest magnitude is exactly zero (a flat stretch of data, a zero field)
// the limited slope stays zero on at least one side of the point, and the
// sign choices at an exact zero would give a derivative of no side; the
// derivative taken there is zero
template <class T, int N>
GRIM_D Dual<T, N> minmod3(Dual<T, N> x, Dual<T, N> y, Dual<T, N> z) {
  typedef Dual<T, N> D;
  D m = fmin(fmin(fabs(x), fabs(y)), fabs(z));
  if (m.v == T(0)) return D(T(0));
  const T sx = x.v < T(0) ? T(-1) : T(1), sy = y.v < T(0) ? T(-1) : T(1), sz = z.v < T(0) ? T(-1) : T(1);
  return m * (T(0.25) * ::fabs(sx + sy) * (sx + sz));
}

// the overloads on plain doubles stay visible beside the ones above
using ::fabs;
using ::fmax;
using ::fmin;

}  // namespace grim

// the torus problem's floors, on the tangent scalar (their local Jacobian)
#define GRIM_KNS adjt
#include "torus.cuh"
#undef GRIM_KNS

namespace grim {

namespace adj {

static inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// Gaussian elimination with partial pivoting (first largest pivot)
GRIM_D void solve5(double A[5][5], double b[5], double x[5]) {
  for (int kk = 0; kk < 5; kk++) {
    int p = kk;
    double best = ::fabs(A[kk][kk]);
    for (int r = kk + 1; r < 5; r++)
      if (::fabs(A[r][kk]) > best) { best = ::fabs(A[r][kk]); p = r; }
    if (p != kk) {
      for (int cc = 0; cc < 5; cc++) { const double t = A[kk][cc]; A[kk][cc] = A[p][cc]; A[p][cc] = t; }
      const double t = b[kk]; b[kk] = b[p]; b[p] = t;
    }
    for (int r = kk + 1; r < 5; r++) {
      const double f = A[r][kk] / A[kk][kk];
      for (int cc = kk; cc < 5; cc++) A[r][cc] -= f * A[kk][cc];
      b[r] -= f * b[kk];
    }
  }
  for (int r = 4; r >= 0; r--) {
    double s = b[r];
    for (int cc = r + 1; cc < 5; cc++) s -= A[r][cc] * x[cc];
    x[r] = s / A[r][r];
  }
}

// the zone's geometry as constants of the tangent scalar
template <class D>
GRIM_D void geo_const(ZoneGeo<D>& Gd, const ZoneGeo<double>& G) {
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) { Gd.gcov[m][n] = D(G.gcov[m][n]); Gd.gcon[m][n] = D(G.gcon[m][n]); }
  Gd.g = D(G.g); Gd.alpha = D(G.alpha); Gd.ialpha = D(G.ialpha);
  Gd.x1 = D(G.x1); Gd.x2 = D(G.x2); Gd.dyn = D(G.dyn);
}

// the element of one zone's primitives p in grid row order (fluid rows,
// then B1..B3)
template <int C, int V, class S>
GRIM_D void elem_rows(ElemT<S, S>& e, const DevCfg& c, const S* p, const ZoneGeo<S>& G) {
  constexpr int NF = 5 + C + V;
  elem_set<C, V>(e, p[0], p[1], p[2], p[3], p[4], p[NF], p[NF + 1], p[NF + 2], C ? p[5] : S(0.),
                 V ? p[5 + C] : S(0.), G, c);
}

// the centre geometry of zone z
GRIM_D void centre_geo(const DevCfg& c, const double* geoC, long long z, ZoneGeo<double>& G) {
  int i, j, k;
  zijk(c, z, i, j, k);
  load_geo(G, c, geoC, z, i, j, 0.5, 0.5);
}

// conserved fluid rows U (nf = 5) of one zone and their Jacobian with
// respect to the 8 primitives (5 fluid, then B)
GRIM_D void cons_jacobian(const DevCfg& c, const double* p, long long z, const ZoneGeo<double>& G0,
                          double J[5][8]) {
  typedef Dual<double, 8> D;
  const long long Z = c.Z;
  D q[8];
  for (int v = 0; v < 5; v++) q[v] = D::var(p[(long long)v * Z + z], v);
  for (int v = 0; v < 3; v++) q[5 + v] = D::var(p[(long long)(c.B1 + v) * Z + z], 5 + v);
  ZoneGeo<D> G;
  geo_const(G, G0);
  ElemT<D, D> e;
  elem_set<0, 0>(e, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], D(0.), D(0.), G, c);
  D U[5];
  fluxes_fluid<0, 0>(e, 0, G.g, U, 5, 5);
  for (int r = 0; r < 5; r++)
    for (int k = 0; k < 8; k++) J[r][k] = U[r].d[k];
}

// Stage adjoint at the stage's solution P (interior zones): lam -> g (dL/d
// divF, dof rows), ubar (+)= mu / dt', bacc (+)= beta
__global__ void k_stage(DevCfg c, const double* __restrict__ geoC, const double* __restrict__ P, double dtp,
                        const double* __restrict__ lam, double* __restrict__ g, double* __restrict__ ubar,
                        double* __restrict__ bacc, int accumulate) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  const long long Z = c.Z;
  const long long z = interior_to_z(c, n);
  // a zone whose adjoint is zero contributes nothing; its state may be one
  // the NaN reset discards, where the Jacobian is not finite
  bool any = false;
  for (int v = 0; v < c.dof; v++) any |= lam[(long long)v * Z + z] != 0.;
  if (!any) {
    for (int v = 0; v < c.dof; v++) g[(long long)v * Z + z] = 0.;
    if (!accumulate) {
      for (int v = 0; v < 5; v++) ubar[(long long)v * Z + z] = 0.;
      for (int k = 0; k < 3; k++) bacc[(long long)k * Z + z] = 0.;
    }
    return;
  }
  ZoneGeo<double> G;
  centre_geo(c, geoC, z, G);
  double J[5][8];
  cons_jacobian(c, P, z, G, J);
  // (J_ff / dt')^T mu = lam_f
  double AT[5][5], b[5], mu[5];
  for (int r = 0; r < 5; r++) {
    b[r] = lam[(long long)r * Z + z];
    for (int k = 0; k < 5; k++) AT[r][k] = J[k][r] / dtp;
  }
  solve5(AT, b, mu);
  for (int v = 0; v < 5; v++) {
    g[(long long)v * Z + z] = -mu[v];
    const double u = mu[v] / dtp;
    ubar[(long long)v * Z + z] = accumulate ? ubar[(long long)v * Z + z] + u : u;
  }
  for (int k = 0; k < 3; k++) {
    double beta = lam[(long long)(c.B1 + k) * Z + z];
    for (int r = 0; r < 5; r++) beta -= J[r][5 + k] / dtp * mu[r];
    g[(long long)(c.B1 + k) * Z + z] = -dtp / G.g * beta;
    bacc[(long long)k * Z + z] = accumulate ? bacc[(long long)k * Z + z] + beta : beta;
  }
}

// out(P0) += dU/dP(P0)^T ubar + [0 ; bacc] (interior zones)
__global__ void k_cons(DevCfg c, const double* __restrict__ geoC, const double* __restrict__ P,
                       const double* __restrict__ ubar, const double* __restrict__ bacc, double* __restrict__ lam) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  const long long Z = c.Z;
  const long long z = interior_to_z(c, n);
  bool any = false;
  for (int r = 0; r < 5; r++) any |= ubar[(long long)r * Z + z] != 0.;
  for (int k = 0; k < 3; k++) any |= bacc[(long long)k * Z + z] != 0.;
  if (!any) return;
  ZoneGeo<double> G;
  centre_geo(c, geoC, z, G);
  double J[5][8];
  cons_jacobian(c, P, z, G, J);
  for (int k = 0; k < 8; k++) {
    double s = 0.;
    for (int r = 0; r < 5; r++)
      if (ubar[(long long)r * Z + z] != 0.) s += J[r][k] * ubar[(long long)r * Z + z];
    if (k >= 5) s += bacc[(long long)(k - 5) * Z + z];
    const long long row = (k < 5) ? k : c.B1 + (k - 5);
    lam[row * Z + z] += s;
  }
}

// The geometric source's transpose (interior zones): out += dS/dP(Ps)^T g
// over the fluid rows, S^nu = -sqrt(-g) T^ka_la Gamma^la_(ka nu) of the
// stage element at the centre (physics.cpp:360-420)
template <int C, int V>
__global__ void k_src_t(DevCfg c, const double* __restrict__ geoC, const double* __restrict__ gamma,
                        const double* __restrict__ P, const double* __restrict__ g, double* __restrict__ out) {
  constexpr int DOF = 8 + C + V;
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  typedef Dual<double, DOF> D;
  const long long Z = c.Z;
  const long long z = interior_to_z(c, n);
  int i, j, k;
  zijk(c, z, i, j, k);
  ZoneGeo<double> G0;
  load_geo(G0, c, geoC, z, i, j, 0.5, 0.5);
  ZoneGeo<D> G;
  geo_const(G, G0);
  D q[DOF];
  for (int v = 0; v < DOF; v++) q[v] = D::var(P[(long long)v * Z + z], v);
  ElemT<D, D> e;
  elem_rows<C, V>(e, c, q, G);
  D T[4][4];
  for (int ka = 0; ka < 4; ka++)
    for (int la = 0; la < 4; la++) T[ka][la] = tmunu<C, V>(e, ka, la);
  const double* gam = gamma + gidx(c, i, j);
  double acc[DOF];
  for (int m = 0; m < DOF; m++) acc[m] = 0.;
  for (int nu = 0; nu < 4; nu++) {
    const double gb = g[(long long)(UU + nu) * Z + z];
    if (gb == 0.) continue;
    D s(0.);
    for (int ka = 0; ka < 4; ka++)
      for (int la = 0; la < 4; la++) s -= T[ka][la] * (G0.g * __ldg(gam + (long long)(la * 16 + ka * 4 + nu) * c.GZ));
    for (int m = 0; m < DOF; m++) acc[m] += s.d[m] * gb;
  }
  for (int m = 0; m < DOF; m++) out[(long long)m * Z + z] += acc[m];
}

GRIM_D bool is_interior(const DevCfg& c, int i, int j, int k) {
  return i >= c.g1 && i < c.N1 + c.g1 && j >= c.g2 && j < c.N2 + c.g2 &&
         (c.dim < 3 || (k >= c.g3 && k < c.N3 + c.g3));
}

// divergence transpose: Ft[d][v][f] = (g[v][f - s_d] - g[v][f]) / dX_d,
// g zero off the interior (the zero-padded convolution of fvmfluxes.cpp in
// 2D, the shifted difference in 3D: the same linear map)
__global__ void k_div_t(DevCfg c, const double* __restrict__ g, double* __restrict__ Ft) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  const long long Z = c.Z;
  for (int d = 0; d < c.dim; d++) {
    const int im = d == 0 ? i - 1 : i, jm = d == 1 ? j - 1 : j, km = d == 2 ? k - 1 : k;
    const bool in0 = is_interior(c, i, j, k), in1 = is_interior(c, im, jm, km);
    const long long zm = zidx(c, im < 0 ? 0 : im, jm < 0 ? 0 : jm, km < 0 ? 0 : km);
    const double idx = 1. / c.dX[d];
    // the torus flux filter zeroes every row of the faces at the poles
    // (problem.cpp:1243-1285): only the zone beside each pole face uses it
    const bool pole = c.problem == GRIM_PROBLEM_TORUS && d == 1 && (j == c.g2 || j == c.N2 + c.g2);
    for (int v = 0; v < c.dof; v++) {
      const double a = in1 ? g[(long long)v * Z + zm] : 0.;
      const double b = in0 ? g[(long long)v * Z + z] : 0.;
      Ft[((long long)d * c.dof + v) * Z + z] = pole ? 0. : (a - b) * idx;
    }
  }
}

// flux-CT transpose, step 1: the edge EMF adjoints from the CT fluxes'
// adjoints.  The CT fluxes of the field rows (constrainedtransport.cpp:3-51)
// are F1_B2 = (e3 + e3[+s2]) / 2, F2_B1 = -(e3 + e3[+s1]) / 2 and, in 3D,
// F1_B3 = -(e2 + e2[+s3]) / 2, F3_B1 = (e2 + e2[+s1]) / 2,
// F2_B3 = (e1 + e1[+s3]) / 2, F3_B2 = -(e1 + e1[+s2]) / 2.
// ebar rows: e3, e1, e2.
GRIM_D const double* ft_row(const DevCfg& c, const double* Ft, int d, int b) {
  return Ft + ((long long)d * c.dof + c.B1 + b) * c.Z;
}
__global__ void k_ct_t_emf(DevCfg c, const double* __restrict__ Ft, double* __restrict__ ebar) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  const long long Z = c.Z, s1 = 1, s2 = c.N1T, s3 = (long long)c.N1T * c.N2T;
  const double* F1B2 = ft_row(c, Ft, 0, 1);
  const double* F2B1 = ft_row(c, Ft, 1, 0);
  double e = 0.5 * F1B2[z] - 0.5 * F2B1[z];
  if (j >= 1) e += 0.5 * F1B2[z - s2];
  if (i >= 1) e -= 0.5 * F2B1[z - s1];
  ebar[z] = e;
  if (c.dim < 3) return;
  const double* F2B3 = ft_row(c, Ft, 1, 2);
  const double* F3B2 = ft_row(c, Ft, 2, 1);
  const double* F1B3 = ft_row(c, Ft, 0, 2);
  const double* F3B1 = ft_row(c, Ft, 2, 0);
  double e1 = 0.5 * F2B3[z] - 0.5 * F3B2[z];
  if (k >= 1) e1 += 0.5 * F2B3[z - s3];
  if (j >= 1) e1 -= 0.5 * F3B2[z - s2];
  double e2 = 0.5 * F3B1[z] - 0.5 * F1B3[z];
  if (i >= 1) e2 += 0.5 * F3B1[z - s1];
  if (k >= 1) e2 -= 0.5 * F1B3[z - s3];
  ebar[Z + z] = e1;
  ebar[2 * Z + z] = e2;
}

// flux-CT transpose, step 2: the raw Riemann fluxes' adjoints of the B
// rows from the edge EMFs e3 = (R1_B2 + R1_B2[-s2] - R2_B1 - R2_B1[-s1]) / 4,
// e1 = (R2_B3 + R2_B3[-s3] - R3_B2 - R3_B2[-s2]) / 4,
// e2 = (R3_B1 + R3_B1[-s1] - R1_B3 - R1_B3[-s3]) / 4 (constrainedtransport.cpp:
// 53-83); a direction's own field row never reaches the divergence; in 2D
// the B3 rows are the raw fluxes and keep their adjoints
__global__ void k_ct_t_raw(DevCfg c, const double* __restrict__ ebar, double* __restrict__ Ft) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  const long long Z = c.Z, s1 = 1, s2 = c.N1T, s3 = (long long)c.N1T * c.N2T;
  auto row = [&](int d, int b) -> double& { return Ft[((long long)d * c.dof + c.B1 + b) * Z + z]; };
  const double ez = ebar[z];
  const double ej = (j + 1 < c.N2T) ? ebar[z + s2] : 0.;
  const double ei = (i + 1 < c.N1T) ? ebar[z + s1] : 0.;
  row(0, 0) = 0.;
  row(0, 1) = 0.25 * ez + 0.25 * ej;
  row(1, 0) = -0.25 * ez - 0.25 * ei;
  row(1, 1) = 0.;
  if (c.dim < 3) return;
  const double* e1 = ebar + Z;
  const double* e2 = ebar + 2 * Z;
  const bool kp = k + 1 < c.N3T, jp = j + 1 < c.N2T, ip = i + 1 < c.N1T;
  row(0, 2) = -0.25 * e2[z] - 0.25 * (kp ? e2[z + s3] : 0.);
  row(1, 2) = 0.25 * e1[z] + 0.25 * (kp ? e1[z + s3] : 0.);
  row(2, 0) = 0.25 * e2[z] + 0.25 * (ip ? e2[z + s1] : 0.);
  row(2, 1) = -0.25 * e1[z] - 0.25 * (jp ? e1[z + s2] : 0.);
  row(2, 2) = 0.;
}

// the Riemann flux of one face (riemannsolver.cpp:202-328) on any scalar
template <int C, int V, class S>
GRIM_D void riemann_flux(const DevCfg& c, int dir, const ZoneGeo<double>& G0, const S* pl, const S* pr, S* F) {
  constexpr int NF = 5 + C + V, DOF = NF + 3;
  ZoneGeo<S> G;
  geo_const(G, G0);
  const int fd = dir + 1;
  S FL[DOF], UL[DOF], FR[DOF], UR[DOF], mnL, mxL, mnR, mxR;
  {
    ElemT<S, S> e;
    elem_rows<C, V>(e, c, pl, G);
    fluxes_fluid<C, V>(e, fd, G.g, FL, 5, 5 + C);
    fluxes_B(e, fd, G.g, FL + NF);
    fluxes_fluid<C, V>(e, 0, G.g, UL, 5, 5 + C);
    fluxes_B(e, 0, G.g, UL + NF);
    char_speeds<C, V>(e, G, dir, c, mnL, mxL);
  }
  {
    ElemT<S, S> e;
    elem_rows<C, V>(e, c, pr, G);
    fluxes_fluid<C, V>(e, fd, G.g, FR, 5, 5 + C);
    fluxes_B(e, fd, G.g, FR + NF);
    fluxes_fluid<C, V>(e, 0, G.g, UR, 5, 5 + C);
    fluxes_B(e, 0, G.g, UR + NF);
    char_speeds<C, V>(e, G, dir, c, mnR, mxR);
  }
  const S cmin = dmin2(mnL, mnR), cmax = dmax2(mxL, mxR);
  if (c.riemann == GRIM_HLL) {
    for (int v = 0; v < DOF; v++) F[v] = (cmax * FL[v] - cmin * FR[v] + cmin * cmax * (UR[v] - UL[v])) / (cmax - cmin);
  } else {
    const S cm = dmax2(cmax, -cmin);
    for (int v = 0; v < DOF; v++) F[v] = S(0.5) * (FL[v] + FR[v] - cm * (UR[v] - UL[v]));
  }
}

// Riemann transpose of the faces along dir: the face between zones
// a = z - s and b = z takes Fbar (dof) and forms the adjoints of its two
// reconstructed states, gl = (dF/dpl)^T Fbar (pl: the right-face state of a)
// and gr = (dF/dpr)^T Fbar (pr: the left-face state of b), into gface
// (rows 0..dof-1 gl, dof..2 dof-1 gr; zero on the faces the stencil does
// not use)
template <int C, int V>
__global__ void k_faces_t(DevCfg c, int dir, const double* __restrict__ geoF, const double* __restrict__ P,
                          const double* __restrict__ Ft, double* __restrict__ gface) {
  constexpr int DOF = 8 + C + V;
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  const int x = dir == 0 ? i : (dir == 1 ? j : k);
  const int NT = dir == 0 ? c.N1T : (dir == 1 ? c.N2T : c.N3T);
  const long long Z = c.Z, s = stride_of(c, dir);
  double fb[DOF];
  bool any = false;
  for (int v = 0; v < DOF; v++) {
    fb[v] = (x < 3 || x > NT - 3) ? 0. : Ft[((long long)dir * c.dof + v) * Z + z];
    any |= fb[v] != 0.;
  }
  if (!any) {
    for (int v = 0; v < 2 * DOF; v++) gface[(long long)v * Z + z] = 0.;
    return;
  }
  // the face states
  double pl[DOF], pr[DOF];
  for (int v = 0; v < DOF; v++) {
    const double* a = P + (long long)v * Z;
    double lo, ro, lo2, ro2;
    recon_faces<double>(c.reconstruction, c.theta, a[z - 3 * s], a[z - 2 * s], a[z - s], a[z], a[z + s], lo, ro);
    recon_faces<double>(c.reconstruction, c.theta, a[z - 2 * s], a[z - s], a[z], a[z + s], a[z + 2 * s], lo2, ro2);
    pl[v] = ro;
    pr[v] = lo2;
  }
  // the face metric (the X3 faces of the axisymmetric metrics: the centre's)
  ZoneGeo<double> G;
  load_geo(G, c, geoF, z, i, j, dir == 0 ? 0. : 0.5, dir == 1 ? 0. : 0.5);
  // dF/dpl and dF/dpr, dof tangent lanes each
  typedef Dual<double, DOF> D8;
  for (int side = 0; side < 2; side++) {
    D8 L[DOF], R[DOF], F[DOF];
    for (int v = 0; v < DOF; v++) {
      L[v] = side == 0 ? D8::var(pl[v], v) : D8(pl[v]);
      R[v] = side == 1 ? D8::var(pr[v], v) : D8(pr[v]);
    }
    riemann_flux<C, V, D8>(c, dir, G, L, R, F);
    // the torus flux filter on the density flux of the inner / outer X1
    // faces: min(F, 0) / max(F, 0), so its derivative is 1 or 0
    double fr0 = fb[0];
    if (c.problem == GRIM_PROBLEM_TORUS && dir == 0 &&
        ((x == c.g1 && F[0].v > 0.) || (x == c.N1 + c.g1 && F[0].v < 0.)))
      fr0 = 0.;
    for (int k2 = 0; k2 < DOF; k2++) {
      double acc = fr0 * F[0].d[k2];
      for (int r = 1; r < DOF; r++)
        if (fb[r] != 0.) acc += fb[r] * F[r].d[k2];
      gface[(long long)(side * DOF + k2) * Z + z] = acc;
    }
  }
}

// Reconstruction transpose along dir, as a gather: zone x collects, in a
// fixed order, the adjoints of the face states of the five zones whose
// stencils hold it (y = x - 2 .. x + 2 along dir): the right-face state of y
// (the left state of face y + 1, adjoint gl there) and its left-face state
// (the right state of face y, adjoint gr), each times its derivative with
// respect to x from a forward-tangent pass of y's reconstruction.  One
// thread per zone and direction, so the sums are the same run to run.
__global__ void k_recon_t(DevCfg c, int dir, const double* __restrict__ P, const double* __restrict__ gface,
                          double* __restrict__ q) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  const int x = dir == 0 ? i : (dir == 1 ? j : k);
  const int NT = dir == 0 ? c.N1T : (dir == 1 ? c.N2T : c.N3T);
  const long long Z = c.Z, s = stride_of(c, dir);
  typedef Dual<double, 5> D5;
  for (int v = 0; v < c.dof; v++) {
    const double* a = P + (long long)v * Z;
    double acc = 0.;
    for (int m = 4; m >= 0; m--) {
      // x is point m of the stencil of y = x + 2 - m
      const int y = x + 2 - m;
      if (y < 2 || y > NT - 3) continue;
      const long long zy = z + (long long)(2 - m) * s;
      const double gl = (y + 1 <= NT - 1) ? gface[(long long)v * Z + zy + s] : 0.;
      const double gr = gface[(long long)(c.dof + v) * Z + zy];
      if (gl == 0. && gr == 0.) continue;
      D5 yb[5];
      for (int mm = 0; mm < 5; mm++) yb[mm] = D5::var(a[zy + (mm - 2) * s], mm);
      D5 lo, ro;
      recon_faces<D5>(c.reconstruction, c.theta, yb[0], yb[1], yb[2], yb[3], yb[4], lo, ro);
      acc += gl * ro.d[m] + gr * lo.d[m];
    }
    q[(long long)v * Z + z] += acc;
  }
}

// The ghost fill's transpose: every ghost zone copies the interior zone
// that each direction's map selects (periodic: the wrapped image; outflow:
// the first / last interior zone; mirror: the reflected zone), so every
// interior zone gathers the adjoints of itself and of the ghost zones that
// copy it: per direction the positions y with map(y) = x, in a fixed order.
GRIM_D int preimages(int x, int g, int N, int NT, int lo, int hi, int* ys) {
  int n = 0;
  ys[n++] = x;
  if (NT == 1) return n;
  // a direction with a periodic side wraps both (grid::communicate's
  // periodic DMDA; the boundary fill then leaves that direction alone)
  const bool per = lo == GRIM_PERIODIC || hi == GRIM_PERIODIC;
  // the lower ghosts y < g
  if (per) {
    if (x - N >= 0 && x - N < g) ys[n++] = x - N;
  } else if (lo == GRIM_MIRROR) {
    if (x < 2 * g) ys[n++] = 2 * g - 1 - x;
  } else if (x == g) {
    for (int y = 0; y < g; y++) ys[n++] = y;
  }
  // the upper ghosts y >= N + g
  if (per) {
    if (x + N >= N + g && x + N < NT) ys[n++] = x + N;
  } else if (hi == GRIM_MIRROR) {
    if (x >= N) ys[n++] = 2 * (N + g) - 1 - x;
  } else if (x == N + g - 1) {
    for (int y = N + g; y < NT; y++) ys[n++] = y;
  }
  return n;
}

__global__ void k_fold(DevCfg c, const double* __restrict__ q, double* __restrict__ out) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  const long long Z = c.Z;
  const long long z = interior_to_z(c, n);
  int i, j, k;
  zijk(c, z, i, j, k);
  int ys1[8], ys2[8], ys3[8];
  const int n1 = preimages(i, c.g1, c.N1, c.N1T, c.bc[0], c.bc[1], ys1);
  const int n2 = c.dim >= 2 ? preimages(j, c.g2, c.N2, c.N2T, c.bc[2], c.bc[3], ys2) : (ys2[0] = j, 1);
  const int n3 = c.dim >= 3 ? preimages(k, c.g3, c.N3, c.N3T, c.bc[4], c.bc[5], ys3) : (ys3[0] = k, 1);
  for (int v = 0; v < c.dof; v++) {
    double s = 0.;
    for (int a = 0; a < n1; a++)
      for (int b = 0; b < n2; b++)
        for (int m = 0; m < n3; m++) s += q[(long long)v * Z + zidx(c, ys1[a], ys2[b], ys3[m])];
    out[(long long)v * Z + z] = s;
  }
}


// ---- extended MHD (conduction, viscosity) -----------------------------------
// The EMHD stage residual of one zone (residual.cpp with the stage
// constants of timestep.cpp: elemOld from P0, the reference element from
// Ps, elemOld itself on the half stage) on the tangent scalar, for the
// three seeds the adjoint needs: the unknowns and the new field, P0, Ps.
// divF and Sexp are the stage's values (their rows enter additively, times
// the row normalisation of q and deltaP).  normQ / normDP are returned for
// those rows' dR / d divF.
template <int C, int V, class D>
GRIM_D void emhd_residual(const DevCfg& c, int stage, double dtp, const D* Pf, const D* Bn, const D* p0,
                          const D* ps, const double* divF, const double* Sexp, const ZoneGeo<D>& G, D* R, D& normQ,
                          D& normDP) {
  constexpr int NF = 5 + C + V, Q = 5, DP = 5 + C;
  ElemT<D, D> eo, er;
  elem_rows<C, V>(eo, c, p0, G);
  if (stage == GRIM_HALF_STEP) er = eo;
  else elem_rows<C, V>(er, c, ps, G);
  D Uold[NF];
  fluxes_fluid<C, V>(eo, 0, G.g, Uold, 5, 5 + C);
  ElemT<D, D> e;
  elem_set<C, V>(e, Pf[0], Pf[1], Pf[2], Pf[3], Pf[4], Bn[0], Bn[1], Bn[2], C ? Pf[Q] : D(0.), V ? Pf[DP] : D(0.),
                 G, c);
  D U[NF];
  fluxes_fluid<C, V>(e, 0, G.g, U, 5, 5 + C);
  for (int v = 0; v < NF; v++) R[v] = (U[v] - Uold[v]) / dtp + divF[v] + Sexp[v];
  D dtuCov[4];
  for (int mu = 0; mu < 4; mu++) dtuCov[mu] = (e.uCov[mu] - eo.uCov[mu]) / dtp;
  D div(0.);
  for (int mu = 0; mu < 4; mu++) div += G.gcon[0][mu] * dtuCov[mu];
  const D rr = er.rho, rtau = er.tau, rT = er.temperature;
  normQ = D(1.);
  normDP = D(1.);
  if (V) {
    const D rnu = er.nu;
    D d0 = -div * rr * rnu;
    for (int mu = 0; mu < 4; mu++) d0 += 3. * rr * rnu * er.bCon[0] * er.bCon[mu] / er.bSqr * dtuCov[mu];
    if (c.hoVisc == 1) d0 = d0 * dsqrt(rtau / rr / rnu / rT);
    D sdt = -G.g * d0 / rtau;
    if (c.hoVisc == 1) sdt = sdt - 0.5 * G.g * div * er.deltaPTilde;
    const D simp = G.g * Pf[DP] / rtau;
    const D sOld = G.g * eo.deltaPTilde / rtau;
    normDP = c.hoVisc ? dsqrt(rr * rnu * rT * rtau) : rtau;
    R[DP] = (R[DP] + 0.5 * (sOld + simp) + sdt) * normDP;
  }
  if (C) {
    const D rchi = er.chi;
    D qq = -rr * rchi * er.bCon[0] / er.bNorm * (e.temperature - eo.temperature) / dtp;
    for (int nu = 0; nu < 4; nu++) qq -= rr * rchi * rT * er.bCon[nu] / er.bNorm * er.uCon[0] * dtuCov[nu];
    if (c.hoCond == 1) qq = qq * (dsqrt(rtau / rr / rchi) / rT);
    D sdt = -G.g * qq / rtau;
    if (c.hoCond == 1) sdt = sdt - 0.5 * G.g * div * er.qTilde;
    const D simp = G.g * Pf[Q] / rtau;
    const D sOld = G.g * eo.qTilde / rtau;
    normQ = c.hoCond ? rT * dsqrt(rr * rchi * rtau) : rtau;
    R[Q] = (R[Q] + 0.5 * (sOld + simp) + sdt) * normQ;
  }
}

// Gaussian elimination with partial pivoting, n x n
template <int N>
GRIM_D void solveN(double A[N][N], double b[N], double x[N]) {
  for (int kk = 0; kk < N; kk++) {
    int p = kk;
    double best = ::fabs(A[kk][kk]);
    for (int r = kk + 1; r < N; r++)
      if (::fabs(A[r][kk]) > best) { best = ::fabs(A[r][kk]); p = r; }
    if (p != kk) {
      for (int cc = 0; cc < N; cc++) { const double t = A[kk][cc]; A[kk][cc] = A[p][cc]; A[p][cc] = t; }
      const double t = b[kk]; b[kk] = b[p]; b[p] = t;
    }
    for (int r = kk + 1; r < N; r++) {
      const double f = A[r][kk] / A[kk][kk];
      for (int cc = kk; cc < N; cc++) A[r][cc] -= f * A[kk][cc];
      b[r] -= f * b[kk];
    }
  }
  for (int r = N - 1; r >= 0; r--) {
    double s = b[r];
    for (int cc = r + 1; cc < N; cc++) s -= A[r][cc] * x[cc];
    x[r] = s / A[r][r];
  }
}

// EMHD stage adjoint at the stage's solution P (interior zones): lam ->
// g (dL/d divF = dL/d Sexp, dof rows), p0bar (+)= dL/dP0 through the stage
// constants and the induction, psl = dL/dPs through the reference element
// (full stage; zero on the half stage, whose reference element is elemOld)
template <int C, int V>
__global__ void k_stage_emhd(DevCfg c, const double* __restrict__ geoC, int stage, double dtp,
                             const double* __restrict__ P, const double* __restrict__ P0,
                             const double* __restrict__ Ps, const double* __restrict__ divF,
                             const double* __restrict__ Sexp, const double* __restrict__ lam, double* __restrict__ g,
                             double* __restrict__ p0bar, double* __restrict__ psl) {
  constexpr int NF = 5 + C + V, DOF = NF + 3, Q = 5, DP = 5 + C;
  typedef Dual<double, DOF> D;
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  const long long Z = c.Z;
  const long long z = interior_to_z(c, n);
  double lv[DOF];
  bool any = false;
  for (int v = 0; v < DOF; v++) {
    lv[v] = lam[(long long)v * Z + z];
    any |= lv[v] != 0.;
  }
  if (!any) {
    for (int v = 0; v < DOF; v++) { g[(long long)v * Z + z] = 0.; psl[(long long)v * Z + z] = 0.; }
    return;
  }
  ZoneGeo<double> G0;
  centre_geo(c, geoC, z, G0);
  ZoneGeo<D> G;
  geo_const(G, G0);
  double pv[DOF], p0v[DOF], psv[DOF], dF[NF], sE[NF];
  for (int v = 0; v < DOF; v++) {
    pv[v] = P[(long long)v * Z + z];
    p0v[v] = P0[(long long)v * Z + z];
    psv[v] = Ps[(long long)v * Z + z];
  }
  for (int v = 0; v < NF; v++) { dF[v] = divF[(long long)v * Z + z]; sE[v] = Sexp[(long long)v * Z + z]; }
  D Pf[NF], Bn[3], a0[DOF], as[DOF], R[NF], nQ, nDP;
  // seed 1: the unknowns and the new field
  for (int v = 0; v < NF; v++) Pf[v] = D::var(pv[v], v);
  for (int k = 0; k < 3; k++) Bn[k] = D::var(pv[NF + k], NF + k);
  for (int v = 0; v < DOF; v++) { a0[v] = D(p0v[v]); as[v] = D(psv[v]); }
  emhd_residual<C, V, D>(c, stage, dtp, Pf, Bn, a0, as, dF, sE, G, R, nQ, nDP);
  double AT[NF][NF], b[NF], mu[NF];
  for (int r = 0; r < NF; r++) {
    b[r] = lv[r];
    for (int k = 0; k < NF; k++) AT[r][k] = R[k].d[r];
  }
  solveN<NF>(AT, b, mu);
  double beta[3];
  for (int k = 0; k < 3; k++) {
    beta[k] = lv[NF + k];
    for (int r = 0; r < NF; r++) beta[k] -= R[r].d[NF + k] * mu[r];
  }
  for (int v = 0; v < NF; v++) {
    const double sc = (C && v == Q) ? nQ.v : ((V && v == DP) ? nDP.v : 1.);
    g[(long long)v * Z + z] = -mu[v] * sc;
  }
  for (int k = 0; k < 3; k++) g[(long long)(NF + k) * Z + z] = -dtp / G0.g * beta[k];
  // seed 2: P0 (elemOld, the old conserved variables, and on the half
  // stage the reference element); the induction adds beta to B0
  for (int v = 0; v < NF; v++) Pf[v] = D(pv[v]);
  for (int k = 0; k < 3; k++) Bn[k] = D(pv[NF + k]);
  for (int v = 0; v < DOF; v++) a0[v] = D::var(p0v[v], v);
  emhd_residual<C, V, D>(c, stage, dtp, Pf, Bn, a0, as, dF, sE, G, R, nQ, nDP);
  for (int v = 0; v < DOF; v++) {
    double s = (v >= NF) ? beta[v - NF] : 0.;
    for (int r = 0; r < NF; r++) s -= R[r].d[v] * mu[r];
    p0bar[(long long)v * Z + z] += s;
  }
  // seed 3: Ps (the full stage's reference element)
  if (stage == GRIM_HALF_STEP) {
    for (int v = 0; v < DOF; v++) psl[(long long)v * Z + z] = 0.;
    return;
  }
  for (int v = 0; v < DOF; v++) { a0[v] = D(p0v[v]); as[v] = D::var(psv[v], v); }
  emhd_residual<C, V, D>(c, stage, dtp, Pf, Bn, a0, as, dF, sE, G, R, nQ, nDP);
  for (int v = 0; v < DOF; v++) {
    double s = 0.;
    for (int r = 0; r < NF; r++) s -= R[r].d[v] * mu[r];
    psl[(long long)v * Z + z] = s;
  }
}

// The EMHD explicit source of one zone (computeEMHDGradients and the
// sources of physics.cpp:502-586): the q and deltaP rows from the stage
// element e and the limited slopes sl[d][m] of u_mu (m < 4) and T (m = 4)
template <int C, int V, class S>
GRIM_D void emhd_source(const DevCfg& c, const ElemT<S, S>& e, const ZoneGeo<S>& G, const double* gam, S sl[3][5],
                        S& SQ, S& SDP) {
  S gu[4][4], gT[4];
  for (int mu = 0; mu < 4; mu++) {
    gu[0][mu] = S(0.);
    gu[1][mu] = sl[0][mu];
    gu[2][mu] = (c.dim > 1) ? sl[1][mu] : S(0.);
    gu[3][mu] = (c.dim > 2) ? sl[2][mu] : S(0.);
    if (gam)
      for (int nu = 0; nu < 4; nu++)
        for (int la = 0; la < 4; la++) gu[nu][mu] -= __ldg(gam + (long long)(la * 16 + nu * 4 + mu) * c.GZ) * e.uCov[la];
  }
  gT[0] = S(0.);
  gT[1] = sl[0][4];
  gT[2] = (c.dim > 1) ? sl[1][4] : S(0.);
  gT[3] = (c.dim > 2) ? sl[2][4] : S(0.);
  S dv(0.);
  for (int mu = 0; mu < 4; mu++)
    for (int nu = 0; nu < 4; nu++) dv += G.gcon[mu][nu] * gu[mu][nu];
  SQ = S(0.);
  SDP = S(0.);
  if (V) {
    S d0 = -dv * e.rho * e.nu;
    for (int mu = 0; mu < 4; mu++)
      for (int nu = 0; nu < 4; nu++) d0 += 3. * e.rho * e.nu * e.bCon[mu] * e.bCon[nu] / e.bSqr * gu[mu][nu];
    const S d0t = (c.hoVisc == 1) ? d0 * dsqrt(e.tau / e.rho / e.nu / e.temperature) : d0;
    S s = -G.g * d0t / e.tau;
    if (c.hoVisc == 1) s = s - 0.5 * G.g * dv * e.deltaPTilde;
    SDP = s;
  }
  if (C) {
    S qq(0.);
    for (int mu = 0; mu < 4; mu++) {
      qq -= e.rho * e.chi * e.bCon[mu] / e.bNorm * gT[mu];
      for (int nu = 0; nu < 4; nu++) qq -= e.rho * e.chi * e.temperature * e.bCon[nu] / e.bNorm * e.uCon[mu] * gu[mu][nu];
    }
    const S qt = (c.hoCond == 1) ? qq * dsqrt(e.tau / e.rho / e.chi) / e.temperature : qq;
    S s = -G.g * qt / e.tau;
    if (c.hoCond == 1) s = s - 0.5 * G.g * dv * e.qTilde;
    SQ = s;
  }
}

// the limited slope of u_mu / T along d at zone z (the forward's st())
GRIM_D double uT_slope(const DevCfg& c, const double* uT, long long z, int d, int m) {
  const long long sd = stride_of(c, d);
  const double* a = uT + (long long)m * c.Z + z;
  return recon_slope(c.reconstruction, c.theta, a[-2 * sd], a[-sd], a[0], a[sd], a[2 * sd], c.dX[d]);
}

// The EMHD source's transpose, step 1 (interior zones): its dependence on
// the zone's own stage element into out, and the adjoints of the slopes it
// reads (sbar, dim x 5 per zone)
template <int C, int V>
__global__ void k_emhd_src_t(DevCfg c, const double* __restrict__ geoC, const double* __restrict__ gamma,
                             const double* __restrict__ Ps, const double* __restrict__ uT,
                             const double* __restrict__ g, double* __restrict__ out, double* __restrict__ sbar) {
  constexpr int DOF = 8 + C + V, Q = 5, DP = 5 + C;
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  const long long Z = c.Z;
  const long long z = interior_to_z(c, n);
  const double gQ = C ? g[(long long)Q * Z + z] : 0., gD = V ? g[(long long)DP * Z + z] : 0.;
  if (gQ == 0. && gD == 0.) {
    for (int m = 0; m < 15; m++) sbar[(long long)m * Z + z] = 0.;
    return;
  }
  int i, j, k;
  zijk(c, z, i, j, k);
  ZoneGeo<double> G0;
  load_geo(G0, c, geoC, z, i, j, 0.5, 0.5);
  const double* gam = gamma ? gamma + gidx(c, i, j) : nullptr;
  double slv[3][5];
  for (int d = 0; d < 3; d++)
    for (int m = 0; m < 5; m++) slv[d][m] = d < c.dim ? uT_slope(c, uT, z, d, m) : 0.;
  {
    // the zone's element, slopes fixed
    typedef Dual<double, DOF> D;
    ZoneGeo<D> G;
    geo_const(G, G0);
    D q[DOF], sl[3][5], SQ, SD;
    for (int v = 0; v < DOF; v++) q[v] = D::var(Ps[(long long)v * Z + z], v);
    for (int d = 0; d < 3; d++)
      for (int m = 0; m < 5; m++) sl[d][m] = D(slv[d][m]);
    ElemT<D, D> e;
    elem_rows<C, V>(e, c, q, G);
    emhd_source<C, V, D>(c, e, G, gam, sl, SQ, SD);
    for (int v = 0; v < DOF; v++) out[(long long)v * Z + z] += SQ.d[v] * gQ + SD.d[v] * gD;
  }
  {
    // the slopes, element fixed
    typedef Dual<double, 15> D;
    ZoneGeo<D> G;
    geo_const(G, G0);
    D q[DOF], sl[3][5], SQ, SD;
    for (int v = 0; v < DOF; v++) q[v] = D(Ps[(long long)v * Z + z]);
    for (int d = 0; d < 3; d++)
      for (int m = 0; m < 5; m++) sl[d][m] = D::var(slv[d][m], d * 5 + m);
    ElemT<D, D> e;
    elem_rows<C, V>(e, c, q, G);
    emhd_source<C, V, D>(c, e, G, gam, sl, SQ, SD);
    for (int m = 0; m < 15; m++) sbar[(long long)m * Z + z] = SQ.d[m] * gQ + SD.d[m] * gD;
  }
}

// step 2 (every zone): the adjoint of its u_mu, T from the slopes of the
// interior zones whose 5-point stencils hold it, gathered in a fixed order
__global__ void k_emhd_slope_t(DevCfg c, const double* __restrict__ uT, const double* __restrict__ sbar,
                               double* __restrict__ uTbar) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  typedef Dual<double, 5> D5;
  double acc[5] = {0., 0., 0., 0., 0.};
  for (int d = 0; d < c.dim; d++) {
    const long long sd = stride_of(c, d);
    const int x = d == 0 ? i : (d == 1 ? j : k);
    const int g0 = d == 0 ? c.g1 : (d == 1 ? c.g2 : c.g3);
    const int N = d == 0 ? c.N1 : (d == 1 ? c.N2 : c.N3);
    for (int p = 0; p < 5; p++) {
      // this zone is point p of the stencil of zone y = x + 2 - p
      const int y = x + 2 - p;
      if (y < g0 || y >= g0 + N) continue;
      const long long zy = z + (long long)(2 - p) * sd;
      int iy, jy, ky;
      zijk(c, zy, iy, jy, ky);
      const bool inside = iy >= c.g1 && iy < c.N1 + c.g1 && (c.dim < 2 || (jy >= c.g2 && jy < c.N2 + c.g2)) &&
                          (c.dim < 3 || (ky >= c.g3 && ky < c.N3 + c.g3));
      if (!inside) continue;
      for (int m = 0; m < 5; m++) {
        const double sb = sbar[(long long)(d * 5 + m) * c.Z + zy];
        if (sb == 0.) continue;
        const double* a = uT + (long long)m * c.Z + zy;
        D5 yb[5];
        for (int mm = 0; mm < 5; mm++) yb[mm] = D5::var(a[(mm - 2) * sd], mm);
        const D5 sl = recon_slope<D5>(c.reconstruction, c.theta, yb[0], yb[1], yb[2], yb[3], yb[4], c.dX[d]);
        acc[m] += sb * sl.d[p];
      }
    }
  }
  for (int m = 0; m < 5; m++) uTbar[(long long)m * c.Z + z] = acc[m];
}

// step 3 (every zone): u_mu, T of the zone's element back to its primitives
template <int C, int V>
__global__ void k_emhd_uT_t(DevCfg c, const double* __restrict__ geoC, const double* __restrict__ Ps,
                            const double* __restrict__ uTbar, double* __restrict__ out) {
  constexpr int DOF = 8 + C + V;
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  const long long Z = c.Z;
  double ub[5];
  bool any = false;
  for (int m = 0; m < 5; m++) { ub[m] = uTbar[(long long)m * Z + z]; any |= ub[m] != 0.; }
  if (!any) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  ZoneGeo<double> G0;
  load_geo(G0, c, geoC, z, i, j, 0.5, 0.5);
  typedef Dual<double, DOF> D;
  ZoneGeo<D> G;
  geo_const(G, G0);
  D q[DOF];
  for (int v = 0; v < DOF; v++) q[v] = D::var(Ps[(long long)v * Z + z], v);
  ElemT<D, D> e;
  elem_rows<C, V>(e, c, q, G);
  for (int v = 0; v < DOF; v++) {
    double s = 0.;
    for (int m = 0; m < 4; m++) s += e.uCov[m].d[v] * ub[m];
    s += e.temperature.d[v] * ub[4];
    out[(long long)v * Z + z] += s;
  }
}

// out[interior] += a[interior] (dof rows)
__global__ void k_add_interior(DevCfg c, const double* __restrict__ a, double* __restrict__ out) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  const long long z = interior_to_z(c, n);
  for (int v = 0; v < c.dof; v++) out[(long long)v * c.Z + z] += a[(long long)v * c.Z + z];
}

// ---- the torus problem's hooks (problem.cpp): floors after each stage,
// the inflow check and the pole fix at the start of each stage
GRIM_D adjt::TorusCfg torus_params(const DevCfg& c) {
  adjt::TorusCfg t;
  t.MaxLorentzFactor = c.maxLF; t.RhoFloorAmpl = c.rhoFloorAmpl; t.UFloorAmpl = c.uFloorAmpl;
  t.RhoFloorSlope = c.rhoFloorSlope; t.UFloorSlope = c.uFloorSlope;
  t.BsqrOverRhoMax = c.bsqOverRhoMax; t.BsqrOverUMax = c.bsqOverUMax;
  return t;
}
// applyFloor's transpose (problem.cpp:542-712), interior zones: lam holds
// dL/d(floored state); lam <- J^T lam with J the floors' Jacobian at the
// stage's Newton solution Psol (one forward-tangent pass, one lane per
// primitive: the fluid rows, then the field)
template <int C, int V>
__global__ void k_floor_t(DevCfg c, const double* __restrict__ geoC, const double* __restrict__ Psol,
                          double* __restrict__ lam) {
  constexpr int NF = 5 + C + V, DOF = NF + 3;
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  typedef Dual<double, DOF> D;
  auto prow = [&](int v) -> long long { return v; };  // [fluid | field] rows, B1 = NF
  const long long Z = c.Z;
  const long long z = interior_to_z(c, n);
  int i, j, k;
  zijk(c, z, i, j, k);
  ZoneGeo<double> G0;
  load_geo(G0, c, geoC, z, i, j, 0.5, 0.5);
  ZoneGeo<D> G;
  geo_const(G, G0);
  // zero adjoint: nothing to transpose (the local Jacobian need not be
  // finite where no derivative flows, e.g. at a zero field)
  bool any = false;
  for (int v = 0; v < DOF; v++) any |= lam[prow(v) * Z + z] != 0.;
  if (!any) return;
  D q[DOF];
  bool nan = false;
  for (int v = 0; v < DOF; v++) {
    q[v] = D::var(Psol[prow(v) * Z + z], v);
    nan |= isnan(q[v].v);
  }
  if (nan) {
    // fullStepDiagnostics' reset: the zone's state no longer depends on it
    for (int v = 0; v < DOF; v++) lam[prow(v) * Z + z] = 0.;
    return;
  }
  const long long gz = gidx(c, i, j);
  adjt::torus_floor_zone<C, V>(c, torus_params(c), q, G, __ldg(geoC + 37LL * c.GZ + gz),
                               __ldg(geoC + 38LL * c.GZ + gz), false);
  double out[DOF];
  for (int v = 0; v < DOF; v++) out[v] = 0.;
  for (int r = 0; r < DOF; r++) {
    const double lr = lam[prow(r) * Z + z];
    if (lr != 0.)
      for (int v = 0; v < DOF; v++) out[v] += q[r].d[v] * lr;
  }
  for (int v = 0; v < DOF; v++) lam[prow(v) * Z + z] = out[v];
}

// fixPoles' transpose (problem.cpp:1046-1215) on the full-grid adjoint a,
// one thread per (i, k) column and pole: the two rows next to the pole take
// row idx2's fluid values (u2 scaled by theta_row / theta_idx2), the ghost
// rows mirror the three rows (fluid from row idx2, field from their own
// row, u2 and B2 negated); every overwritten entry's adjoint goes back to
// the entry it copies and is cleared
__global__ void k_poles_t(DevCfg c, const double* __restrict__ geoC, double* __restrict__ a) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long cols = (long long)c.N1T * c.N3T;
  if (n >= 2 * cols) return;
  const bool top = n >= cols;
  const long long m = top ? n - cols : n;
  const int i = (int)(m % c.N1T), k = (int)(m / c.N1T);
  const long long Z = c.Z;
  const int ng = c.ng;
  auto at = [&](int v, int j) -> double& { return a[(long long)v * Z + zidx(c, i, j, k)]; };
  auto theta = [&](int j) -> double {
    const double th = __ldg(geoC + 35LL * c.GZ + gidx(c, i, j));
    return top ? th * (-1.) + M_PI : th;
  };
  const int idx0 = top ? c.N2 + ng - 1 : ng;
  const int row[3] = {idx0, top ? idx0 - 1 : ng + 1, top ? idx0 - 2 : ng + 2};
  double th[3];
  for (int g = 0; g < 3; g++) th[g] = theta(row[g]);
  // the fluid rows (with EMHD q and deltaP, which fixPoles scales and
  // mirrors as it does u2)
  const int nf = c.nf;
  auto scaled = [&](int v) { return v == U2 || (c.conduction && v == c.Q) || (c.viscosity && v == c.DP); };
  double acc[7];
  for (int v = 0; v < nf; v++) acc[v] = at(v, row[2]);
  // only nonzero adjoints are carried: the ratio of thetas is not finite
  // in the innermost ghost column of some grids, where the forward's values
  // are not finite either and nothing downstream reads them
  for (int g = 0; g < 2; g++)
    for (int v = 0; v < nf; v++) {
      const double cf = scaled(v) ? th[g] / th[2] : 1.;
      if (at(v, row[g]) != 0.) acc[v] += cf * at(v, row[g]);
      at(v, row[g]) = 0.;
    }
  for (int g = 0; g < 3; g++) {
    const int dst = top ? c.N2 + ng + g : ng - 1 - g;
    for (int v = 0; v < nf; v++) {
      const double cf = scaled(v) ? -(g < 2 ? th[g] / th[2] : 1.) : 1.;
      if (at(v, dst) != 0.) acc[v] += cf * at(v, dst);
      at(v, dst) = 0.;
    }
    for (int b = 0; b < 3; b++) {
      const double cf = (b == 1) ? -1. : 1.;
      at(c.B1 + b, row[g]) += cf * at(c.B1 + b, dst);
      at(c.B1 + b, dst) = 0.;
    }
  }
  for (int v = 0; v < nf; v++) at(v, row[2]) = acc[v];
}

// inflowCheck's transpose (problem.cpp:941-1044) on the X1 ghost zones of
// the full-grid adjoint a: the ghost's velocities after the check are a
// function of its velocities before it (Pfill, the boundary fill's copy):
// u / gamma, the radial component clamped against inflow, the Lorentz
// factor capped; a's velocity rows <- J^T a
__global__ void k_inflow_t(DevCfg c, const double* __restrict__ geoC, const double* __restrict__ Pfill,
                           double* __restrict__ a) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long cols = (long long)2 * c.ng * c.N2T * c.N3T;
  if (n >= cols) return;
  typedef Dual<double, 3> D;
  const int gi = (int)(n % (2 * c.ng));
  const long long r = n / (2 * c.ng);
  const int j = (int)(r % c.N2T), k = (int)(r / c.N2T);
  const bool right = gi >= c.ng;
  const int i = right ? (c.N1 + c.ng + (gi - c.ng)) : gi;
  const long long Z = c.Z;
  const long long z = zidx(c, i, j, k);
  if (a[(long long)U1 * Z + z] == 0. && a[(long long)U2 * Z + z] == 0. && a[(long long)U3 * Z + z] == 0.) return;
  ZoneGeo<double> G0;
  geo_load<double>(G0, geoC, c.GZ, gidx(c, i, j));
  ZoneGeo<D> G;
  geo_const(G, G0);
  D u[3];
  for (int d = 0; d < 3; d++) u[d] = D::var(Pfill[(long long)(U1 + d) * Z + z], d);
  ElemT<D, D> e;
  elem_set<0, 0>(e, D(Pfill[z]), D(Pfill[Z + z]), u[0], u[1], u[2], D(Pfill[(long long)c.B1 * Z + z]),
                 D(Pfill[(long long)(c.B1 + 1) * Z + z]), D(Pfill[(long long)(c.B1 + 2) * Z + z]), D(0.), D(0.), G,
                 c);
  for (int d = 0; d < 3; d++) u[d] = u[d] / e.gam;
  if (right) {
    const long long ze = gidx(c, c.N1 + c.ng - 1, j);
    const double minUr = __ldg(geoC + 17LL * c.GZ + ze) * __ldg(geoC + 33LL * c.GZ + ze);
    u[0] = fmax(D(minUr), u[0]);
  } else {
    u[0] = fmin(D(G0.gcon[0][1] * G0.alpha), u[0]);
  }
  D vSqr(0.);
  for (int p = 0; p < 3; p++)
    for (int q = 0; q < 3; q++) vSqr += G0.gcov[p + 1][q + 1] * u[p] * u[q];
  const double vSqrMax = 1. - 1. / c.maxLF / c.maxLF;
  vSqr = fmax(fmin(vSqr, D(vSqrMax)), D(1.e-13));
  const D lf = 1. / dsqrt(1. - vSqr);
  double ab[3], out[3] = {0., 0., 0.};
  for (int d = 0; d < 3; d++) ab[d] = a[(long long)(U1 + d) * Z + z];
  for (int d = 0; d < 3; d++) {
    const D ud = u[d] * lf;
    for (int m2 = 0; m2 < 3; m2++) out[m2] += ud.d[m2] * ab[d];
  }
  for (int d = 0; d < 3; d++) a[(long long)(U1 + d) * Z + z] = out[d];
}

}  // namespace adj

static __global__ void k_zero_ghosts(DevCfg c, double* __restrict__ a) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  if (adj::is_interior(c, i, j, k)) return;
  for (int v = 0; v < c.dof; v++) a[(long long)v * c.Z + z] = 0.;
}

// ---- host side: one step's adjoint (all buffers dof x Z unless noted)
void adjoint_zero_ghosts(const DevCfg& c, double* a, cudaStream_t s) {
  k_zero_ghosts<<<adj::nblk(c.Z, 256), 256, 0, s>>>(c, a);
}

// q = the stencil's transpose over the whole grid (ghost entries not yet
// folded): divergence, flux-CT, Riemann solver, reconstruction
static void stencil_q(const DevCfg& c, const AdjointGeo& geo, const double* P, const double* g, double* Ft,
                      double* ebar, double* q, double* gface, cudaStream_t s) {
  using namespace adj;
  const size_t bZ = (size_t)c.Z * sizeof(double);
  k_div_t<<<nblk(c.Z, 128), 128, 0, s>>>(c, g, Ft);
  k_ct_t_emf<<<nblk(c.Z, 256), 256, 0, s>>>(c, Ft, ebar);
  k_ct_t_raw<<<nblk(c.Z, 256), 256, 0, s>>>(c, ebar, Ft);
  cudaMemsetAsync(q, 0, (size_t)c.dof * bZ, s);
  for (int d = 0; d < c.dim; d++) {
    if (c.conduction && c.viscosity) k_faces_t<1, 1><<<nblk(c.Z, 32), 32, 0, s>>>(c, d, geo.geoF[d], P, Ft, gface);
    else if (c.conduction) k_faces_t<1, 0><<<nblk(c.Z, 32), 32, 0, s>>>(c, d, geo.geoF[d], P, Ft, gface);
    else if (c.viscosity) k_faces_t<0, 1><<<nblk(c.Z, 32), 32, 0, s>>>(c, d, geo.geoF[d], P, Ft, gface);
    else k_faces_t<0, 0><<<nblk(c.Z, 64), 64, 0, s>>>(c, d, geo.geoF[d], P, Ft, gface);
    k_recon_t<<<nblk(c.Z, 64), 64, 0, s>>>(c, d, P, gface, q);
  }
}

void adjoint_stencil_t(const DevCfg& c, const AdjointGeo& geo, const double* P, const double* g, double* Ft,
                       double* ebar, double* q, double* gface, double* out, cudaStream_t s) {
  stencil_q(c, geo, P, g, Ft, ebar, q, gface, s);
  adj::k_fold<<<adj::nblk(c.Zint, 128), 128, 0, s>>>(c, q, out);
}

template <int C, int V>
static void adjoint_step_t(const DevCfg& c, const AdjointGeo& geo, double dt, const AdjointStates& st, double* lam,
                           const AdjointBufs& w, cudaStream_t s) {
  using namespace adj;
  constexpr bool emhd = C || V;
  const bool torus = c.problem == GRIM_PROBLEM_TORUS;
  const size_t rows = (size_t)c.dof * c.Z * sizeof(double);
  // the start-of-stage hooks' and the ghost fill's transposes: q -> out
  auto hooks_fold = [&](const double* Pfill, double* out) {
    if (torus) {
      k_poles_t<<<nblk(2LL * c.N1T * c.N3T, 128), 128, 0, s>>>(c, geo.geoC, w.q);
      k_inflow_t<<<nblk(2LL * c.ng * c.N2T * c.N3T, 64), 64, 0, s>>>(c, geo.geoC, Pfill, w.q);
    }
    k_fold<<<nblk(c.Zint, 128), 128, 0, s>>>(c, w.q, out);
  };
  // the explicit sources' transposes at the stage input Ps, into q
  auto sources = [&](const double* Ps) {
    if (geo.gamma) k_src_t<C, V><<<nblk(c.Zint, 64), 64, 0, s>>>(c, geo.geoC, geo.gamma, Ps, w.g, w.q);
    if constexpr (emhd) {
      fast::emhd_prepass(c, Ps, geo.geoC, w.uTs, s);
      k_emhd_src_t<C, V><<<nblk(c.Zint, 32), 32, 0, s>>>(c, geo.geoC, geo.gamma, Ps, w.uTs, w.g, w.q, w.sbar);
      k_emhd_slope_t<<<nblk(c.Z, 64), 64, 0, s>>>(c, w.uTs, w.sbar, w.uTbar);
      k_emhd_uT_t<C, V><<<nblk(c.Z, 64), 64, 0, s>>>(c, geo.geoC, Ps, w.uTbar, w.q);
    }
  };
  // full stage: the floors at its finish, then the stage at its Newton solution
  if (torus) k_floor_t<C, V><<<nblk(c.Zint, 64), 64, 0, s>>>(c, geo.geoC, st.P1Sol, lam);
  if constexpr (emhd) {
    cudaMemsetAsync(w.p0bar, 0, rows, s);
    k_stage_emhd<C, V><<<nblk(c.Zint, 32), 32, 0, s>>>(c, geo.geoC, GRIM_FULL_STEP, dt, st.P1Sol, st.P0eff, st.PhEff,
                                                      st.divF1, st.Sexp1, lam, w.g, w.p0bar, w.psl);
  } else {
    k_stage<<<nblk(c.Zint, 128), 128, 0, s>>>(c, geo.geoC, st.P1Sol, dt, lam, w.g, w.ubar, w.bacc, 0);
  }
  stencil_q(c, geo, st.PhEff, w.g, w.Ft, w.ebar, w.q, w.gface, s);
  sources(st.PhEff);
  if constexpr (emhd) k_add_interior<<<nblk(c.Zint, 128), 128, 0, s>>>(c, w.psl, w.q);
  hooks_fold(st.PhFill, w.lamh);
  // half stage
  if (torus) k_floor_t<C, V><<<nblk(c.Zint, 64), 64, 0, s>>>(c, geo.geoC, st.PhSol, w.lamh);
  if constexpr (emhd) {
    k_stage_emhd<C, V><<<nblk(c.Zint, 32), 32, 0, s>>>(c, geo.geoC, GRIM_HALF_STEP, 0.5 * dt, st.PhSol, st.P0eff,
                                                      st.P0eff, st.divFh, st.Sexph, w.lamh, w.g, w.p0bar, w.psl);
  } else {
    k_stage<<<nblk(c.Zint, 128), 128, 0, s>>>(c, geo.geoC, st.PhSol, 0.5 * dt, w.lamh, w.g, w.ubar, w.bacc, 1);
  }
  stencil_q(c, geo, st.P0eff, w.g, w.Ft, w.ebar, w.q, w.gface, s);
  sources(st.P0eff);
  if constexpr (emhd) k_add_interior<<<nblk(c.Zint, 128), 128, 0, s>>>(c, w.p0bar, w.q);
  else k_cons<<<nblk(c.Zint, 128), 128, 0, s>>>(c, geo.geoC, st.P0eff, w.ubar, w.bacc, w.q);
  hooks_fold(st.P0fill, lam);
}

void adjoint_step(const DevCfg& c, const AdjointGeo& geo, double dt, const AdjointStates& st, double* lam,
                  const AdjointBufs& w, cudaStream_t s) {
  if (c.conduction && c.viscosity) adjoint_step_t<1, 1>(c, geo, dt, st, lam, w, s);
  else if (c.conduction) adjoint_step_t<1, 0>(c, geo, dt, st, lam, w, s);
  else if (c.viscosity) adjoint_step_t<0, 1>(c, geo, dt, st, lam, w, s);
  else adjoint_step_t<0, 0>(c, geo, dt, st, lam, w, s);
}

}  // namespace grim
