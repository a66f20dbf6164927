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
// Scope: ideal MHD, Minkowski or modified Kerr-Schild, 2D or 3D, periodic /
// outflow / mirror boundaries, no problem hooks, dt held fixed over the
// run; the runtime rejects anything else.  Every accumulation is a gather
// in a fixed order (no atomics), so a gradient is the same bits run to run.
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
template <class T, int N>
GRIM_D Dual<T, N> fmin(const Dual<T, N>& a, const Dual<T, N>& b) { return (b.v < a.v) ? b : a; }
template <class T, int N>
GRIM_D Dual<T, N> fmax(const Dual<T, N>& a, const Dual<T, N>& b) { return (b.v > a.v) ? b : a; }
template <class T, int N>
GRIM_D Dual<T, N> copysign(T a, const Dual<T, N>& b) { return Dual<T, N>(::copysign(a, b.v)); }

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

// lam_out(P0) += dU/dP(P0)^T ubar + [0 ; bacc]
__global__ void k_cons(DevCfg c, const double* __restrict__ geoC, const double* __restrict__ P,
                       const double* __restrict__ ubar, const double* __restrict__ bacc, double* __restrict__ lam) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  const long long Z = c.Z;
  const long long z = interior_to_z(c, n);
  ZoneGeo<double> G;
  centre_geo(c, geoC, z, G);
  double J[5][8];
  cons_jacobian(c, P, z, G, J);
  for (int k = 0; k < 8; k++) {
    double s = 0.;
    for (int r = 0; r < 5; r++) s += J[r][k] * ubar[(long long)r * Z + z];
    if (k >= 5) s += bacc[(long long)(k - 5) * Z + z];
    const long long row = (k < 5) ? k : c.B1 + (k - 5);
    lam[row * Z + z] += s;
  }
}

// The geometric source's transpose (interior zones): out += dS/dP(Ps)^T g
// over the fluid rows, S^nu = -sqrt(-g) T^ka_la Gamma^la_(ka nu) of the
// stage element at the centre (physics.cpp:360-420)
__global__ void k_src_t(DevCfg c, const double* __restrict__ geoC, const double* __restrict__ gamma,
                        const double* __restrict__ P, const double* __restrict__ g, double* __restrict__ out) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  typedef Dual<double, 8> D;
  const long long Z = c.Z;
  const long long z = interior_to_z(c, n);
  int i, j, k;
  zijk(c, z, i, j, k);
  ZoneGeo<double> G0;
  load_geo(G0, c, geoC, z, i, j, 0.5, 0.5);
  ZoneGeo<D> G;
  geo_const(G, G0);
  D q[8];
  for (int v = 0; v < 5; v++) q[v] = D::var(P[(long long)v * Z + z], v);
  for (int v = 0; v < 3; v++) q[5 + v] = D::var(P[(long long)(c.B1 + v) * Z + z], 5 + v);
  ElemT<D, D> e;
  elem_set<0, 0>(e, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], D(0.), D(0.), G, c);
  D T[4][4];
  for (int ka = 0; ka < 4; ka++)
    for (int la = 0; la < 4; la++) T[ka][la] = tmunu<0, 0>(e, ka, la);
  const double* gam = gamma + gidx(c, i, j);
  double acc[8] = {0., 0., 0., 0., 0., 0., 0., 0.};
  for (int nu = 0; nu < 4; nu++) {
    D s(0.);
    for (int ka = 0; ka < 4; ka++)
      for (int la = 0; la < 4; la++) s -= T[ka][la] * (G0.g * __ldg(gam + (long long)(la * 16 + ka * 4 + nu) * c.GZ));
    const double gb = g[(long long)(UU + nu) * Z + z];
    for (int m = 0; m < 8; m++) acc[m] += s.d[m] * gb;
  }
  for (int m = 0; m < 8; m++) {
    const long long row = (m < 5) ? m : c.B1 + (m - 5);
    out[row * Z + z] += acc[m];
  }
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
    for (int v = 0; v < c.dof; v++) {
      const double a = in1 ? g[(long long)v * Z + zm] : 0.;
      const double b = in0 ? g[(long long)v * Z + z] : 0.;
      Ft[((long long)d * c.dof + v) * Z + z] = (a - b) * idx;
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
template <class S>
GRIM_D void riemann_flux(const DevCfg& c, int dir, const ZoneGeo<double>& G0, const S* pl, const S* pr, S* F) {
  ZoneGeo<S> G;
  geo_const(G, G0);
  const int fd = dir + 1;
  S FL[8], UL[8], FR[8], UR[8], mnL, mxL, mnR, mxR;
  {
    ElemT<S, S> e;
    elem_set<0, 0>(e, pl[0], pl[1], pl[2], pl[3], pl[4], pl[5], pl[6], pl[7], S(0.), S(0.), G, c);
    fluxes_fluid<0, 0>(e, fd, G.g, FL, 5, 5);
    fluxes_B(e, fd, G.g, FL + 5);
    fluxes_fluid<0, 0>(e, 0, G.g, UL, 5, 5);
    fluxes_B(e, 0, G.g, UL + 5);
    char_speeds<0, 0>(e, G, dir, c, mnL, mxL);
  }
  {
    ElemT<S, S> e;
    elem_set<0, 0>(e, pr[0], pr[1], pr[2], pr[3], pr[4], pr[5], pr[6], pr[7], S(0.), S(0.), G, c);
    fluxes_fluid<0, 0>(e, fd, G.g, FR, 5, 5);
    fluxes_B(e, fd, G.g, FR + 5);
    fluxes_fluid<0, 0>(e, 0, G.g, UR, 5, 5);
    fluxes_B(e, 0, G.g, UR + 5);
    char_speeds<0, 0>(e, G, dir, c, mnR, mxR);
  }
  const S cmin = dmin2(mnL, mnR), cmax = dmax2(mxL, mxR);
  if (c.riemann == GRIM_HLL) {
    for (int v = 0; v < 8; v++) F[v] = (cmax * FL[v] - cmin * FR[v] + cmin * cmax * (UR[v] - UL[v])) / (cmax - cmin);
  } else {
    const S cm = dmax2(cmax, -cmin);
    for (int v = 0; v < 8; v++) F[v] = S(0.5) * (FL[v] + FR[v] - cm * (UR[v] - UL[v]));
  }
}

// Riemann transpose of the faces along dir: the face between zones
// a = z - s and b = z takes Fbar (dof) and forms the adjoints of its two
// reconstructed states, gl = (dF/dpl)^T Fbar (pl: the right-face state of a)
// and gr = (dF/dpr)^T Fbar (pr: the left-face state of b), into gface
// (rows 0..7 gl, 8..15 gr; zero on the faces the stencil does not use)
__global__ void k_faces_t(DevCfg c, int dir, const double* __restrict__ geoF, const double* __restrict__ P,
                          const double* __restrict__ Ft, double* __restrict__ gface) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  const int x = dir == 0 ? i : (dir == 1 ? j : k);
  const int NT = dir == 0 ? c.N1T : (dir == 1 ? c.N2T : c.N3T);
  const long long Z = c.Z, s = stride_of(c, dir);
  double fb[8];
  bool any = false;
  for (int v = 0; v < 8; v++) {
    fb[v] = (x < 3 || x > NT - 3) ? 0. : Ft[((long long)dir * c.dof + v) * Z + z];
    any |= fb[v] != 0.;
  }
  if (!any) {
    for (int v = 0; v < 16; v++) gface[(long long)v * Z + z] = 0.;
    return;
  }
  // the face states
  double pl[8], pr[8];
  for (int v = 0; v < 8; v++) {
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
  // dF/dpl and dF/dpr, 8 tangent lanes each
  typedef Dual<double, 8> D8;
  for (int side = 0; side < 2; side++) {
    D8 L[8], R[8], F[8];
    for (int v = 0; v < 8; v++) {
      L[v] = side == 0 ? D8::var(pl[v], v) : D8(pl[v]);
      R[v] = side == 1 ? D8::var(pr[v], v) : D8(pr[v]);
    }
    riemann_flux<D8>(c, dir, G, L, R, F);
    for (int k2 = 0; k2 < 8; k2++) {
      double acc = 0.;
      for (int r = 0; r < 8; r++) acc += fb[r] * F[r].d[k2];
      gface[(long long)(side * 8 + k2) * Z + z] = acc;
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
  for (int v = 0; v < 8; v++) {
    const double* a = P + (long long)v * Z;
    double acc = 0.;
    for (int m = 4; m >= 0; m--) {
      // x is point m of the stencil of y = x + 2 - m
      const int y = x + 2 - m;
      if (y < 2 || y > NT - 3) continue;
      const long long zy = z + (long long)(2 - m) * s;
      const double gl = (y + 1 <= NT - 1) ? gface[(long long)v * Z + zy + s] : 0.;
      const double gr = gface[(long long)(8 + v) * Z + zy];
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

void adjoint_stencil_t(const DevCfg& c, const AdjointGeo& geo, const double* P, const double* g, double* Ft,
                       double* ebar, double* q, double* gface, double* out, cudaStream_t s) {
  using namespace adj;
  const size_t bZ = (size_t)c.Z * sizeof(double);
  k_div_t<<<nblk(c.Z, 128), 128, 0, s>>>(c, g, Ft);
  k_ct_t_emf<<<nblk(c.Z, 256), 256, 0, s>>>(c, Ft, ebar);
  k_ct_t_raw<<<nblk(c.Z, 256), 256, 0, s>>>(c, ebar, Ft);
  cudaMemsetAsync(q, 0, (size_t)c.dof * bZ, s);
  for (int d = 0; d < c.dim; d++) {
    k_faces_t<<<nblk(c.Z, 64), 64, 0, s>>>(c, d, geo.geoF[d], P, Ft, gface);
    k_recon_t<<<nblk(c.Z, 64), 64, 0, s>>>(c, d, P, gface, q);
  }
  k_fold<<<nblk(c.Zint, 128), 128, 0, s>>>(c, q, out);
}

void adjoint_step(const DevCfg& c, const AdjointGeo& geo, double dt, const double* P0, const double* Ph,
                  const double* P1, double* lam, const AdjointBufs& w, cudaStream_t s) {
  using namespace adj;
  // full stage at P1
  k_stage<<<nblk(c.Zint, 128), 128, 0, s>>>(c, geo.geoC, P1, dt, lam, w.g, w.ubar, w.bacc, 0);
  adjoint_stencil_t(c, geo, Ph, w.g, w.Ft, w.ebar, w.q, w.gface, w.lamh, s);
  if (geo.gamma) k_src_t<<<nblk(c.Zint, 64), 64, 0, s>>>(c, geo.geoC, geo.gamma, Ph, w.g, w.lamh);
  // half stage at Ph
  k_stage<<<nblk(c.Zint, 128), 128, 0, s>>>(c, geo.geoC, Ph, 0.5 * dt, w.lamh, w.g, w.ubar, w.bacc, 1);
  adjoint_stencil_t(c, geo, P0, w.g, w.Ft, w.ebar, w.q, w.gface, lam, s);
  if (geo.gamma) k_src_t<<<nblk(c.Zint, 64), 64, 0, s>>>(c, geo.geoC, geo.gamma, P0, w.g, lam);
  k_cons<<<nblk(c.Zint, 128), 128, 0, s>>>(c, geo.geoC, P0, w.ubar, w.bacc, lam);
}

}  // namespace grim
