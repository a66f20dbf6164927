/*
 * grim_oracle.cpp -- CPU oracle for the implicit GRMHD/EMHD timestep.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that tests/, bench.py's cpu_baseline
 * leg and __graft_entry__.smoke() compare the CUDA product against.  Nothing
 * in grim_b200/ links or calls this file.
 *
 * It restates, in FP64 and in the reference's operation order, the
 * array-at-a-time pipeline of AFD-Illinois/grim:
 *   every ArrayFire elementwise expression  -> a loop over all zones
 *   af::shift(a, s1, s2, s3)[i]             -> a[i - s] with circular wrap
 *   af::convolve(F, {1,-1,0}/dX)            -> zero-padded forward difference
 *   af::solve (batched)                     -> pivoted Gaussian elimination
 * Full-grid temporaries are kept exactly where the reference keeps them
 * (primLeft/primRight, fluxes per direction, EMFs, divFluxes, sources,
 * cons/consOld, residual, Jacobian), so intermediate arrays can be compared
 * one to one with the product's.
 *
 * Build: g++ -O2 -fopenmp -ffp-contract=off -fno-fast-math (see Makefile).
 */
#include "grim_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

/* --- enums (reference src/params.hpp:32-94) ----------------------------- */
enum { CENTER = 0, LEFT = 1, RIGHT = 2, TOP = 3, BOTTOM = 4 };
enum { PERIODIC = 0, OUTFLOW = 1, MIRROR = 2, DIRICHLET = 3 };
enum { MINKOWSKI = 0, MODIFIED_KERR_SCHILD = 1 };
enum { MINMOD = 0, WENO5 = 1, PPM = 2, MP5 = 3 };
enum { HLL = 0, LOCAL_LAX_FRIEDRICH = 1 };
enum { CLOSURE_CONST_TAU = 0, CLOSURE_TORUS = 1, CLOSURE_TAU_PROFILE = 2 };
enum { HALF_STEP = 0, FULL_STEP = 1 };
enum { RHO = 0, UU = 1, U1 = 2, U2 = 3, U3 = 4 };

static const int NDIM = 4;
typedef std::vector<double> Arr;

#define ZLOOP _Pragma("omp parallel for schedule(static)") for (long z = 0; z < Z; z++)

struct Layout {
  int N1, N2, N3, dim, ng;
  int g1, g2, g3;
  int N1T, N2T, N3T;
  long Z;
  void init(const orc_config& c) {
    dim = c.dim; ng = c.numGhost;
    N1 = c.N1; N2 = (dim >= 2) ? c.N2 : 1; N3 = (dim >= 3) ? c.N3 : 1;
    g1 = ng; g2 = (dim >= 2) ? ng : 0; g3 = (dim >= 3) ? ng : 0;
    N1T = N1 + 2 * g1; N2T = N2 + 2 * g2; N3T = N3 + 2 * g3;
    Z = (long)N1T * N2T * N3T;
  }
  long idx(int i, int j, int k) const { return i + (long)N1T * (j + (long)N2T * k); }
  void ijk(long z, int& i, int& j, int& k) const {
    i = (int)(z % N1T); long r = z / N1T; j = (int)(r % N2T); k = (int)(r / N2T);
  }
  bool interior(long z) const {
    int i, j, k; ijk(z, i, j, k);
    return i >= g1 && i < N1 + g1 && j >= g2 && j < N2 + g2 && k >= g3 && k < N3 + g3;
  }
};

/* af::shift(a, s1, s2, s3)[i,j,k] = a[i-s1, j-s2, k-s3], circular */
static inline int wrapi(int i, int n) { int r = i % n; return r < 0 ? r + n : r; }
static void shift(const Layout& L, const double* a, int s1, int s2, int s3, double* out) {
  const long Z = L.Z;
  ZLOOP {
    int i, j, k; L.ijk(z, i, j, k);
    out[z] = a[L.idx(wrapi(i - s1, L.N1T), wrapi(j - s2, L.N2T), wrapi(k - s3, L.N3T))];
  }
}

struct Grid {
  int nv = 0; long Z = 0; Arr d;
  void init(int nv_, long Z_) { nv = nv_; Z = Z_; d.assign((size_t)nv * Z, 0.0); }
  double* v(int var) { return d.data() + (size_t)var * Z; }
  const double* v(int var) const { return d.data() + (size_t)var * Z; }
};

struct Params {
  orc_config c;
  int Q, DP, B1, B2, B3, nf, dof;
  void init(const orc_config& cc) {
    c = cc;
    Q = 5; DP = 5 + c.conduction;
    nf = 5 + c.conduction + c.viscosity;
    B1 = nf; B2 = nf + 1; B3 = nf + 2; dof = nf + 3;
  }
};

/* ======================================================================== */
/* Geometry -- src/geometry/geometry.cpp, CoordinateChangeFunctionsArray.hpp */
/* ======================================================================== */

struct CoordMap {
  const orc_config* c;
  /* CoordinateChangeFunctionsArray.hpp:4-9 */
  double GammieRadius(double X1) const { return std::exp(X1); }
  /* :11-16 (uses params::hSlope) */
  double GammieTheta(double X2) const {
    return M_PI * X2 + 0.5 * (1 - c->hSlope) * std::sin(2. * M_PI * X2);
  }
  /* :22-46 */
  double ThetaNoCyl(double X1, double X2) const {
    if (c->DerefineThetaHorizon) {
      double cTh0 = std::cos(M_PI * X2);
      double cTh1 = std::cos(GammieTheta(X2));
      double cTh = cTh1 + std::exp(c->X1Start) / std::exp(X1) * (cTh0 - cTh1);
      return std::acos(cTh);
    }
    return GammieTheta(X2);
  }
  /* :57-66 */
  static double Ftr(double x) {
    double c1 = (x <= 0) ? 1. : 0.;
    double c2 = (x >= 1) ? 1. : 0.;
    double res = c2;
    res = res + (c1 - 1) * (c2 - 1) *
                    (std::cos(x * 5 * M_PI) + 70 * std::sin(((2 * x - 1) * M_PI) / 2.) +
                     5 * std::sin(((2 * x - 1) * 3 * M_PI) / 2.) + 64.) / 128.;
    return res;
  }
  /* :83-91 */
  static double Fangle(double x) {
    double c1 = (x <= -1) ? 1. : 0.;
    double c2 = (x >= 1) ? 1. : 0.;
    return c2 * x + (c1 - 1) * (c2 - 1) *
                        (x + 1. + (-140 * std::sin(((x + 1) * M_PI) / 2.) +
                                   (10 * std::sin(((x + 1) * 3 * M_PI) / 2.)) / 3. +
                                   (2 * std::sin(((x + 1) * 5 * M_PI) / 2.)) / 5.) /
                                      (64. * M_PI)) / 2.;
  }
  /* :93-115 */
  static double limlin(double x, double x0, double dx, double y0) {
    return y0 - dx * Fangle((x - x0) * (-1.) / dx);
  }
  static double mins(double f1, double f2, double df) { return limlin(f1, f2, df, f2); }
  static double maxs(double f1, double f2, double df) { return mins(-f1, -f2, df) * (-1.); }
  /* :119-126 */
  static double minmaxs(double f1, double f2, double df, double dir) {
    double cond = (dir >= 0) ? 1. : 0.;
    return cond * maxs(f1, f2, df) + (1 - cond) * mins(f1, f2, df);
  }
  /* :129-138 */
  double sinth0(const double X0[3], const double X[3]) const {
    return GammieRadius(X0[0]) * std::sin(ThetaNoCyl(X0[0], X0[1])) / GammieRadius(X[0]);
  }
  /* :140-149 */
  double sinth1in(const double X0[3], const double X[3]) const {
    return GammieRadius(X0[0]) * std::sin(ThetaNoCyl(X0[0], X[1])) / GammieRadius(X[0]);
  }
  /* :152-170 */
  double th2in(const double X0[3], const double X[3]) const {
    double th0 = std::asin(sinth0(X0, X));
    double a = ThetaNoCyl(X[0], X[1]);
    double b = ThetaNoCyl(X[0], X0[1]);
    double m = ThetaNoCyl(X[0], 0.5);
    return (a - b) / (m - b) * (m - th0) + th0;
  }
  /* :172-177 */
  double func1(const double*, const double X[3]) const { return std::sin(ThetaNoCyl(X[0], X[1])); }
  /* :179-195 */
  double func2(const double X0[3], const double X[3]) const {
    double Xca[3] = {X[0], 0., X[2]};
    double sth1in = sinth1in(X0, X);
    double sth2in = std::sin(th2in(X0, X));
    double sth1inaxis = sinth1in(X0, Xca);
    double sth2inaxis = std::sin(th2in(X0, Xca));
    return minmaxs(sth1in, sth2in, std::fabs(sth2inaxis - sth1inaxis) + 1.e-20, X[0] - X0[0]);
  }
  /* geometry.cpp:510-629 */
  void XtoX(const double X[3], double x[3]) const {
    if (c->metric == MINKOWSKI) { x[0] = X[0]; x[1] = X[1]; x[2] = X[2]; return; }
    x[0] = GammieRadius(X[0]);
    x[1] = ThetaNoCyl(X[0], X[1]);
    x[2] = X[2];
    if (c->DoCylindrify) {
      double Xgrid[3] = {X[0], X[1], X[2]};
      double xGam[3] = {x[0], x[1], x[2]};
      double isMirrored = (Xgrid[1] > 0.5) ? 1. : 0.;
      Xgrid[1] = (1 - isMirrored) * Xgrid[1] + isMirrored * (1. - Xgrid[1]);
      xGam[1] = (1 - isMirrored) * xGam[1] + isMirrored * (M_PI - xGam[1]);
      double isGhost = (Xgrid[1] < 0.) ? 1. : 0.;
      Xgrid[1] = (1 - isGhost) * Xgrid[1] + isGhost * (-(1.0) * Xgrid[1]);
      xGam[1] = (1 - isGhost) * xGam[1] + isGhost * (-(1.0) * xGam[1]);
      double X0[3] = {c->X1cyl, c->X2cyl, 0.};
      double R_cyl = GammieRadius(X0[0]);
      double X1_tr = std::log(0.5 * (R_cyl + std::exp(c->X1Start)));
      double Xtr[3] = {X1_tr, Xgrid[1], Xgrid[2]};
      double f1 = func1(X0, Xgrid);
      double f2 = func2(X0, Xgrid);
      double dftr = func2(X0, Xtr) - func1(X0, Xtr);
      double sinth = maxs(xGam[0] * f1, xGam[0] * f2,
                          GammieRadius(Xtr[0]) * std::fabs(dftr) + 1.e-20) / xGam[0];
      double th = std::asin(sinth);
      th = th * (1 - isGhost * 2);
      x[0] = xGam[0];
      x[1] = isMirrored * (M_PI - th) + (1 - isMirrored) * th;
      x[2] = xGam[2];
    }
  }
  /* geometry.cpp:255-424: gCov[4][4] at coordinates X (hSlope: geometry member) */
  void gCov(const double X[3], double g[4][4]) const {
    for (int m = 0; m < 4; m++) for (int n = 0; n < 4; n++) g[m][n] = 0.;
    if (c->metric == MINKOWSKI) {
      g[0][0] = -1.; g[1][1] = 1.; g[2][2] = 1.; g[3][3] = 1.;
      return;
    }
    const double eps = 1.e-5, a = c->blackHoleSpin, h = c->hSlope;
    double x[3]; XtoX(X, x);
    double r = x[0], theta = x[1];
    double dr_dX1 = r, dr_dX2 = 0.;
    double dtheta_dX2 = M_PI + M_PI * (1 - h) * std::cos(2 * M_PI * X[1]);
    double dtheta_dX1 = 0.;
    if (c->DoCylindrify) {
      double Xp[3] = {X[0] + eps, X[1], X[2]}, Xm[3] = {X[0] - eps, X[1], X[2]};
      double xp[3], xm[3]; XtoX(Xp, xp); XtoX(Xm, xm);
      dr_dX1 = (xp[0] - xm[0]) / (2. * eps);
      dtheta_dX1 = (xp[1] - xm[1]) / (2. * eps);
      double Yp[3] = {X[0], X[1] + eps, X[2]}, Ym[3] = {X[0], X[1] - eps, X[2]};
      XtoX(Yp, xp); XtoX(Ym, xm);
      dr_dX2 = (xp[0] - xm[0]) / (2. * eps);
      dtheta_dX2 = (xp[1] - xm[1]) / (2. * eps);
    }
    double ac = a * std::cos(theta);
    double sigma = r * r + ac * ac;
    double st = std::sin(theta), s2 = st * st;
    double as = a * st, as2 = as * as;
    g[0][0] = -(1. - 2. * r / sigma);
    g[0][1] = (2. * r / sigma) * dr_dX1;
    g[0][2] = (2. * r / sigma) * dr_dX2;
    g[0][3] = -(2. * a * r * s2 / sigma);
    g[1][0] = g[0][1];
    g[1][1] = (1. + 2 * r / sigma) * dr_dX1 * dr_dX1 + (sigma)*dtheta_dX1 * dtheta_dX1;
    g[1][2] = (1. + 2 * r / sigma) * dr_dX1 * dr_dX2 + (sigma)*dtheta_dX1 * dtheta_dX2;
    g[1][3] = -a * (1. + 2. * r / sigma) * s2 * dr_dX1;
    g[2][0] = g[0][2];
    g[2][1] = g[1][2];
    g[2][2] = sigma * dtheta_dX2 * dtheta_dX2 + (1. + 2 * r / sigma) * dr_dX2 * dr_dX2;
    g[2][3] = -a * (1. + 2. * r / sigma) * s2 * dr_dX2;
    g[3][0] = g[0][3];
    g[3][1] = g[1][3];
    g[3][2] = g[2][3];
    g[3][3] = (s2 * (sigma + as2 * (1. + 2 * r / sigma)));
  }
};

/* geometry.cpp:123-253 (cofactor inverse of a symmetric 4x4) */
static void detAndInverse(const double G[4][4], double& gDet, double C[4][4]) {
#define g(a, b) G[a][b]
  gDet = g(0,0)*g(1,1)*g(2,2)*g(3,3) + g(0,0)*g(1,2)*g(2,3)*g(3,1)
       + g(0,0)*g(1,3)*g(2,1)*g(3,2) + g(0,1)*g(1,0)*g(2,3)*g(3,2)
       + g(0,1)*g(1,2)*g(2,0)*g(3,3) + g(0,1)*g(1,3)*g(2,2)*g(3,0)
       + g(0,2)*g(1,0)*g(2,1)*g(3,3) + g(0,2)*g(1,1)*g(2,3)*g(3,0)
       + g(0,2)*g(1,3)*g(2,0)*g(3,1) + g(0,3)*g(1,0)*g(2,2)*g(3,1)
       + g(0,3)*g(1,1)*g(2,0)*g(3,2) + g(0,3)*g(1,2)*g(2,1)*g(3,0)
       - g(0,0)*g(1,1)*g(2,3)*g(3,2) - g(0,0)*g(1,2)*g(2,1)*g(3,3)
       - g(0,0)*g(1,3)*g(2,2)*g(3,1) - g(0,1)*g(1,0)*g(2,2)*g(3,3)
       - g(0,1)*g(1,2)*g(2,3)*g(3,0) - g(0,1)*g(1,3)*g(2,0)*g(3,2)
       - g(0,2)*g(1,0)*g(2,3)*g(3,1) - g(0,2)*g(1,1)*g(2,0)*g(3,3)
       - g(0,2)*g(1,3)*g(2,1)*g(3,0) - g(0,3)*g(1,0)*g(2,1)*g(3,2)
       - g(0,3)*g(1,1)*g(2,2)*g(3,0) - g(0,3)*g(1,2)*g(2,0)*g(3,1);
  C[0][0] = (g(1,1)*g(2,2)*g(3,3) + g(1,2)*g(2,3)*g(3,1) + g(1,3)*g(2,1)*g(3,2)
           - g(1,1)*g(2,3)*g(3,2) - g(1,2)*g(2,1)*g(3,3) - g(1,3)*g(2,2)*g(3,1)) / gDet;
  C[0][1] = (g(0,1)*g(2,3)*g(3,2) + g(0,2)*g(2,1)*g(3,3) + g(0,3)*g(2,2)*g(3,1)
           - g(0,1)*g(2,2)*g(3,3) - g(0,2)*g(2,3)*g(3,1) - g(0,3)*g(2,1)*g(3,2)) / gDet;
  C[0][2] = (g(0,1)*g(1,2)*g(3,3) + g(0,2)*g(1,3)*g(3,1) + g(0,3)*g(1,1)*g(3,2)
           - g(0,1)*g(1,3)*g(3,2) - g(0,2)*g(1,1)*g(3,3) - g(0,3)*g(1,2)*g(3,1)) / gDet;
  C[0][3] = (g(0,1)*g(1,3)*g(2,2) + g(0,2)*g(1,1)*g(2,3) + g(0,3)*g(1,2)*g(2,1)
           - g(0,1)*g(1,2)*g(2,3) - g(0,2)*g(1,3)*g(2,1) - g(0,3)*g(1,1)*g(2,2)) / gDet;
  C[1][0] = C[0][1];
  C[1][1] = (g(0,0)*g(2,2)*g(3,3) + g(0,2)*g(2,3)*g(3,0) + g(0,3)*g(2,0)*g(3,2)
           - g(0,0)*g(2,3)*g(3,2) - g(0,2)*g(2,0)*g(3,3) - g(0,3)*g(2,2)*g(3,0)) / gDet;
  C[1][2] = (g(0,0)*g(1,3)*g(3,2) + g(0,2)*g(1,0)*g(3,3) + g(0,3)*g(1,2)*g(3,0)
           - g(0,0)*g(1,2)*g(3,3) - g(0,2)*g(1,3)*g(3,0) - g(0,3)*g(1,0)*g(3,2)) / gDet;
  C[1][3] = (g(0,0)*g(1,2)*g(2,3) + g(0,2)*g(1,3)*g(2,0) + g(0,3)*g(1,0)*g(2,2)
           - g(0,0)*g(1,3)*g(2,2) - g(0,2)*g(1,0)*g(2,3) - g(0,3)*g(1,2)*g(2,0)) / gDet;
  C[2][0] = C[0][2];
  C[2][1] = C[1][2];
  C[2][2] = (g(0,0)*g(1,1)*g(3,3) + g(0,1)*g(1,3)*g(3,0) + g(0,3)*g(1,0)*g(3,1)
           - g(0,0)*g(1,3)*g(3,1) - g(0,1)*g(1,0)*g(3,3) - g(0,3)*g(1,1)*g(3,0)) / gDet;
  C[2][3] = (g(0,0)*g(1,3)*g(2,1) + g(0,1)*g(1,0)*g(2,3) + g(0,3)*g(1,1)*g(2,0)
           - g(0,0)*g(1,1)*g(2,3) - g(0,1)*g(1,3)*g(2,0) - g(0,3)*g(1,0)*g(2,1)) / gDet;
  C[3][0] = C[0][3];
  C[3][1] = C[1][3];
  C[3][2] = C[2][3];
  C[3][3] = (g(0,0)*g(1,1)*g(2,2) + g(0,1)*g(1,2)*g(2,0) + g(0,2)*g(1,0)*g(2,1)
           - g(0,0)*g(1,2)*g(2,1) - g(0,1)*g(1,0)*g(2,2) - g(0,2)*g(1,1)*g(2,0)) / gDet;
#undef g
}

struct Geom {
  Arr gCov[4][4], gCon[4][4], g, alpha;
  Arr gamma[4][4][4]; /* gammaUpDownDown, center only */
  Arr x[3];           /* physical coordinates xCoords */
  Arr dyn, minRho, minU; /* x1^1.5 and the radial floors (geometry only) */
  bool hasGamma = false;
  /* coordinatesGrid::setXCoords (grid.cpp:168-249) + geometry ctor
   * (geometry.cpp:4-59) + computeConnectionCoeffs (:61-119, center only) */
  void build(const Layout& L, const orc_config& c, int location, bool withGamma) {
    const long Z = L.Z;
    for (int m = 0; m < 4; m++) for (int n = 0; n < 4; n++) { gCov[m][n].assign(Z, 0.); gCon[m][n].assign(Z, 0.); }
    g.assign(Z, 0.); alpha.assign(Z, 0.);
    for (int d = 0; d < 3; d++) x[d].assign(Z, 0.);
    dyn.assign(Z, 0.); minRho.assign(Z, 0.); minU.assign(Z, 0.);
    hasGamma = withGamma;
    if (withGamma) for (int a = 0; a < 4; a++) for (int b = 0; b < 4; b++) for (int e = 0; e < 4; e++) gamma[a][b][e].assign(Z, 0.);
    const double dX1 = (c.X1End - c.X1Start) / L.N1;
    const double dX2 = (c.X2End - c.X2Start) / L.N2;
    const double dX3 = (c.X3End - c.X3Start) / L.N3;
    double o1 = 0.5, o2 = 0.5, o3 = 0.5;
    if (location == LEFT) o1 = 0.; else if (location == RIGHT) o1 = 1.;
    else if (location == BOTTOM) o2 = 0.; else if (location == TOP) o2 = 1.;
    CoordMap cm; cm.c = &c;
    ZLOOP {
      int i, j, k; L.ijk(z, i, j, k);
      double X[3];
      X[0] = c.X1Start + ((double)(i - L.g1) + o1) * dX1;
      X[1] = c.X2Start + ((double)(j - L.g2) + o2) * dX2;
      X[2] = c.X3Start + ((double)(k - L.g3) + o3) * dX3;
      double xx[3]; cm.XtoX(X, xx);
      for (int d = 0; d < 3; d++) x[d][z] = xx[d];
      /* torus/problem.cpp:9-13 and :547-548: functions of the radius only */
      dyn[z] = std::pow(xx[0], 1.5);
      minRho[z] = std::pow(xx[0], c.RhoFloorSlope) * c.RhoFloorAmpl;
      minU[z] = std::pow(xx[0], c.UFloorSlope) * c.UFloorAmpl;
      double G[4][4], C[4][4], det;
      cm.gCov(X, G);
      detAndInverse(G, det, C);
      for (int m = 0; m < 4; m++) for (int n = 0; n < 4; n++) { gCov[m][n][z] = G[m][n]; gCon[m][n][z] = C[m][n]; }
      g[z] = std::sqrt(-det);
      alpha[z] = 1. / std::sqrt(-C[0][0]);
      if (withGamma) {
        const double eps = 1.e-5;
        double Gp[3][4][4], Gm[3][4][4];
        for (int d = 0; d < 3; d++) {
          double Xp[3] = {X[0], X[1], X[2]}, Xm[3] = {X[0], X[1], X[2]};
          Xp[d] += eps; Xm[d] -= eps;
          cm.gCov(Xp, Gp[d]); cm.gCov(Xm, Gm[d]);
        }
        double gDDD[4][4][4];
        for (int eta = 0; eta < 4; eta++) for (int mu = 0; mu < 4; mu++) for (int nu = 0; nu < 4; nu++) {
          /* geometry.cpp:631-680 */
          double out = 0.;
          if (nu > 0) { out += 0.5 * Gp[nu - 1][eta][mu] / (2. * eps); out -= 0.5 * Gm[nu - 1][eta][mu] / (2. * eps); }
          if (mu > 0) { out += 0.5 * Gp[mu - 1][eta][nu] / (2. * eps); out -= 0.5 * Gm[mu - 1][eta][nu] / (2. * eps); }
          if (eta > 0) { out -= 0.5 * Gp[eta - 1][mu][nu] / (2. * eps); out += 0.5 * Gm[eta - 1][mu][nu] / (2. * eps); }
          gDDD[eta][mu][nu] = out;
        }
        for (int mu = 0; mu < 4; mu++) for (int nu = 0; nu < 4; nu++) for (int la = 0; la < 4; la++) {
          double s = 0.;
          for (int eta = 0; eta < 4; eta++) s += C[mu][eta] * gDDD[eta][nu][la];
          gamma[mu][nu][la][z] = s;
        }
      }
    }
  }
};

/* ======================================================================== */
/* fluidElement -- src/physics/physics.cpp, riemannsolver.cpp:54-200         */
/* ======================================================================== */

struct Recon;
struct Elem {
  const Layout* L = nullptr; const Params* P = nullptr; const Geom* geom = nullptr;
  const Recon* recon = nullptr;
  Arr rho, u, u1, u2, u3, B1, B2, B3, pressure, temperature, soundSpeed, gammaLF;
  Arr uCon[4], uCov[4], bCon[4], bCov[4], bSqr, bNorm;
  Arr qTilde, deltaPTilde, q, deltaP, tau, chi_emhd, nu_emhd;
  Arr NUp[4], TUD[4][4];
  Arr gradT[4], dtuCov[4], graduCov[4][4], divuCov, deltaP0, q0;

  void alloc(const Layout& l, const Params& p) {
    L = &l; P = &p; const long Z = l.Z;
    Arr* all[] = {&rho, &u, &u1, &u2, &u3, &B1, &B2, &B3, &pressure, &temperature, &soundSpeed, &gammaLF,
                  &bSqr, &bNorm, &qTilde, &deltaPTilde, &q, &deltaP, &tau, &chi_emhd, &nu_emhd,
                  &divuCov, &deltaP0, &q0};
    for (Arr* a : all) a->assign(Z, 0.);
    for (int m = 0; m < 4; m++) {
      uCon[m].assign(Z, 0.); uCov[m].assign(Z, 0.); bCon[m].assign(Z, 0.); bCov[m].assign(Z, 0.);
      NUp[m].assign(Z, 0.); gradT[m].assign(Z, 0.); dtuCov[m].assign(Z, 0.);
      for (int n = 0; n < 4; n++) { TUD[m][n].assign(Z, 0.); graduCov[m][n].assign(Z, 0.); }
    }
  }

  /* setFluidElementParameters (problem hook) for one zone */
  void closure(long z) {
    const orc_config& c = P->c;
    const double cs = soundSpeed[z];
    if (c.closure == CLOSURE_CONST_TAU) {
      /* linear_modes/problem.cpp:3-8 */
      tau[z] = c.closureTau0;
      chi_emhd[z] = cs * cs * tau[z];
      nu_emhd[z] = cs * cs * tau[z];
    } else if (c.closure == CLOSURE_TAU_PROFILE) {
      /* relaxation time varying linearly with the physical X2 coordinate */
      double s = (geom->x[1][z] - c.X2Start) / (c.X2End - c.X2Start);
      tau[z] = c.closureTau0 + (c.closureTau1 - c.closureTau0) * s;
      chi_emhd[z] = cs * cs * tau[z];
      nu_emhd[z] = cs * cs * tau[z];
    } else {
      /* torus/problem.cpp:7-55 */
      double Dyn = geom->dyn[z];
      double t = Dyn;
      if (c.conduction) {
        double Qmax = c.ConductionClosureFactor * rho[z] * std::pow(cs, 3.);
        double lambda = 0.01;
        double yCon = std::fabs(q[z]) / Qmax;
        yCon = std::exp(-(yCon - 1.) / lambda);
        double fdCon = yCon / (yCon + 1.) + 1.e-5;
        t = std::min(t, Dyn * fdCon);
      }
      if (c.viscosity) {
        const double fl = c.bSqrFloorInFluidElement, p = pressure[z], dP = deltaP[z];
        double dPmod = std::max(p - 2. / 3. * dP, fl) / std::max(p + 1. / 3. * dP, fl);
        double dPmaxPlus = std::min(c.ViscosityClosureFactor * bSqr[z] * 0.5 * dPmod, 1.49 * p / 1.07);
        double dPmaxMinus = std::max(-c.ViscosityClosureFactor * bSqr[z], -2.99 * p / 1.07);
        double cond = (dP > 0.) ? 1. : 0.;
        double dPmax = cond * dPmaxPlus + (1. - cond) * dPmaxMinus;
        double lambda = 0.01;
        double yVis = std::fabs(dP) / (std::fabs(dPmax) + fl);
        yVis = std::exp(-(yVis - 1.) / lambda);
        double fdVis = yVis / (yVis + 1.) + 1.e-5;
        t = std::min(t, Dyn * fdVis);
      }
      tau[z] = t;
      double maxAlpha = (1. - cs * cs) / (2. * cs * cs + 1.e-12);
      chi_emhd[z] = std::min(maxAlpha, c.ConductionAlpha) * cs * cs * t;
      nu_emhd[z] = std::min(maxAlpha, c.ViscosityAlpha) * cs * cs * t;
    }
  }

  /* physics.cpp:53-183 */
  void set(const Grid& prim, const Geom& G) {
    geom = &G;
    const orc_config& c = P->c;
    const long Z = L->Z;
    const double Gam = c.adiabaticIndex;
    ZLOOP {
      rho[z] = std::max(prim.v(RHO)[z], c.rhoFloorInFluidElement);
      u[z] = std::max(prim.v(UU)[z], c.uFloorInFluidElement);
      u1[z] = prim.v(U1)[z]; u2[z] = prim.v(U2)[z]; u3[z] = prim.v(U3)[z];
      B1[z] = prim.v(P->B1)[z]; B2[z] = prim.v(P->B2)[z]; B3[z] = prim.v(P->B3)[z];
      pressure[z] = (Gam - 1.) * u[z];
      temperature[z] = std::max(pressure[z] / rho[z], c.temperatureFloorInFluidElement);
      soundSpeed[z] = std::sqrt(Gam * pressure[z] / (rho[z] + Gam * u[z]));
      const double g11 = G.gCov[1][1][z], g22 = G.gCov[2][2][z], g33 = G.gCov[3][3][z];
      const double g12 = G.gCov[1][2][z], g13 = G.gCov[1][3][z], g23 = G.gCov[2][3][z];
      const double a1 = u1[z], a2 = u2[z], a3 = u3[z];
      gammaLF[z] = std::sqrt(1 + g11 * a1 * a1 + g22 * a2 * a2 + g33 * a3 * a3 +
                             2 * (g12 * a1 * a2 + g13 * a1 * a3 + g23 * a2 * a3));
      const double gam = gammaLF[z], al = G.alpha[z];
      uCon[0][z] = gam / al;
      uCon[1][z] = a1 - gam * G.gCon[0][1][z] * al;
      uCon[2][z] = a2 - gam * G.gCon[0][2][z] * al;
      uCon[3][z] = a3 - gam * G.gCon[0][3][z] * al;
      for (int mu = 0; mu < 4; mu++)
        uCov[mu][z] = G.gCov[mu][0][z] * uCon[0][z] + G.gCov[mu][1][z] * uCon[1][z] +
                      G.gCov[mu][2][z] * uCon[2][z] + G.gCov[mu][3][z] * uCon[3][z];
      bCon[0][z] = B1[z] * uCov[1][z] + B2[z] * uCov[2][z] + B3[z] * uCov[3][z];
      bCon[1][z] = (B1[z] + bCon[0][z] * uCon[1][z]) / uCon[0][z];
      bCon[2][z] = (B2[z] + bCon[0][z] * uCon[2][z]) / uCon[0][z];
      bCon[3][z] = (B3[z] + bCon[0][z] * uCon[3][z]) / uCon[0][z];
      for (int mu = 0; mu < 4; mu++)
        bCov[mu][z] = G.gCov[mu][0][z] * bCon[0][z] + G.gCov[mu][1][z] * bCon[1][z] +
                      G.gCov[mu][2][z] * bCon[2][z] + G.gCov[mu][3][z] * bCon[3][z];
      bSqr[z] = bCon[0][z] * bCov[0][z] + bCon[1][z] * bCov[1][z] + bCon[2][z] * bCov[2][z] +
                bCon[3][z] * bCov[3][z] + c.bSqrFloorInFluidElement;
      bNorm[z] = std::sqrt(bSqr[z]);
      const double cs = soundSpeed[z];
      if (c.conduction == 1) {
        qTilde[z] = prim.v(P->Q)[z];
        if (c.highOrderTermsConduction == 1)
          q[z] = qTilde[z] * temperature[z] * std::sqrt(rho[z] * c.ConductionAlpha * cs * cs);
        else
          q[z] = qTilde[z];
      }
      if (c.viscosity == 1) {
        deltaPTilde[z] = prim.v(P->DP)[z];
        if (c.highOrderTermsViscosity == 1)
          deltaP[z] = deltaPTilde[z] * std::sqrt(temperature[z] * rho[z] * c.ViscosityAlpha * cs * cs);
        else
          deltaP[z] = deltaPTilde[z];
      }
      closure(z);
      const double w = rho[z] + u[z] + pressure[z] + bSqr[z];
      const double pt = pressure[z] + 0.5 * bSqr[z];
      for (int mu = 0; mu < 4; mu++) {
        NUp[mu][z] = rho[z] * uCon[mu][z];
        for (int nu = 0; nu < 4; nu++) {
          double d = (mu == nu) ? 1. : 0.;
          double T = w * uCon[mu][z] * uCov[nu][z] + pt * d - bCon[mu][z] * bCov[nu][z];
          if (c.conduction == 1)
            T += q[z] / bNorm[z] * (uCon[mu][z] * bCov[nu][z] + bCon[mu][z] * uCov[nu][z]);
          if (c.viscosity == 1)
            T += (-deltaP[z]) * (bCon[mu][z] * bCov[nu][z] / bSqr[z] -
                                 (1. / 3.) * (d + uCon[mu][z] * uCov[nu][z]));
          TUD[mu][nu][z] = T;
        }
      }
    }
  }

  /* physics.cpp:185-217 */
  void computeFluxes(int dir, Grid& flux) const {
    const long Z = L->Z;
    const Params& p = *P;
    ZLOOP {
      const double g = geom->g[z];
      double fr = g * NUp[dir][z];
      flux.v(RHO)[z] = fr;
      flux.v(UU)[z] = g * TUD[dir][0][z] + fr;
      flux.v(U1)[z] = g * TUD[dir][1][z];
      flux.v(U2)[z] = g * TUD[dir][2][z];
      flux.v(U3)[z] = g * TUD[dir][3][z];
      flux.v(p.B1)[z] = g * (bCon[1][z] * uCon[dir][z] - bCon[dir][z] * uCon[1][z]);
      flux.v(p.B2)[z] = g * (bCon[2][z] * uCon[dir][z] - bCon[dir][z] * uCon[2][z]);
      flux.v(p.B3)[z] = g * (bCon[3][z] * uCon[dir][z] - bCon[dir][z] * uCon[3][z]);
      if (p.c.conduction) flux.v(p.Q)[z] = g * (uCon[dir][z] * qTilde[z]);
      if (p.c.viscosity) flux.v(p.DP)[z] = g * (uCon[dir][z] * deltaPTilde[z]);
    }
  }

  /* riemannsolver.cpp:54-200; dir is 0,1,2 for X1,X2,X3 */
  void computeMinMaxCharSpeeds(int dir, double* minSpeed, double* maxSpeed) const {
    const orc_config& c = P->c;
    const long Z = L->Z;
    const double Gam = c.adiabaticIndex;
    const int sdir = dir + 1;
    ZLOOP {
      double cAlvenSqr = bSqr[z] / (rho[z] + Gam * u[z] + bSqr[z]);
      double csSqr = soundSpeed[z] * soundSpeed[z];
      double cVisSqr = 0.;
      if (c.viscosity) cVisSqr = 4. / 3. / (rho[z] + Gam * u[z]) * rho[z] * nu_emhd[z] / tau[z];
      double cConSqr = 0.;
      if (c.conduction) cConSqr = (Gam - 1.) * chi_emhd[z] / tau[z];
      cConSqr = 0.5 * (csSqr + cConSqr + std::sqrt(csSqr * csSqr + cConSqr * cConSqr));
      csSqr = cConSqr + cVisSqr;
      csSqr = csSqr + cAlvenSqr - csSqr * cAlvenSqr;
      double cond = (csSqr > 1.) ? 1. : 0.;
      csSqr = csSqr * (1. - cond) + cond;
      /* ACov = e_sdir, BCov = e_0: the contractions below are the reference's
       * sums with the zero terms dropped (they add signed zeros only) */
      const double ASqr = geom->gCon[sdir][sdir][z];
      const double BSqr = geom->gCon[0][0][z];
      const double ADotU = uCon[sdir][z];
      const double BDotU = uCon[0][z];
      const double ADotB = geom->gCon[sdir][0][z];
      double A = (BDotU * BDotU) - (BSqr + BDotU * BDotU) * csSqr;
      double B = 2. * (ADotU * BDotU - (ADotB + ADotU * BDotU) * csSqr);
      double C = ADotU * ADotU - (ASqr + ADotU * ADotU) * csSqr;
      double discr = std::sqrt(std::max(B * B - 4. * A * C, 1.e-16));
      double mn = -(-B + discr) / 2. / A;
      double mx = -(-B - discr) / 2. / A;
      if (mn > -1.e-15) mn = -1.e-15;
      if (mx < 1.e-15) mx = 1.e-15;
      minSpeed[z] = mn; maxSpeed[z] = mx;
    }
  }

  /* physics.cpp:219-317; `this` is the element whose rho, tau, ... are used */
  void computeTimeDerivSources(const Elem& elemOld, const Elem& elemNew, double dt, Grid& src) {
    const orc_config& c = P->c;
    const Params& p = *P;
    const long Z = L->Z;
    std::fill(src.d.begin(), src.d.end(), 0.);
    if (!(c.conduction || c.viscosity)) return;
    ZLOOP {
      for (int mu = 0; mu < 4; mu++) dtuCov[mu][z] = (elemNew.uCov[mu][z] - elemOld.uCov[mu][z]) / dt;
      double div = 0.;
      for (int mu = 0; mu < 4; mu++) div += geom->gCon[0][mu][z] * dtuCov[mu][z];
      divuCov[z] = div;
      const double g = geom->g[z];
      if (c.viscosity) {
        double d0 = -div * rho[z] * nu_emhd[z];
        for (int mu = 0; mu < 4; mu++)
          d0 += 3. * rho[z] * nu_emhd[z] * bCon[0][z] * bCon[mu][z] / bSqr[z] * dtuCov[mu][z];
        if (c.highOrderTermsViscosity == 1)
          d0 *= std::sqrt(tau[z] / rho[z] / nu_emhd[z] / temperature[z]);
        deltaP0[z] = d0;
        double s = -g * (d0) / tau[z];
        if (c.highOrderTermsViscosity == 1) s -= 0.5 * g * div * deltaPTilde[z];
        src.v(p.DP)[z] = s;
      }
      if (c.conduction) {
        double qq = -rho[z] * chi_emhd[z] * bCon[0][z] / bNorm[z] *
                    (elemNew.temperature[z] - elemOld.temperature[z]) / dt;
        for (int nu = 0; nu < 4; nu++)
          qq -= rho[z] * chi_emhd[z] * temperature[z] * bCon[nu][z] / bNorm[z] * uCon[0][z] * dtuCov[nu][z];
        if (c.highOrderTermsConduction == 1) qq *= std::sqrt(tau[z] / rho[z] / chi_emhd[z]) / temperature[z];
        q0[z] = qq;
        double s = -g * (qq) / tau[z];
        if (c.highOrderTermsConduction == 1) s -= 0.5 * g * div * qTilde[z];
        src.v(p.Q)[z] = s;
      }
    }
  }

  /* physics.cpp:320-358 */
  void computeImplicitSources(Grid& src, const Arr& tauDamp) const {
    const orc_config& c = P->c;
    const long Z = L->Z;
    std::fill(src.d.begin(), src.d.end(), 0.);
    if (!(c.conduction || c.viscosity)) return;
    ZLOOP {
      if (c.viscosity) src.v(P->DP)[z] = geom->g[z] * (deltaPTilde[z]) / tauDamp[z];
      if (c.conduction) src.v(P->Q)[z] = geom->g[z] * (qTilde[z]) / tauDamp[z];
    }
  }

  void computeEMHDGradients(const double dX[3]);
  void computeExplicitSources(const double dX[3], Grid& src);
};

/* ======================================================================== */
/* Reconstruction -- src/reconstruction/{minmod,weno5,ppm}.cpp             */
/* ======================================================================== */

struct Recon {
  const Layout* L; const orc_config* c;
  /* minmod.cpp:3-19 (ArrayFire sign: 1 for x<0, 0 otherwise) */
  static double afsign(double x) { return (x < 0.) ? 1. : 0.; }
  static double minmod(double x, double y, double z) {
    double m = std::min(std::min(std::fabs(x), std::fabs(y)), std::fabs(z));
    double sx = 1. - 2. * afsign(x), sy = 1. - 2. * afsign(y), sz = 1. - 2. * afsign(z);
    return 0.25 * std::fabs(sx + sy) * (sx + sz) * m;
  }
  void shifts(int dir, int s, int& a, int& b, int& cc) const {
    a = b = cc = 0; if (dir == 0) a = s; else if (dir == 1) b = s; else cc = s;
  }
  /* stencil values y0..y4 = in[i-2], in[i-1], in[i], in[i+1], in[i+2] */
  void stencil(const double* in, int dir, Arr y[5]) const {
    const long Z = L->Z;
    for (int m = 0; m < 5; m++) y[m].assign(Z, 0.);
    int a, b, cc;
    shifts(dir, 2, a, b, cc); shift(*L, in, a, b, cc, y[0].data());
    shifts(dir, 1, a, b, cc); shift(*L, in, a, b, cc, y[1].data());
    std::memcpy(y[2].data(), in, sizeof(double) * Z);
    shifts(dir, -1, a, b, cc); shift(*L, in, a, b, cc, y[3].data());
    shifts(dir, -2, a, b, cc); shift(*L, in, a, b, cc, y[4].data());
  }
  /* minmod.cpp:21-71 */
  void slopeMM(int dir, double dX, const double* in, double* out) const {
    const long Z = L->Z;
    Arr y[5]; stencil(in, dir, y);
    const double th = c->slopeLimTheta;
    ZLOOP {
      double fwd = (y[3][z] - y[2][z]) / dX;
      double bwd = (y[2][z] - y[1][z]) / dX;
      double cen = bwd + fwd;
      out[z] = minmod(th * bwd, 0.5 * cen, th * fwd);
    }
  }
  /* weno5.cpp:39-65: the live code is the centred 5-point derivative */
  void slope5pt(int dir, double dX, const double* in, double* out) const {
    const long Z = L->Z;
    Arr y[5]; stencil(in, dir, y);
    ZLOOP { out[z] = (-y[4][z] + 8. * y[3][z] - 8. * y[1][z] + y[0][z]) / 12. / dX; }
  }
  /* PPM limited face values (ppm.cpp:41-75 and :120-159) */
  static void ppmFaces(double y0, double y1, double y2, double y3, double y4, double& leftV, double& rightV) {
    double d0 = 2. * (y1 - y0), d1 = 2. * (y2 - y1), d2 = 2. * (y3 - y2), d3 = 2. * (y4 - y3);
    double D1 = 0.5 * (y2 - y0), D2 = 0.5 * (y3 - y1), D3 = 0.5 * (y4 - y2);
    double cz1 = (d1 * d0 <= 0.) ? 1. : 0.;
    double s1 = ((D1 > 0.) ? 1. : 0.) * 2. - 1.;
    double DQ1 = (1. - cz1) * s1 * std::min(std::fabs(D1), std::min(std::fabs(d0), std::fabs(d1)));
    double cz2 = (d2 * d1 <= 0.) ? 1. : 0.;
    double s2 = ((D2 > 0.) ? 1. : 0.) * 2. - 1.;
    double DQ2 = (1. - cz2) * s2 * std::min(std::fabs(D2), std::min(std::fabs(d1), std::fabs(d2)));
    double cz3 = (d3 * d2 <= 0.) ? 1. : 0.;
    double s3 = ((D3 > 0.) ? 1. : 0.) * 2. - 1.;
    double DQ3 = (1. - cz3) * s3 * std::min(std::fabs(D3), std::min(std::fabs(d2), std::fabs(d3)));
    leftV = 0.5 * (y2 + y1) - 1. / 6. * (DQ2 - DQ1);
    rightV = 0.5 * (y3 + y2) - 1. / 6. * (DQ3 - DQ2);
    double corr1 = ((rightV - y2) * (y2 - leftV) <= 0.) ? 1. : 0.;
    double qd = rightV - leftV;
    double qe = 6. * (y2 - 0.5 * (rightV + leftV));
    double corr2 = (qd * (qd - qe) < 0.) ? 1. : 0.;
    double corr3 = (qd * (qd + qe) < 0.) ? 1. : 0.;
    leftV = leftV * (1. - corr1) + corr1 * y2;
    rightV = rightV * (1. - corr1) + corr1 * y2;
    leftV = leftV * (1. - corr2) + corr2 * (3. * y2 - 2. * rightV);
    rightV = rightV * corr2 + (1. - corr2) * rightV * (1. - corr3) + (1. - corr2) * corr3 * (3. * y2 - 2. * leftV);
  }
  /* ppm.cpp:3-77 */
  void slopePPM(int dir, double dX, const double* in, double* out) const {
    const long Z = L->Z;
    Arr y[5]; stencil(in, dir, y);
    ZLOOP {
      double l, r; ppmFaces(y[0][z], y[1][z], y[2][z], y[3][z], y[4][z], l, r);
      out[z] = (r - l) / dX;
    }
  }
  /* reconstruction.cpp:39-64; MP5 has no reference slope: the centred
   * 5-point derivative is used for its EMHD gradients */
  void slope(int dir, double dX, const double* in, double* out) const {
    switch (c->reconstruction) {
      case WENO5: slope5pt(dir, dX, in, out); return;
      case PPM: slopePPM(dir, dX, in, out); return;
      case MP5: slope5pt(dir, dX, in, out); return;
      default: slopeMM(dir, dX, in, out); return;
    }
  }
  /* Suresh & Huynh (1997) MP5 interface value at i+1/2 from the left-biased
   * stencil v[i-2..i+2] (alpha = 4); no counterpart in the reference. */
  static double mm2(double a, double b) { return 0.5 * (std::copysign(1., a) + std::copysign(1., b)) * std::min(std::fabs(a), std::fabs(b)); }
  static double mm4(double a, double b, double c, double d) {
    double s = 0.125 * (std::copysign(1., a) + std::copysign(1., b)) *
               std::fabs((std::copysign(1., a) + std::copysign(1., c)) * (std::copysign(1., a) + std::copysign(1., d)));
    return s * std::min(std::min(std::fabs(a), std::fabs(b)), std::min(std::fabs(c), std::fabs(d)));
  }
  static double mp5(double vm2, double vm1, double v0, double vp1, double vp2) {
    const double alpha = 4.;
    double f = (2. * vm2 - 13. * vm1 + 47. * v0 + 27. * vp1 - 3. * vp2) / 60.;
    double vmp = v0 + mm2(vp1 - v0, alpha * (v0 - vm1));
    if ((f - v0) * (f - vmp) <= 0.) return f;
    double djm1 = vm2 - 2. * vm1 + v0;
    double dj = vm1 - 2. * v0 + vp1;
    double djp1 = v0 - 2. * vp1 + vp2;
    double dm4jph = mm4(4. * dj - djp1, 4. * djp1 - dj, dj, djp1);
    double dm4jmh = mm4(4. * dj - djm1, 4. * djm1 - dj, dj, djm1);
    double vul = v0 + alpha * (v0 - vm1);
    double vav = 0.5 * (v0 + vp1);
    double vmd = vav - 0.5 * dm4jph;
    double vlc = v0 + 0.5 * (v0 - vm1) + 4. / 3. * dm4jmh;
    double vmin = std::max(std::min(std::min(v0, vp1), vmd), std::min(std::min(v0, vul), vlc));
    double vmax = std::min(std::max(std::max(v0, vp1), vmd), std::max(std::max(v0, vul), vlc));
    return f + mm2(vmin - f, vmax - f);
  }
  /* reconstruction.cpp:3-36 + the per-scheme reconstruct routines */
  void reconstruct(const Grid& prim, int dir, Grid& primLeft, Grid& primRight) const {
    const long Z = L->Z;
    for (int var = 0; var < prim.nv; var++) {
      const double* in = prim.v(var);
      double* lo = primLeft.v(var);
      double* ro = primRight.v(var);
      if (c->reconstruction == MINMOD) {
        /* minmod.cpp:73-95 (dX = 1) */
        Arr s(Z); slopeMM(dir, 1., in, s.data());
        ZLOOP { lo[z] = in[z] - 0.5 * s[z]; ro[z] = in[z] + 0.5 * s[z]; }
        continue;
      }
      Arr y[5]; stencil(in, dir, y);
      if (c->reconstruction == WENO5) {
        /* weno5.cpp:111-257 */
        const double eps2 = 1.0e-17;
        ZLOOP {
          double y0 = y[0][z], y1 = y[1][z], y2 = y[2][z], y3 = y[3][z], y4 = y[4][z];
          double beta1 = ((4.0 / 3.0) * y0 * y0 - (19.0 / 3.0) * y0 * y1 + (25.0 / 3.0) * y1 * y1 +
                          (11.0 / 3.0) * y0 * y2 - (31.0 / 3.0) * y1 * y2 + (10.0 / 3.0) * y2 * y2) +
                         eps2 * (1.0 + std::fabs(y0) + std::fabs(y1) + std::fabs(y2));
          double beta2 = ((4.0 / 3.0) * y1 * y1 - (13.0 / 3.0) * y1 * y2 + (13.0 / 3.0) * y2 * y2 +
                          (5.0 / 3.0) * y1 * y3 - (13.0 / 3.0) * y2 * y3 + (4.0 / 3.0) * y3 * y3) +
                         eps2 * (1.0 + std::fabs(y1) + std::fabs(y2) + std::fabs(y3));
          double beta3 = ((10.0 / 3.0) * y2 * y2 - (31.0 / 3.0) * y2 * y3 + (25.0 / 3.0) * y3 * y3 +
                          (11.0 / 3.0) * y2 * y4 - (19.0 / 3.0) * y3 * y4 + (4.0 / 3.0) * y4 * y4) +
                         eps2 * (1.0 + std::fabs(y2) + std::fabs(y3) + std::fabs(y4));
          double w1r = 1.0 / (16.0 * beta1 * beta1);
          double w2r = 5.0 / (8.0 * beta2 * beta2);
          double w3r = 5.0 / (16.0 * beta3 * beta3);
          double w1l = 5.0 / (16.0 * beta1 * beta1);
          double w2l = 5.0 / (8.0 * beta2 * beta2);
          double w3l = 1.0 / (16.0 * beta3 * beta3);
          double denl = w1l + w2l + w3l;
          double denr = w1r + w2r + w3r;
          double u1r = 0.375 * y0 - 1.25 * y1 + 1.875 * y2;
          double u2r = -0.125 * y1 + 0.75 * y2 + 0.375 * y3;
          double u3r = 0.375 * y2 + 0.75 * y3 - 0.125 * y4;
          double u1l = -0.125 * y0 + 0.75 * y1 + 0.375 * y2;
          double u2l = 0.375 * y1 + 0.75 * y2 - 0.125 * y3;
          double u3l = 1.875 * y2 - 1.25 * y3 + 0.375 * y4;
          lo[z] = (w1l * u1l + w2l * u2l + w3l * u3l) / denl;
          ro[z] = (w1r * u1r + w2r * u2r + w3r * u3r) / denr;
        }
      } else if (c->reconstruction == PPM) {
        /* ppm.cpp:81-164 */
        ZLOOP { ppmFaces(y[0][z], y[1][z], y[2][z], y[3][z], y[4][z], lo[z], ro[z]); }
      } else {
        /* MP5: right face from the left-biased stencil, left face mirrored */
        ZLOOP {
          ro[z] = mp5(y[0][z], y[1][z], y[2][z], y[3][z], y[4][z]);
          lo[z] = mp5(y[4][z], y[3][z], y[2][z], y[1][z], y[0][z]);
        }
      }
    }
  }
};


/* physics.cpp:502-586 */
void Elem::computeEMHDGradients(const double dX[3]) {
  const orc_config& c = P->c;
  const long Z = L->Z;
  const Recon& R = *recon;
  Arr tmp(Z);
  for (int mu = 0; mu < NDIM; mu++) {
    std::fill(graduCov[0][mu].begin(), graduCov[0][mu].end(), 0.);
    R.slope(0, dX[0], uCov[mu].data(), graduCov[1][mu].data());
    std::fill(graduCov[2][mu].begin(), graduCov[2][mu].end(), 0.);
    if (c.dim > 1) R.slope(1, dX[1], uCov[mu].data(), graduCov[2][mu].data());
    std::fill(graduCov[3][mu].begin(), graduCov[3][mu].end(), 0.);
    if (c.dim > 2) R.slope(2, dX[2], uCov[mu].data(), graduCov[3][mu].data());
    ZLOOP {
      for (int nu = 0; nu < NDIM; nu++)
        for (int la = 0; la < NDIM; la++)
          graduCov[nu][mu][z] -= geom->gamma[la][nu][mu][z] * uCov[la][z];
    }
  }
  if (c.conduction) {
    std::fill(gradT[0].begin(), gradT[0].end(), 0.);
    R.slope(0, dX[0], temperature.data(), gradT[1].data());
    std::fill(gradT[2].begin(), gradT[2].end(), 0.);
    if (c.dim > 1) R.slope(1, dX[1], temperature.data(), gradT[2].data());
    std::fill(gradT[3].begin(), gradT[3].end(), 0.);
    if (c.dim > 2) R.slope(2, dX[2], temperature.data(), gradT[3].data());
  }
}

/* physics.cpp:360-500 */
void Elem::computeExplicitSources(const double dX[3], Grid& src) {
  const orc_config& c = P->c;
  const Params& p = *P;
  const long Z = L->Z;
  std::fill(src.d.begin(), src.d.end(), 0.);
  if (c.metric != MINKOWSKI) {
    ZLOOP {
      for (int nu = 0; nu < NDIM; nu++)
        for (int ka = 0; ka < NDIM; ka++)
          for (int la = 0; la < NDIM; la++)
            src.v(UU + nu)[z] -= geom->g[z] * TUD[ka][la][z] * geom->gamma[la][ka][nu][z];
    }
  }
  if (c.conduction || c.viscosity) {
    computeEMHDGradients(dX);
    ZLOOP {
      double div = 0.;
      for (int mu = 0; mu < NDIM; mu++)
        for (int nu = 0; nu < NDIM; nu++) div += geom->gCon[mu][nu][z] * graduCov[mu][nu][z];
      divuCov[z] = div;
      const double g = geom->g[z];
      if (c.viscosity) {
        double d0 = -div * rho[z] * nu_emhd[z];
        for (int mu = 0; mu < NDIM; mu++)
          for (int nu = 0; nu < NDIM; nu++)
            d0 += 3. * rho[z] * nu_emhd[z] * bCon[mu][z] * bCon[nu][z] / bSqr[z] * graduCov[mu][nu][z];
        deltaP0[z] = d0;
        double d0t = (c.highOrderTermsViscosity == 1) ? d0 * std::sqrt(tau[z] / rho[z] / nu_emhd[z] / temperature[z]) : d0;
        double s = -g * (d0t) / tau[z];
        if (c.highOrderTermsViscosity == 1) s -= 0.5 * g * div * deltaPTilde[z];
        src.v(p.DP)[z] = s;
      }
      if (c.conduction) {
        double qq = 0.;
        for (int mu = 0; mu < NDIM; mu++) {
          qq -= rho[z] * chi_emhd[z] * bCon[mu][z] / bNorm[z] * gradT[mu][z];
          for (int nu = 0; nu < NDIM; nu++)
            qq -= rho[z] * chi_emhd[z] * temperature[z] * bCon[nu][z] / bNorm[z] * uCon[mu][z] * graduCov[mu][nu][z];
        }
        q0[z] = qq;
        double qt = (c.highOrderTermsConduction == 1) ? qq * std::sqrt(tau[z] / rho[z] / chi_emhd[z]) / temperature[z] : qq;
        double s = -g * (qt) / tau[z];
        if (c.highOrderTermsConduction == 1) s -= 0.5 * g * div * qTilde[z];
        src.v(p.Q)[z] = s;
      }
    }
  }
}

/* pivoted Gaussian elimination of one n x n system (row-major A, in place) */
static int solveDense(int n, double* A, double* b, double* x) {
  for (int k = 0; k < n; k++) {
    int p = k; double best = std::fabs(A[k * n + k]);
    for (int i = k + 1; i < n; i++) {
      double v = std::fabs(A[i * n + k]);
      if (v > best) { best = v; p = i; }
    }
    if (p != k) {
      for (int j = 0; j < n; j++) std::swap(A[k * n + j], A[p * n + j]);
      std::swap(b[k], b[p]);
    }
    const double akk = A[k * n + k];
    for (int i = k + 1; i < n; i++) {
      double l = A[i * n + k] / akk;
      for (int j = k + 1; j < n; j++) A[i * n + j] -= l * A[k * n + j];
      b[i] -= l * b[k];
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = b[i];
    for (int j = i + 1; j < n; j++) s -= A[i * n + j] * x[j];
    x[i] = s / A[i * n + i];
  }
  return 0;
}

/* ======================================================================== */
/* timeStepper -- src/timestepper/ (all files)                                    */
/* ======================================================================== */

struct Stepper {
  Layout L; Params P; Recon R;
  Geom geomLeft, geomRight, geomBottom, geomTop, geomCenter;
  double dX[3];
  double time = 0, dt = 0;
  int currentStep = HALF_STEP;
  Grid prim, primOld, primHalfStep, cons, consOld;
  Grid sourcesExplicit, sourcesImplicit, sourcesImplicitOld, sourcesTimeDer;
  Grid primLeft, primRight, fluxesX1, fluxesX2, fluxesX3, divFluxes;
  Arr emfX1, emfX2, emfX3;
  Grid residual, residualPlusEps, primGuessPlusEps, primGuessLineSearchTrial;
  Arr residualMask;
  Elem elem, elemOld, elemHalfStep, elemFace;
  Grid fluxLeft, fluxRight, consLeft, consRight;
  Arr minSpeedLeft, maxSpeedLeft, minSpeedRight, maxSpeedRight;
  int lastIters[2] = {0, 0};

  void init(const orc_config& c) {
    L.init(c); P.init(c); R.L = &L; R.c = &P.c;
    const long Z = L.Z;
    dX[0] = (c.X1End - c.X1Start) / L.N1;
    dX[1] = (c.X2End - c.X2Start) / L.N2;
    dX[2] = (c.X3End - c.X3Start) / L.N3;
    time = c.time; dt = c.dt;
    geomLeft.build(L, c, LEFT, false);
    geomRight.build(L, c, RIGHT, false);
    geomBottom.build(L, c, BOTTOM, false);
    geomTop.build(L, c, TOP, false);
    geomCenter.build(L, c, CENTER, true);
    const int dof = P.dof, nf = P.nf;
    for (Grid* g : {&prim, &primOld, &primHalfStep, &cons, &consOld, &sourcesExplicit, &sourcesImplicit,
                    &sourcesImplicitOld, &sourcesTimeDer, &primLeft, &primRight, &fluxesX1, &fluxesX2,
                    &fluxesX3, &divFluxes, &primGuessPlusEps, &primGuessLineSearchTrial, &fluxLeft,
                    &fluxRight, &consLeft, &consRight})
      g->init(dof, Z);
    residual.init(nf, Z); residualPlusEps.init(nf, Z);
    emfX1.assign(Z, 0.); emfX2.assign(Z, 0.); emfX3.assign(Z, 0.);
    minSpeedLeft.assign(Z, 1.); maxSpeedLeft.assign(Z, 1.); minSpeedRight.assign(Z, 1.); maxSpeedRight.assign(Z, 1.);
    residualMask.assign(Z, 0.);
    for (long z = 0; z < Z; z++) if (L.interior(z)) residualMask[z] = 1.;
    elem.alloc(L, P); elemOld.alloc(L, P); elemHalfStep.alloc(L, P); elemFace.alloc(L, P);
    for (Elem* e : {&elem, &elemOld, &elemHalfStep, &elemFace}) e->recon = &R;
    /* timestepper.cpp:287-295: the elements are first set on the zero grids */
    elem.set(prim, geomCenter); elemOld.set(primOld, geomCenter); elemHalfStep.set(primHalfStep, geomCenter);
    elemFace.set(prim, geomCenter);
  }

  /* boundary.cpp:5-241 (periodic directions are left to communicate()) */
  void applyBoundaryConditions(double* d, int nv) const {
    const orc_config& c = P.c;
    const int ng = L.ng, N1 = L.N1, N2 = L.N2, N3 = L.N3;
    auto at = [&](int v, int i, int j, int k) -> double& { return d[(size_t)v * L.Z + L.idx(i, j, k)]; };
    for (int v = 0; v < nv; v++) {
      /* X1 */
      for (int k = 0; k < L.N3T; k++) for (int j = 0; j < L.N2T; j++) {
        for (int g = 0; g < ng; g++) {
          if (c.boundaryLeft == MIRROR) at(v, g, j, k) = at(v, 2 * ng - 1 - g, j, k);
          else if (c.boundaryLeft == OUTFLOW) at(v, g, j, k) = at(v, ng, j, k);
          if (c.boundaryRight == MIRROR) at(v, N1 + ng + g, j, k) = at(v, N1 + ng - 1 - g, j, k);
          else if (c.boundaryRight == OUTFLOW) at(v, N1 + ng + g, j, k) = at(v, N1 + ng - 1, j, k);
        }
      }
      /* X2 */
      if (L.dim >= 2)
        for (int k = 0; k < L.N3T; k++) for (int i = 0; i < L.N1T; i++) {
          for (int g = 0; g < ng; g++) {
            if (c.boundaryBottom == MIRROR) at(v, i, g, k) = at(v, i, 2 * ng - 1 - g, k);
            else if (c.boundaryBottom == OUTFLOW) at(v, i, g, k) = at(v, i, ng, k);
            if (c.boundaryTop == MIRROR) at(v, i, N2 + ng + g, k) = at(v, i, N2 + ng - 1 - g, k);
            else if (c.boundaryTop == OUTFLOW) at(v, i, N2 + ng + g, k) = at(v, i, N2 + ng - 1, k);
          }
        }
      /* X3 */
      if (L.dim >= 3)
        for (int j = 0; j < L.N2T; j++) for (int i = 0; i < L.N1T; i++) {
          for (int g = 0; g < ng; g++) {
            if (c.boundaryBack == MIRROR) at(v, i, j, g) = at(v, i, j, 2 * ng - 1 - g);
            else if (c.boundaryBack == OUTFLOW) at(v, i, j, g) = at(v, i, j, ng);
            if (c.boundaryFront == MIRROR) at(v, i, j, N3 + ng + g) = at(v, i, j, N3 + ng - 1 - g);
            else if (c.boundaryFront == OUTFLOW) at(v, i, j, N3 + ng + g) = at(v, i, j, N3 + ng - 1);
          }
        }
    }
  }

  /* grid::communicate (grid.cpp:306-360) with PETSc DMDA semantics:
   * periodic ghost zones (corners included) are wrapped from the interior;
   * ghost zones on a non-periodic (DM_BOUNDARY_GHOSTED) edge are read back
   * from the never-written local vector, i.e. zero. */
  void communicate(double* d, int nv) const {
    const orc_config& c = P.c;
    const bool p1 = (c.boundaryLeft == PERIODIC || c.boundaryRight == PERIODIC);
    const bool p2 = (c.boundaryBottom == PERIODIC || c.boundaryTop == PERIODIC);
    const bool p3 = (c.boundaryBack == PERIODIC || c.boundaryFront == PERIODIC);
    const long Z = L.Z;
    for (int v = 0; v < nv; v++) {
      double* a = d + (size_t)v * Z;
      Arr src(a, a + Z);
      ZLOOP {
        int i, j, k; L.ijk(z, i, j, k);
        bool zero = false;
        auto mapd = [&](int x, int g, int N, bool per) -> int {
          if (x >= g && x < N + g) return x;
          if (!per) { zero = true; return x; }
          return g + wrapi(x - g, N);
        };
        int si = mapd(i, L.g1, L.N1, p1);
        int sj = mapd(j, L.g2, L.N2, p2);
        int sk = mapd(k, L.g3, L.N3, p3);
        a[z] = zero ? 0. : src[L.idx(si, sj, sk)];
      }
    }
  }

  /* riemannsolver.cpp:202-328 */
  void riemannSolve(const Grid& pL, const Grid& pR, const Geom& gL, const Geom& gR, int dir, Grid& flux) {
    const long Z = L.Z;
    const int fluxDirection = dir + 1;
    int s1 = (dir == 0), s2 = (dir == 1), s3 = (dir == 2);
    elemFace.set(pR, gR);
    elemFace.computeFluxes(fluxDirection, fluxLeft);
    elemFace.computeFluxes(0, consLeft);
    elemFace.computeMinMaxCharSpeeds(dir, minSpeedLeft.data(), maxSpeedLeft.data());
    elemFace.set(pL, gL);
    elemFace.computeFluxes(fluxDirection, fluxRight);
    elemFace.computeFluxes(0, consRight);
    elemFace.computeMinMaxCharSpeeds(dir, minSpeedRight.data(), maxSpeedRight.data());
    Arr t(Z);
    shift(L, minSpeedLeft.data(), s1, s2, s3, t.data()); minSpeedLeft = t;
    shift(L, maxSpeedLeft.data(), s1, s2, s3, t.data()); maxSpeedLeft = t;
    ZLOOP {
      minSpeedLeft[z] = std::min(minSpeedLeft[z], minSpeedRight[z]);
      maxSpeedLeft[z] = std::max(maxSpeedLeft[z], maxSpeedRight[z]);
    }
    Arr fl(Z), cl(Z);
    for (int var = 0; var < pL.nv; var++) {
      shift(L, fluxLeft.v(var), s1, s2, s3, fl.data());
      shift(L, consLeft.v(var), s1, s2, s3, cl.data());
      const double* fr = fluxRight.v(var);
      const double* cr = consRight.v(var);
      double* out = flux.v(var);
      if (P.c.riemannSolver == HLL) {
        ZLOOP {
          const double cmin = minSpeedLeft[z], cmax = maxSpeedLeft[z];
          out[z] = (cmax * fl[z] - cmin * fr[z] + cmin * cmax * (cr[z] - cl[z])) / (cmax - cmin);
        }
      } else {
        ZLOOP {
          const double cmin = minSpeedLeft[z], cmax = maxSpeedLeft[z];
          out[z] = 0.5 * (fl[z] + fr[z] - std::max(cmax, -cmin) * (cr[z] - cl[z]));
        }
      }
    }
  }

  /* constrainedtransport.cpp:53-83 */
  void computeEMF() {
    if (L.dim < 2) return;
    const long Z = L.Z;
    const Params& p = P;
    Arr a(Z), b(Z);
    shift(L, fluxesX1.v(p.B2), 0, 1, 0, a.data());
    shift(L, fluxesX2.v(p.B1), 1, 0, 0, b.data());
    ZLOOP { emfX3[z] = 0.25 * (fluxesX1.v(p.B2)[z] + a[z] - fluxesX2.v(p.B1)[z] - b[z]); }
    if (L.dim == 3) {
      shift(L, fluxesX2.v(p.B3), 0, 0, 1, a.data());
      shift(L, fluxesX3.v(p.B2), 0, 1, 0, b.data());
      ZLOOP { emfX1[z] = 0.25 * (fluxesX2.v(p.B3)[z] + a[z] - fluxesX3.v(p.B2)[z] - b[z]); }
      shift(L, fluxesX3.v(p.B1), 1, 0, 0, a.data());
      shift(L, fluxesX1.v(p.B3), 0, 0, 1, b.data());
      ZLOOP { emfX2[z] = 0.25 * (fluxesX3.v(p.B1)[z] + a[z] - fluxesX1.v(p.B3)[z] - b[z]); }
    }
  }

  /* constrainedtransport.cpp:3-51 */
  void fluxCT() {
    if (L.dim < 2) return;
    computeEMF();
    const long Z = L.Z;
    const Params& p = P;
    Arr a(Z);
    std::fill(fluxesX1.v(p.B1), fluxesX1.v(p.B1) + Z, 0.);
    shift(L, emfX3.data(), 0, -1, 0, a.data());
    ZLOOP { fluxesX1.v(p.B2)[z] = 0.5 * (emfX3[z] + a[z]); }
    shift(L, emfX3.data(), -1, 0, 0, a.data());
    ZLOOP { fluxesX2.v(p.B1)[z] = -0.5 * (emfX3[z] + a[z]); }
    std::fill(fluxesX2.v(p.B2), fluxesX2.v(p.B2) + Z, 0.);
    if (L.dim == 3) {
      shift(L, emfX2.data(), 0, 0, -1, a.data());
      ZLOOP { fluxesX1.v(p.B3)[z] = -0.5 * (emfX2[z] + a[z]); }
      shift(L, emfX1.data(), 0, 0, -1, a.data());
      ZLOOP { fluxesX2.v(p.B3)[z] = 0.5 * (emfX1[z] + a[z]); }
      shift(L, emfX2.data(), -1, 0, 0, a.data());
      ZLOOP { fluxesX3.v(p.B1)[z] = 0.5 * (emfX2[z] + a[z]); }
      shift(L, emfX1.data(), 0, -1, 0, a.data());
      ZLOOP { fluxesX3.v(p.B2)[z] = -0.5 * (emfX1[z] + a[z]); }
      std::fill(fluxesX3.v(p.B3), fluxesX3.v(p.B3) + Z, 0.);
    }
  }

  /* fvmfluxes.cpp:3-183 */
  void computeDivOfFluxes(const Grid& primFlux) {
    const long Z = L.Z;
    R.reconstruct(primFlux, 0, primLeft, primRight);
    riemannSolve(primLeft, primRight, geomLeft, geomRight, 0, fluxesX1);
    if (L.dim >= 2) {
      R.reconstruct(primFlux, 1, primLeft, primRight);
      riemannSolve(primLeft, primRight, geomBottom, geomTop, 1, fluxesX2);
    }
    if (L.dim >= 3) {
      R.reconstruct(primFlux, 2, primLeft, primRight);
      riemannSolve(primLeft, primRight, geomCenter, geomCenter, 2, fluxesX3);
    }
    fluxCT();
    applyProblemSpecificFluxFilter();
    const double i1 = 1. / dX[0], i2 = 1. / dX[1];
    for (int var = 0; var < primFlux.nv; var++) {
      const double* F1 = fluxesX1.v(var);
      const double* F2 = fluxesX2.v(var);
      const double* F3 = fluxesX3.v(var);
      double* out = divFluxes.v(var);
      if (L.dim <= 2) {
        /* af::convolve with the filter {1,-1,0}/dX, zero padded */
        ZLOOP {
          int i, j, k; L.ijk(z, i, j, k);
          double f1p = (i + 1 < L.N1T) ? F1[z + 1] : 0.;
          double d1 = f1p * i1 + F1[z] * (-i1);
          if (L.dim == 2) {
            double f2p = (j + 1 < L.N2T) ? F2[z + L.N1T] : 0.;
            double d2 = f2p * i2 + F2[z] * (-i2);
            out[z] = d1 + d2;
          } else {
            out[z] = d1;
          }
        }
      } else {
        ZLOOP {
          int i, j, k; L.ijk(z, i, j, k);
          double a1 = F1[L.idx(wrapi(i + 1, L.N1T), j, k)];
          double a2 = F2[L.idx(i, wrapi(j + 1, L.N2T), k)];
          double a3 = F3[L.idx(i, j, wrapi(k + 1, L.N3T))];
          out[z] = (a1 - F1[z]) / dX[0] + (a2 - F2[z]) / dX[1] + (a3 - F3[z]) / dX[2];
        }
      }
    }
  }

  bool torus() const { return P.c.problem == 1; }

  /* torus/problem.cpp:1243-1285 */
  void applyProblemSpecificFluxFilter() {
    if (!torus()) return;
    const int ng = L.ng, N1 = L.N1, N2 = L.N2;
    for (int k = 0; k < L.N3T; k++)
      for (int j = 0; j < L.N2T; j++) {
        double& a = fluxesX1.v(RHO)[L.idx(ng, j, k)];
        a = std::min(a, 0.);
        double& b = fluxesX1.v(RHO)[L.idx(N1 + ng, j, k)];
        b = std::max(b, 0.);
      }
    if (L.dim < 2) return;
    for (int k = 0; k < L.N3T; k++)
      for (int i = 0; i < L.N1T; i++) {
        for (int var = 0; var < P.dof; var++) fluxesX2.v(var)[L.idx(i, ng, k)] = 0.;
        fluxesX1.v(P.B2)[L.idx(i, ng - 1, k)] = fluxesX1.v(P.B2)[L.idx(i, ng, k)] * (-1.0);
        for (int var = 0; var < P.dof; var++) fluxesX2.v(var)[L.idx(i, N2 + ng, k)] = 0.;
        fluxesX1.v(P.B2)[L.idx(i, N2 + ng, k)] = fluxesX1.v(P.B2)[L.idx(i, N2 + ng - 1, k)] * (-1.0);
      }
  }

  /* inflowCheck (torus/problem.cpp:941-1044) */
  void inflowCheck(Grid& prim, Elem& elemBC) {
    const int ng = L.ng, N1 = L.N1;
    const double vSqrMax = 1. - 1. / P.c.MaxLorentzFactor / P.c.MaxLorentzFactor;
    const double vSqrMin = 1.e-13;
    const Geom& G = geomCenter;
    for (int side = 0; side < 2; side++) {  // right boundary first, then left
      const bool right = (side == 0);
      elemBC.set(prim, G);
      for (int k = 0; k < L.N3T; k++)
        for (int j = 0; j < L.N2T; j++)
          for (int gi = 0; gi < ng; gi++) {
            const int i = right ? N1 + ng + gi : gi;
            const long z = L.idx(i, j, k);
            double* U[3] = {&prim.v(U1)[z], &prim.v(U2)[z], &prim.v(U3)[z]};
            for (int a = 0; a < 3; a++) *U[a] = *U[a] / elemBC.gammaLF[z];
            if (right) {
              const long ze = L.idx(N1 + ng - 1, j, k);
              const double minUr = G.gCon[0][1][ze] * G.alpha[ze];
              *U[0] = std::max(minUr, *U[0]);
            } else {
              *U[0] = std::min(G.gCon[0][1][z] * G.alpha[z], *U[0]);
            }
            double vSqr = *U[0] * 0.;
            for (int a = 0; a < 3; a++)
              for (int b = 0; b < 3; b++) vSqr += G.gCov[a + 1][b + 1][z] * *U[a] * *U[b];
            vSqr = std::max(std::min(vSqr, vSqrMax), vSqrMin);
            const double lf = 1. / std::sqrt(1. - vSqr);
            for (int a = 0; a < 3; a++) *U[a] = *U[a] * lf;
          }
      elemBC.set(prim, G);
    }
  }

  /* fixPoles (torus/problem.cpp:1046-1215) */
  void fixPoles(Grid& prim) {
    const int ng = L.ng, N2 = L.N2;
    const Geom& G = geomCenter;
    for (int pole = 0; pole < 2; pole++) {
      const bool top = (pole == 1);
      const int idx0 = top ? N2 + ng - 1 : ng;
      const int idx1 = top ? idx0 - 1 : ng + 1;
      const int idx2 = top ? idx0 - 2 : ng + 2;
      for (int k = 0; k < L.N3T; k++)
        for (int i = 0; i < L.N1T; i++) {
          auto at = [&](int v, int j) -> double& { return prim.v(v)[L.idx(i, j, k)]; };
          auto th = [&](int j) -> double {
            double t = G.x[1][L.idx(i, j, k)];
            return top ? t * (-1.) + M_PI : t;
          };
          for (int jj : {idx0, idx1}) {
            at(RHO, jj) = at(RHO, idx2);
            at(UU, jj) = at(UU, idx2);
            at(U1, jj) = at(U1, idx2);
            at(U2, jj) = at(U2, idx2) * th(jj) / th(idx2);
            at(U3, jj) = at(U3, idx2);
            if (P.c.conduction) at(P.Q, jj) = at(P.Q, idx2) * th(jj) / th(idx2);
            if (P.c.viscosity) at(P.DP, jj) = at(P.DP, idx2) * th(jj) / th(idx2);
          }
          for (int g = 0; g < ng; g++) {
            const int dst = top ? N2 + ng + g : ng - 1 - g;
            const int src = top ? N2 + ng - 1 - g : ng + g;
            at(RHO, dst) = at(RHO, src);
            at(UU, dst) = at(UU, src);
            at(U1, dst) = at(U1, src);
            at(U3, dst) = at(U3, src);
            at(U2, dst) = at(U2, src) * (-1.0);
            at(P.B1, dst) = at(P.B1, src);
            at(P.B3, dst) = at(P.B3, src);
            at(P.B2, dst) = at(P.B2, src) * (-1.0);
            if (P.c.conduction) at(P.Q, dst) = at(P.Q, src) * (-1.0);
            if (P.c.viscosity) at(P.DP, dst) = at(P.DP, src) * (-1.0);
          }
        }
    }
  }

  /* setProblemSpecificBCs (torus/problem.cpp:1217-1241) */
  void setProblemSpecificBCs(Grid& prim) {
    if (!torus()) return;
    Elem& e = (currentStep == HALF_STEP) ? elemOld : elemHalfStep;
    inflowCheck(prim, e);
    if (L.dim >= 2) fixPoles(prim);
  }

  /* applyFloor (torus/problem.cpp:542-712) */
  void applyFloor(Grid& prim, Elem& elem) {
    const orc_config& c = P.c;
    const long Z = L.Z;
    const Geom& G = geomCenter;
    Arr minRho(Z), minU(Z), rho_pre(Z), u_pre(Z), usefloor(Z), bsq1(Z);
    double* rho = prim.v(RHO);
    double* u = prim.v(UU);
    ZLOOP {
      minRho[z] = G.minRho[z];
      minU[z] = G.minU[z];
      rho_pre[z] = rho[z] * 1.;
      u_pre[z] = u[z] * 1.;
      double cd = (rho[z] < minRho[z]) ? 1. : 0.;
      usefloor[z] = cd;
      rho[z] = cd * minRho[z] + (1. - cd) * rho[z];
      cd = (u[z] < minU[z]) ? 1. : 0.;
      usefloor[z] = std::max(cd, usefloor[z]);
      u[z] = cd * minU[z] + (1. - cd) * u[z];
    }
    elem.set(prim, G);
    ZLOOP {
      const double bSqr = elem.bSqr[z];
      bsq1[z] = bSqr;
      double cd = (bSqr > c.BsqrOverRhoMax * rho[z]) ? 1. : 0.;
      usefloor[z] = std::max(cd, usefloor[z]);
      rho[z] = rho[z] * (1. - cd) + cd * bSqr / c.BsqrOverRhoMax;
      cd = (bSqr > c.BsqrOverUMax * u[z]) ? 1. : 0.;
      usefloor[z] = std::max(cd, usefloor[z]);
      u[z] = u[z] * (1. - cd) + cd * bSqr / c.BsqrOverUMax;
    }
    ZLOOP {
      const double bSqr = bsq1[z];
      const double zero = usefloor[z] * 0.;
      const double trans = std::max(std::min(zero + 1., (bSqr - 0.1 * rho[z]) / rho[z]), zero) *
                           ((usefloor[z] > zero) ? 1. : 0.);
      const double betapar = -elem.bCon[0][z] / bSqr / elem.uCon[0][z];
      double betasqr = betapar * betapar * bSqr;
      const double betasqrmax = 1. - 1. / c.MaxLorentzFactor / c.MaxLorentzFactor;
      betasqr = std::min(betasqr, betasqrmax);
      const double gamma = 1. / std::sqrt(1. - betasqr);
      double ucondr[4];
      for (int m = 0; m < 4; m++) ucondr[m] = gamma * (elem.uCon[m][z] + betapar * elem.bCon[m][z]);
      const double Bcon[4] = {zero, prim.v(P.B1)[z], prim.v(P.B2)[z], prim.v(P.B3)[z]};
      double Bcov[4];
      for (int m = 0; m < 4; m++) {
        Bcov[m] = zero;
        for (int n = 0; n < 4; n++) Bcov[m] += G.gCov[n][m][z] * Bcon[n];
      }
      double udotB = zero, bSqr_fl = zero;
      for (int n = 0; n < 4; n++) {
        udotB += Bcov[n] * elem.uCon[n][z];
        bSqr_fl += Bcov[n] * Bcon[n];
      }
      double bNorm = std::sqrt(bSqr_fl);
      const double bMin = std::sqrt(c.bSqrFloorInFluidElement);
      bNorm = std::max(bNorm, bMin);
      const double wold = rho_pre[z] + u_pre[z] * c.adiabaticIndex;
      const double QdotB = udotB * wold * elem.uCon[0][z];
      const double wnew = rho[z] + u[z] * c.adiabaticIndex;
      const double x = 2. * QdotB / (bNorm * wnew * ucondr[0]);
      const double vpar = x / (ucondr[0] * (1. + std::sqrt(1. + x * x)));
      const double inv = 1. / ucondr[0];
      double vcon[4];
      vcon[0] = zero + 1.;
      for (int m = 1; m < 4; m++) vcon[m] = vpar * Bcon[m] / bNorm + ucondr[m] * inv;
      double vsqr = zero;
      for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) vsqr += G.gCov[m][n][z] * vcon[m] * vcon[n];
      const double cv = (vsqr >= 0. || vsqr < 1. / G.gCon[0][0][z]) ? 1. : 0.;
      vsqr = (1. - cv) * vsqr + cv / G.gCon[0][0][z];
      const double ut = std::sqrt(-1. / vsqr);
      for (int m = 1; m < 4; m++) {
        const double utcon = ut * (vcon[m] - G.gCon[0][m][z] / G.gCon[0][0][z]);
        prim.v(UU + m)[z] = prim.v(UU + m)[z] * (1. - trans) + trans * utcon;
      }
    }
    elem.set(prim, G);
    const double gm2 = c.MaxLorentzFactor * c.MaxLorentzFactor;
    ZLOOP {
      const double lf2 = elem.gammaLF[z] * elem.gammaLF[z];
      if (lf2 > gm2) {
        double mf = std::sqrt(std::max((lf2 - 1.) / (gm2 - 1.), 1.));
        mf = 1. / mf;
        prim.v(U1)[z] *= mf;
        prim.v(U2)[z] *= mf;
        prim.v(U3)[z] *= mf;
      }
    }
    elem.set(prim, G);
    if (c.conduction) {
      ZLOOP {
        const double Qmax = 1.07 * c.ConductionClosureFactor * rho[z] * std::pow(elem.soundSpeed[z], 3.);
        const double lim = std::max(std::fabs(elem.q[z]) / Qmax, 1.);
        prim.v(P.Q)[z] = prim.v(P.Q)[z] / lim;
      }
    }
    if (c.viscosity) {
      ZLOOP {
        const double pr = elem.pressure[z], dP = elem.deltaP[z], bs = elem.bSqr[z];
        const double dPmod = std::max(pr - 2. / 3. * dP, 0.01 * c.bSqrFloorInFluidElement) /
                             std::max(pr + 1. / 3. * dP, c.bSqrFloorInFluidElement);
        const double dPmaxPlus = std::min(1.07 * c.ViscosityClosureFactor * bs * 0.5 * dPmod, 1.49 * pr);
        const double dPmaxMinus = std::max(-1.07 * c.ViscosityClosureFactor * bs, -2.99 * pr);
        const double cd = (dP > 0.) ? 1. : 0.;
        prim.v(P.DP)[z] = prim.v(P.DP)[z] * (cd / std::max(dP / dPmaxPlus, 1.) +
                                             (1. - cd) / std::max(dP / dPmaxMinus, 1.));
      }
    }
    if (c.conduction || c.viscosity) elem.set(prim, G);
  }

  /* NaN reset of fullStepDiagnostics (torus/problem.cpp:725-744) */
  void nanReset(Grid& prim) {
    long bad = 0;
    for (long z = 0; z < L.Z; z++) {
      if (!L.interior(z)) continue;
      for (int v = 0; v < P.dof; v++) if (std::isnan(prim.v(v)[z])) { bad++; break; }
    }
    if (bad == 0) return;
    for (long z = 0; z < L.Z; z++) {
      bool isn = false;
      for (int v = 0; v < P.dof; v++) isn |= std::isnan(prim.v(v)[z]);
      if (isn) for (int v = 0; v < P.dof; v++) prim.v(v)[z] = 0.;
    }
  }

  void halfStepDiagnostics() {
    if (torus()) applyFloor(primHalfStep, elemHalfStep);
  }
  void fullStepDiagnostics() {
    if (torus()) {
      nanReset(primOld);
      applyFloor(primOld, elemOld);
    } else if (P.c.elemOldFromFullStep) {
      /* linear_modes/problem.cpp:287 */
      elemOld.set(primOld, geomCenter);
    }
  }
  /* the tail of the torus initialConditions (problem.cpp:525-540) */
  void problemInit() {
    if (!torus()) return;
    applyFloor(primOld, elemOld);
    fullStepDiagnostics();
  }

  /* residual.cpp:3-180 */
  void computeResidual(const Grid& primGuess, Grid& res) {
    const orc_config& c = P.c;
    const long Z = L.Z;
    const int nf = P.nf;
    elem.set(primGuess, geomCenter);
    elem.computeFluxes(0, cons);
    const bool half = (currentStep == HALF_STEP);
    Elem& ref = half ? elemOld : elemHalfStep;
    elem.computeImplicitSources(sourcesImplicit, ref.tau);
    ref.computeTimeDerivSources(elemOld, elem, half ? dt / 2 : dt, sourcesTimeDer);
    const double dtp = half ? (dt / 2.) : dt;
    for (int var = 0; var < nf; var++) {
      const double* U = cons.v(var); const double* Uo = consOld.v(var);
      const double* D = divFluxes.v(var); const double* Se = sourcesExplicit.v(var);
      const double* Sio = sourcesImplicitOld.v(var); const double* Si = sourcesImplicit.v(var);
      const double* St = sourcesTimeDer.v(var);
      double* r = res.v(var);
      ZLOOP { r[z] = (U[z] - Uo[z]) / dtp + D[z] + Se[z] + 0.5 * (Sio[z] + Si[z]) + St[z]; }
    }
    if (c.conduction) {
      double* r = res.v(P.Q);
      if (c.highOrderTermsConduction) {
        ZLOOP { r[z] *= ref.temperature[z] * std::sqrt(ref.rho[z] * ref.chi_emhd[z] * ref.tau[z]); }
      } else {
        ZLOOP { r[z] *= ref.tau[z]; }
      }
    }
    if (c.viscosity) {
      double* r = res.v(P.DP);
      if (c.highOrderTermsViscosity) {
        ZLOOP { r[z] *= std::sqrt(ref.rho[z] * ref.nu_emhd[z] * ref.temperature[z] * ref.tau[z]); }
      } else {
        ZLOOP { r[z] *= ref.tau[z]; }
      }
    }
    for (int var = 0; var < nf; var++) {
      double* r = res.v(var);
      ZLOOP { r[z] *= residualMask[z]; }
    }
  }

  /* FD Jacobian columns (solve.cpp:82-109): jac[z][i][j] = dR_i/dP_j */
  void jacobianFD(Grid& primGuess, std::vector<double>& jac) {
    const long Z = L.Z;
    const int nf = P.nf;
    jac.assign((size_t)Z * nf * nf, 0.);
    for (int var = 0; var < nf; var++) std::memcpy(primGuessPlusEps.v(var), primGuess.v(var), sizeof(double) * Z);
    for (int row = 0; row < nf; row++) {
      const double eps = P.c.JacobianAssembleEpsilon;
      double* pe = primGuessPlusEps.v(row);
      const double* pg = primGuess.v(row);
      ZLOOP {
        double small = (std::fabs(pg[z]) < .5 * eps) ? 1. : 0.;
        pe[z] = pg[z] + eps * pg[z] * (1. - small) + small * eps;
      }
      computeResidual(primGuessPlusEps, residualPlusEps);
      for (int col = 0; col < nf; col++) {
        const double* rp = residualPlusEps.v(col);
        const double* r0 = residual.v(col);
        ZLOOP { jac[((size_t)z * nf + col) * nf + row] = (rp[z] - r0[z]) / (pe[z] - pg[z]); }
      }
      std::memcpy(pe, pg, sizeof(double) * Z);
    }
  }

  double zoneL2(const Grid& r, long z) const {
    double s = 0.;
    for (int v = 0; v < P.nf; v++) s += r.v(v)[z] * r.v(v)[z];
    return s;
  }

  /* solve.cpp:3-201 (global convergence test, all zones updated) */
  int solve(Grid& primGuess) {
    const orc_config& c = P.c;
    const long Z = L.Z;
    const int nf = P.nf;
    std::vector<double> jac, dP((size_t)Z * nf, 0.), l2(Z, 0.), l2first(Z, 0.), step(Z, 1.);
    int it = 0;
    for (; it < c.maxNonLinearIter; it++) {
      ZLOOP {
        primGuess.v(RHO)[z] = std::max(primGuess.v(RHO)[z], c.rhoFloorInFluidElement);
        primGuess.v(UU)[z] = std::max(primGuess.v(UU)[z], c.uFloorInFluidElement);
      }
      computeResidual(primGuess, residual);
      long notConverged = 0;
      for (long z = 0; z < Z; z++) {
        if (!L.interior(z)) continue;
        l2[z] = zoneL2(residual, z);
        if (it == 0) l2first[z] = l2[z];
        double tol = std::max(c.nonlinearsolve_atol, c.nonlinearsolve_rtol * c.nonlinearsolve_rtol * l2first[z]);
        if (l2[z] > tol) notConverged++;
      }
      if (notConverged == 0) break;
      jacobianFD(primGuess, jac);
      /* batched dense solve (solve.cpp:116-128, :203-230), interior zones */
      ZLOOP {
        if (!L.interior(z)) { for (int v = 0; v < nf; v++) dP[z * nf + v] = 0.; continue; }
        double A[64], b[8], x[8];
        std::memcpy(A, &jac[(size_t)z * nf * nf], sizeof(double) * nf * nf);
        for (int v = 0; v < nf; v++) b[v] = -residual.v(v)[z];
        solveDense(nf, A, b, x);
        for (int v = 0; v < nf; v++) dP[z * nf + v] = x[v];
      }
      /* quadratic backtracking (solve.cpp:130-191) */
      std::vector<double> f0(Z), fPrime0(Z);
      for (long z = 0; z < Z; z++) { f0[z] = 0.5 * l2[z]; fPrime0[z] = -2. * f0[z]; step[z] = 1.; }
      for (int ls = 0; ls < c.maxLineSearchIters; ls++) {
        for (int v = 0; v < nf; v++) {
          double* t = primGuessLineSearchTrial.v(v); const double* pg = primGuess.v(v);
          ZLOOP { t[z] = pg[z] + step[z] * dP[z * nf + v]; }
        }
        computeResidual(primGuessLineSearchTrial, residual);
        const double alpha = 1e-4, EPS = c.linesearchfloor;
        long cnt = 0;
        for (long z = 0; z < Z; z++) {
          if (!L.interior(z)) continue;
          double f1 = 0.5 * zoneL2(residual, z);
          double lam = step[z];
          double cond = (f1 > (f0[z] * (1. - alpha * lam) + EPS)) ? 1. : 0.;
          double denom = (f1 - f0[z] - fPrime0[z] * lam) * cond + (1. - cond);
          double next = -fPrime0[z] * lam * lam / denom / 2.;
          step[z] = lam * (1. - cond) + cond * next;
          if (cond > 0) cnt++;
        }
        if (cnt == 0) break;
      }
      for (int v = 0; v < nf; v++) {
        double* pg = primGuess.v(v);
        ZLOOP { pg[z] = pg[z] + step[z] * dP[z * nf + v]; }
      }
    }
    return it;
  }

  void copyVars(const Grid& a, Grid& b, int nv) {
    std::memcpy(b.d.data(), a.d.data(), sizeof(double) * (size_t)nv * L.Z);
  }

  /* timestep.cpp:336-400 (elemOld holds whatever state it was last set to) */
  void computeDt() {
    const long Z = L.Z;
    Arr mn(Z), mx(Z), acc(Z, 0.);
    for (int d = 0; d < L.dim; d++) {
      elemOld.computeMinMaxCharSpeeds(d, mn.data(), mx.data());
      ZLOOP {
        double a = mn[z] / dX[d], b = mx[z] / dX[d];
        double m = std::max(b, std::fabs(a));
        acc[z] = (d == 0) ? m : acc[z] + m;
      }
    }
    double maxInvDt = -INFINITY;
    for (long z = 0; z < Z; z++) maxInvDt = std::max(maxInvDt, acc[z]);
    double newDt = P.c.CourantFactor / maxInvDt;
    if (newDt > P.c.maxDtIncrement * dt) newDt = P.c.maxDtIncrement * dt;
    dt = newDt;
  }

  void stageSetup(int stage) {
    const orc_config& c = P.c;
    const long Z = L.Z;
    const int nf = P.nf, dof = P.dof;
    currentStep = stage;
    if (stage == HALF_STEP) {
      applyBoundaryConditions(primOld.d.data(), dof);
      setProblemSpecificBCs(primOld);
      elemOld.set(primOld, geomCenter);
      elemOld.computeFluxes(0, consOld);
      elemOld.computeExplicitSources(dX, sourcesExplicit);
      elemOld.computeImplicitSources(sourcesImplicitOld, elemOld.tau);
      computeDivOfFluxes(primOld);
      for (int var = 0; var < nf; var++) std::memcpy(prim.v(var), primOld.v(var), sizeof(double) * Z);
    } else {
      applyBoundaryConditions(primHalfStep.d.data(), dof);
      setProblemSpecificBCs(primHalfStep);
      elemHalfStep.set(primHalfStep, geomCenter);
      elemHalfStep.computeExplicitSources(dX, sourcesExplicit);
      elemOld.computeImplicitSources(sourcesImplicitOld, elemHalfStep.tau);
      computeDivOfFluxes(primHalfStep);
    }
    const double fac = (stage == HALF_STEP) ? 0.5 * dt : dt;
    for (int b = 0; b < 3; b++) {
      const int v = P.B1 + b;
      const double* co = consOld.v(v); const double* D = divFluxes.v(v);
      double* cn = cons.v(v); double* pr = prim.v(v);
      ZLOOP { cn[z] = co[z] - fac * D[z]; pr[z] = cn[z] / geomCenter.g[z]; }
    }
    for (int b = 0; b < 3; b++) {
      std::memcpy(primGuessPlusEps.v(P.B1 + b), prim.v(P.B1 + b), sizeof(double) * Z);
      std::memcpy(primGuessLineSearchTrial.v(P.B1 + b), prim.v(P.B1 + b), sizeof(double) * Z);
    }
    (void)c;
  }

  /* timestep.cpp:3-334 */
  void timeStep() {
    const int dof = P.dof;
    computeDt();
    stageSetup(HALF_STEP);
    lastIters[0] = solve(prim);
    copyVars(prim, primHalfStep, dof);
    communicate(primHalfStep.d.data(), dof);
    halfStepDiagnostics();
    stageSetup(FULL_STEP);
    lastIters[1] = solve(prim);
    copyVars(prim, primOld, dof);
    communicate(primOld.d.data(), dof);
    time += dt;
    fullStepDiagnostics();
  }
};

}  // namespace orc

using namespace orc;

struct orc_handle { Stepper s; };

extern "C" {

int orc_create(const orc_config* cfg, orc_handle** out) {
  if (!cfg || !out) return -1;
  if (cfg->dim < 1 || cfg->dim > 3 || cfg->numGhost < 3) return -2;
  orc_handle* h = new orc_handle();
  h->s.init(*cfg);
  *out = h;
  return 0;
}
void orc_destroy(orc_handle* h) { delete h; }
int orc_num_vars(const orc_handle* h, int* dof, int* nf) { *dof = h->s.P.dof; *nf = h->s.P.nf; return 0; }
int orc_dims(const orc_handle* h, int* a, int* b, int* c) { *a = h->s.L.N1T; *b = h->s.L.N2T; *c = h->s.L.N3T; return 0; }

static Grid* pick(orc_handle* h, int which) {
  if (which == ORC_PRIM_OLD) return &h->s.primOld;
  if (which == ORC_PRIM) return &h->s.prim;
  if (which == ORC_PRIM_HALF) return &h->s.primHalfStep;
  return nullptr;
}
int orc_set_prims(orc_handle* h, int which, const double* src) {
  Grid* g = pick(h, which); if (!g) return -1;
  std::memcpy(g->d.data(), src, sizeof(double) * g->d.size()); return 0;
}
int orc_get_prims(const orc_handle* h, int which, double* dst) {
  Grid* g = pick(const_cast<orc_handle*>(h), which); if (!g) return -1;
  std::memcpy(dst, g->d.data(), sizeof(double) * g->d.size()); return 0;
}
int orc_time_step(orc_handle* h, int n) { for (int i = 0; i < n; i++) h->s.timeStep(); return 0; }
int orc_get_time(const orc_handle* h, double* t, double* dt) { *t = h->s.time; *dt = h->s.dt; return 0; }
int orc_set_time(orc_handle* h, double t, double dt) { h->s.time = t; h->s.dt = dt; return 0; }
int orc_compute_dt(orc_handle* h) { h->s.computeDt(); return 0; }
int orc_apply_boundaries(const orc_handle* h, double* prim, int nv) {
  h->s.communicate(prim, nv);
  h->s.applyBoundaryConditions(prim, nv);
  return 0;
}
int orc_geometry(const orc_handle* h, int location, double* out, double* gamma, double* xc) {
  const Stepper& s = h->s;
  const Geom* g = nullptr;
  switch (location) {
    case CENTER: g = &s.geomCenter; break; case LEFT: g = &s.geomLeft; break;
    case RIGHT: g = &s.geomRight; break; case TOP: g = &s.geomTop; break;
    case BOTTOM: g = &s.geomBottom; break; default: return -1;
  }
  const long Z = s.L.Z;
  if (out) {
    for (int m = 0; m < 4; m++) for (int n = 0; n < 4; n++) {
      std::memcpy(out + (size_t)(m * 4 + n) * Z, g->gCov[m][n].data(), sizeof(double) * Z);
      std::memcpy(out + (size_t)(16 + m * 4 + n) * Z, g->gCon[m][n].data(), sizeof(double) * Z);
    }
    std::memcpy(out + (size_t)32 * Z, g->g.data(), sizeof(double) * Z);
    std::memcpy(out + (size_t)33 * Z, g->alpha.data(), sizeof(double) * Z);
  }
  if (gamma && g->hasGamma)
    for (int a = 0; a < 4; a++) for (int b = 0; b < 4; b++) for (int c = 0; c < 4; c++)
      std::memcpy(gamma + (size_t)(a * 16 + b * 4 + c) * Z, g->gamma[a][b][c].data(), sizeof(double) * Z);
  if (xc) {
    std::memcpy(xc, g->x[0].data(), sizeof(double) * Z);
    std::memcpy(xc + Z, g->x[1].data(), sizeof(double) * Z);
    std::memcpy(xc + 2 * Z, g->dyn.data(), sizeof(double) * Z);
    std::memcpy(xc + 3 * Z, g->minRho.data(), sizeof(double) * Z);
    std::memcpy(xc + 4 * Z, g->minU.data(), sizeof(double) * Z);
  }
  return 0;
}
int orc_div_fluxes(orc_handle* h, const double* prim, double* divF, double* fluxes, double* emf) {
  Stepper& s = h->s;
  const long Z = s.L.Z; const int dof = s.P.dof;
  Grid p; p.init(dof, Z); std::memcpy(p.d.data(), prim, sizeof(double) * p.d.size());
  s.computeDivOfFluxes(p);
  if (divF) std::memcpy(divF, s.divFluxes.d.data(), sizeof(double) * s.divFluxes.d.size());
  if (fluxes) {
    std::memcpy(fluxes, s.fluxesX1.d.data(), sizeof(double) * dof * Z);
    std::memcpy(fluxes + (size_t)dof * Z, s.fluxesX2.d.data(), sizeof(double) * dof * Z);
    std::memcpy(fluxes + (size_t)2 * dof * Z, s.fluxesX3.d.data(), sizeof(double) * dof * Z);
  }
  if (emf) {
    std::memcpy(emf, s.emfX1.data(), sizeof(double) * Z);
    std::memcpy(emf + Z, s.emfX2.data(), sizeof(double) * Z);
    std::memcpy(emf + 2 * Z, s.emfX3.data(), sizeof(double) * Z);
  }
  return 0;
}
int orc_reconstruct(orc_handle* h, const double* prim, int dir, double* pl, double* pr) {
  Stepper& s = h->s;
  const long Z = s.L.Z; const int dof = s.P.dof;
  Grid p; p.init(dof, Z); std::memcpy(p.d.data(), prim, sizeof(double) * p.d.size());
  s.R.reconstruct(p, dir, s.primLeft, s.primRight);
  std::memcpy(pl, s.primLeft.d.data(), sizeof(double) * dof * Z);
  std::memcpy(pr, s.primRight.d.data(), sizeof(double) * dof * Z);
  return 0;
}
int orc_conserved(orc_handle* h, const double* prim, double* cons) {
  Stepper& s = h->s;
  const long Z = s.L.Z; const int dof = s.P.dof;
  Grid p; p.init(dof, Z); std::memcpy(p.d.data(), prim, sizeof(double) * p.d.size());
  Elem e; e.alloc(s.L, s.P); e.set(p, s.geomCenter);
  Grid c; c.init(dof, Z); e.computeFluxes(0, c);
  std::memcpy(cons, c.d.data(), sizeof(double) * c.d.size());
  return 0;
}
/* fluidElement::set then computeFluxes(dir) (physics.cpp:53-217) at the
 * zone centres, dir = 0 (the conserved variables), 1, 2, 3 */
int orc_element_fluxes(orc_handle* h, const double* prim, int dir, double* out) {
  if (dir < 0 || dir > 3) return -1;
  Stepper& s = h->s;
  const long Z = s.L.Z; const int dof = s.P.dof;
  Grid p; p.init(dof, Z); std::memcpy(p.d.data(), prim, sizeof(double) * p.d.size());
  Elem e; e.alloc(s.L, s.P); e.set(p, s.geomCenter);
  Grid f; f.init(dof, Z); e.computeFluxes(dir, f);
  std::memcpy(out, f.d.data(), sizeof(double) * f.d.size());
  return 0;
}
/* the stage grids stageSetup left (timestep.cpp:26-79 / 180-237):
 * 0 consOld (dof rows), 1 divFluxes and 2 sourcesExplicit (the nf fluid rows) */
int orc_get_stage_grid(const orc_handle* h, int which, double* out) {
  const Stepper& s = h->s;
  const Grid* g = which == 0 ? &s.consOld : which == 1 ? &s.divFluxes : which == 2 ? &s.sourcesExplicit : nullptr;
  if (!g) return -1;
  const int rows = which == 0 ? s.P.dof : s.P.nf;
  std::memcpy(out, g->d.data(), sizeof(double) * (size_t)rows * s.L.Z);
  return 0;
}
/* computeDivB (constrainedtransport.cpp:85-110), 2D */
int orc_compute_divb(orc_handle* h, const double* prim, double* divB) {
  Stepper& s = h->s;
  const Layout& L = s.L;
  const long Z = L.Z;
  for (long z = 0; z < Z; z++) divB[z] = 0.;
  if (L.dim != 2) return 0;
  std::vector<double> gB1(Z), gB2(Z), a(Z), b(Z), c(Z), d(Z), e(Z), f(Z);
  const double* B1 = prim + (long)s.P.B1 * Z;
  const double* B2 = prim + (long)s.P.B2 * Z;
  for (long z = 0; z < Z; z++) { gB1[z] = s.geomCenter.g[z] * B1[z]; gB2[z] = s.geomCenter.g[z] * B2[z]; }
  shift(L, gB1.data(), 0, 1, 0, a.data());
  shift(L, gB1.data(), 1, 0, 0, b.data());
  shift(L, gB1.data(), 1, 1, 0, c.data());
  shift(L, gB2.data(), 1, 0, 0, d.data());
  shift(L, gB2.data(), 0, 1, 0, e.data());
  shift(L, gB2.data(), 1, 1, 0, f.data());
  for (long z = 0; z < Z; z++)
    divB[z] = (gB1[z] + a[z] - b[z] - c[z]) / (2. * s.dX[0]) + (gB2[z] + d[z] - e[z] - f[z]) / (2. * s.dX[1]);
  return 0;
}
/* The torus observers (ObserversTorus.hpp:6-253, called from
 * fullStepDiagnostics, torus/problem.cpp:754-778) on primOld with its
 * element at the zone centres; the integrands in the reference's operation
 * order, summed zone by zone in index order.  out: baryon mass, magnetic
 * energy, thermal energy, rho max, beta min, Mdot in (i = 3), Mdot out
 * (i = N1 + 2), unbound and relativistic unbound Mdot out. */
int orc_torus_observers(orc_handle* h, double* out) {
  Stepper& s = h->s;
  const Layout& L = s.L;
  const long Z = L.Z;
  const Geom& G = s.geomCenter;
  Elem e; e.alloc(L, s.P); e.set(s.primOld, G);
  double volElem = s.dX[0];
  if (L.dim > 1) volElem *= s.dX[1];
  if (L.dim > 2) volElem *= s.dX[2];
  const double* rho = s.primOld.v(RHO);
  const double* u = s.primOld.v(UU);
  double mass = 0., emag = 0., eth = 0., rhoMax = -INFINITY, betaMin = INFINITY;
  double mIn = 0., mOut = 0., unb = 0., rel = 0.;
  for (long z = 0; z < Z; z++) {
    if (!L.interior(z)) continue;
    int i, j, k; L.ijk(z, i, j, k);
    mass += rho[z] * volElem * G.g[z] * e.gammaLF[z] / G.alpha[z];
    emag += volElem * e.bSqr[z] * G.g[z] * e.gammaLF[z] / G.alpha[z];
    eth += volElem * u[z] * G.g[z] * e.gammaLF[z] / G.alpha[z];
    rhoMax = std::max(rhoMax, rho[z]);
    betaMin = std::min(betaMin, 2. * (e.pressure[z] + 1.e-13) / (e.bSqr[z] + 1.e-18));
    const double mi = rho[z] * volElem * G.g[z] * e.uCon[1][z];
    if (i == 3) mIn += mi;
    if (i == L.N1 + 2) {
      mOut += mi;
      const double bern = (1. + u[z] / rho[z] * s.P.c.adiabaticIndex) * e.uCov[0][z];
      const double ub = mi * ((bern < -1.) ? 1. : 0.);
      unb += ub;
      rel += ub * ((e.gammaLF[z] > 2.) ? 1. : 0.);
    }
  }
  const double r[9] = {mass, emag, eth, rhoMax, betaMin, mIn, mOut, unb, rel};
  for (int v = 0; v < 9; v++) out[v] = r[v];
  return 0;
}
int orc_char_speeds(orc_handle* h, const double* prim, int dir, double* mn, double* mx) {
  Stepper& s = h->s;
  const long Z = s.L.Z; const int dof = s.P.dof;
  Grid p; p.init(dof, Z); std::memcpy(p.d.data(), prim, sizeof(double) * p.d.size());
  Elem e; e.alloc(s.L, s.P); e.set(p, s.geomCenter);
  e.computeMinMaxCharSpeeds(dir, mn, mx);
  return 0;
}
int orc_stage_setup(orc_handle* h, int stage) { h->s.stageSetup(stage); return 0; }
int orc_residual(orc_handle* h, const double* pg, double* res) {
  Stepper& s = h->s;
  const long Z = s.L.Z; const int dof = s.P.dof, nf = s.P.nf;
  Grid p; p.init(dof, Z); std::memcpy(p.d.data(), pg, sizeof(double) * p.d.size());
  s.computeResidual(p, s.residual);
  std::memcpy(res, s.residual.d.data(), sizeof(double) * nf * Z);
  return 0;
}
int orc_jacobian_fd(orc_handle* h, const double* pg, double* jac) {
  Stepper& s = h->s;
  const long Z = s.L.Z; const int dof = s.P.dof, nf = s.P.nf;
  Grid p; p.init(dof, Z); std::memcpy(p.d.data(), pg, sizeof(double) * p.d.size());
  s.computeResidual(p, s.residual);
  std::vector<double> J;
  s.jacobianFD(p, J);
  std::memcpy(jac, J.data(), sizeof(double) * Z * nf * nf);
  return 0;
}
int orc_newton(orc_handle* h, int* iters) {
  int it = h->s.solve(h->s.prim);
  if (iters) *iters = it;
  return 0;
}
int orc_batch_solve(int n, int batch, const double* A, const double* b, double* x) {
  if (n < 1 || n > 8) return -1;
  for (int z = 0; z < batch; z++) {
    double a[64], bb[8];
    std::memcpy(a, A + (size_t)z * n * n, sizeof(double) * n * n);
    std::memcpy(bb, b + (size_t)z * n, sizeof(double) * n);
    solveDense(n, a, bb, x + (size_t)z * n);
  }
  return 0;
}
int orc_last_newton_stats(const orc_handle* h, int* a, int* b) { *a = h->s.lastIters[0]; *b = h->s.lastIters[1]; return 0; }
int orc_problem_init(orc_handle* h) { h->s.problemInit(); return 0; }
int orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#endif
  (void)n; return 0;
}

}  // extern "C"
