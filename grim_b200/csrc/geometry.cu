// geometry.cu -- metric, inverse metric, sqrt(-g), lapse and Christoffel
// symbols per zone and location, computed once at handle creation
// (src/geometry/geometry.cpp:4-680, CoordinateChangeFunctionsArray.hpp).
//
// Stored layout per location: 39 x Z doubles, SoA:
//   [0,16) gCov[mu][nu], [16,32) gCon[mu][nu], 32 g, 33 alpha, 34 x1, 35 x2,
//   36 x1^1.5, 37 RhoFloorAmpl x1^RhoFloorSlope, 38 UFloorAmpl x1^UFloorSlope
// and for the zone centre 64 x Z Christoffels gammaUpDownDown[mu][nu][la].
// Compiled without FMA contraction like the parity kernels.
#include "common.cuh"

namespace grim {

struct GeoParams {
  int metric, derefine, cylindrify;
  double a, hSlope, X1Start, X1cyl, X2cyl;
  double rhoFloorAmpl, rhoFloorSlope, uFloorAmpl, uFloorSlope;
};

// CoordinateChangeFunctionsArray.hpp:4-16
__device__ double GammieRadius(double X1) { return exp(X1); }
__device__ double GammieTheta(const GeoParams& p, double X2) {
  return M_PI * X2 + 0.5 * (1 - p.hSlope) * sin(2. * M_PI * X2);
}
// :22-46
__device__ double ThetaNoCyl(const GeoParams& p, double X1, double X2) {
  if (p.derefine) {
    double cTh0 = cos(M_PI * X2);
    double cTh1 = cos(GammieTheta(p, X2));
    double cTh = cTh1 + exp(p.X1Start) / exp(X1) * (cTh0 - cTh1);
    return acos(cTh);
  }
  return GammieTheta(p, X2);
}
// :83-126
__device__ double Fangle(double x) {
  double c1 = (x <= -1) ? 1. : 0.;
  double c2 = (x >= 1) ? 1. : 0.;
  return c2 * x + (c1 - 1) * (c2 - 1) *
                      (x + 1. + (-140 * sin(((x + 1) * M_PI) / 2.) + (10 * sin(((x + 1) * 3 * M_PI) / 2.)) / 3. +
                                 (2 * sin(((x + 1) * 5 * M_PI) / 2.)) / 5.) /
                                    (64. * M_PI)) / 2.;
}
__device__ double limlin(double x, double x0, double dx, double y0) { return y0 - dx * Fangle((x - x0) * (-1.) / dx); }
__device__ double mins(double f1, double f2, double df) { return limlin(f1, f2, df, f2); }
__device__ double maxs(double f1, double f2, double df) { return mins(-f1, -f2, df) * (-1.); }
__device__ double minmaxs(double f1, double f2, double df, double dir) {
  double cond = (dir >= 0) ? 1. : 0.;
  return cond * maxs(f1, f2, df) + (1 - cond) * mins(f1, f2, df);
}
// :129-195
__device__ double sinth0(const GeoParams& p, const double* X0, const double* X) {
  return GammieRadius(X0[0]) * sin(ThetaNoCyl(p, X0[0], X0[1])) / GammieRadius(X[0]);
}
__device__ double sinth1in(const GeoParams& p, const double* X0, const double* X) {
  return GammieRadius(X0[0]) * sin(ThetaNoCyl(p, X0[0], X[1])) / GammieRadius(X[0]);
}
__device__ double th2in(const GeoParams& p, const double* X0, const double* X) {
  double th0 = asin(sinth0(p, X0, X));
  double a = ThetaNoCyl(p, X[0], X[1]);
  double b = ThetaNoCyl(p, X[0], X0[1]);
  double m = ThetaNoCyl(p, X[0], 0.5);
  return (a - b) / (m - b) * (m - th0) + th0;
}
__device__ double func1(const GeoParams& p, const double* X) { return sin(ThetaNoCyl(p, X[0], X[1])); }
__device__ double func2(const GeoParams& p, const double* X0, const double* X) {
  double Xca[3] = {X[0], 0., X[2]};
  double sth1in = sinth1in(p, X0, X);
  double sth2in = sin(th2in(p, X0, X));
  double sth1inaxis = sinth1in(p, X0, Xca);
  double sth2inaxis = sin(th2in(p, X0, Xca));
  return minmaxs(sth1in, sth2in, fabs(sth2inaxis - sth1inaxis) + 1.e-20, X[0] - X0[0]);
}
// geometry.cpp:510-629
__device__ void XtoX(const GeoParams& p, const double* X, double* x) {
  if (p.metric == GRIM_MINKOWSKI) { x[0] = X[0]; x[1] = X[1]; x[2] = X[2]; return; }
  x[0] = GammieRadius(X[0]);
  x[1] = ThetaNoCyl(p, X[0], X[1]);
  x[2] = X[2];
  if (p.cylindrify) {
    double Xg[3] = {X[0], X[1], X[2]};
    double xG[3] = {x[0], x[1], x[2]};
    double isM = (Xg[1] > 0.5) ? 1. : 0.;
    Xg[1] = (1 - isM) * Xg[1] + isM * (1. - Xg[1]);
    xG[1] = (1 - isM) * xG[1] + isM * (M_PI - xG[1]);
    double isG = (Xg[1] < 0.) ? 1. : 0.;
    Xg[1] = (1 - isG) * Xg[1] + isG * (-(1.0) * Xg[1]);
    xG[1] = (1 - isG) * xG[1] + isG * (-(1.0) * xG[1]);
    double X0[3] = {p.X1cyl, p.X2cyl, 0.};
    double R_cyl = GammieRadius(X0[0]);
    double X1_tr = log(0.5 * (R_cyl + exp(p.X1Start)));
    double Xtr[3] = {X1_tr, Xg[1], Xg[2]};
    double f1 = func1(p, Xg);
    double f2 = func2(p, X0, Xg);
    double dftr = func2(p, X0, Xtr) - func1(p, Xtr);
    double sinth = maxs(xG[0] * f1, xG[0] * f2, GammieRadius(Xtr[0]) * fabs(dftr) + 1.e-20) / xG[0];
    double th = asin(sinth);
    th = th * (1 - isG * 2);
    x[0] = xG[0];
    x[1] = isM * (M_PI - th) + (1 - isM) * th;
    x[2] = xG[2];
  }
}
// geometry.cpp:255-424
__device__ void gcov_at(const GeoParams& p, const double* X, double g[4][4]) {
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) g[m][n] = 0.;
  if (p.metric == GRIM_MINKOWSKI) {
    g[0][0] = -1.; g[1][1] = 1.; g[2][2] = 1.; g[3][3] = 1.;
    return;
  }
  const double eps = 1.e-5, a = p.a, h = p.hSlope;
  double x[3];
  XtoX(p, X, x);
  double r = x[0], theta = x[1];
  double dr_dX1 = r, dr_dX2 = 0.;
  double dtheta_dX2 = M_PI + M_PI * (1 - h) * cos(2 * M_PI * X[1]);
  double dtheta_dX1 = 0.;
  if (p.cylindrify) {
    double Xp[3] = {X[0] + eps, X[1], X[2]}, Xm[3] = {X[0] - eps, X[1], X[2]};
    double xp[3], xm[3];
    XtoX(p, Xp, xp);
    XtoX(p, Xm, xm);
    dr_dX1 = (xp[0] - xm[0]) / (2. * eps);
    dtheta_dX1 = (xp[1] - xm[1]) / (2. * eps);
    double Yp[3] = {X[0], X[1] + eps, X[2]}, Ym[3] = {X[0], X[1] - eps, X[2]};
    XtoX(p, Yp, xp);
    XtoX(p, Ym, xm);
    dr_dX2 = (xp[0] - xm[0]) / (2. * eps);
    dtheta_dX2 = (xp[1] - xm[1]) / (2. * eps);
  }
  double ac = a * cos(theta);
  double sigma = r * r + ac * ac;
  double st = sin(theta), s2 = st * st;
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
// geometry.cpp:123-253
__device__ void det_inverse(const double G[4][4], double& D, double C[4][4]) {
#define g(a, b) G[a][b]
  D = g(0,0)*g(1,1)*g(2,2)*g(3,3) + g(0,0)*g(1,2)*g(2,3)*g(3,1)
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
           - g(1,1)*g(2,3)*g(3,2) - g(1,2)*g(2,1)*g(3,3) - g(1,3)*g(2,2)*g(3,1)) / D;
  C[0][1] = (g(0,1)*g(2,3)*g(3,2) + g(0,2)*g(2,1)*g(3,3) + g(0,3)*g(2,2)*g(3,1)
           - g(0,1)*g(2,2)*g(3,3) - g(0,2)*g(2,3)*g(3,1) - g(0,3)*g(2,1)*g(3,2)) / D;
  C[0][2] = (g(0,1)*g(1,2)*g(3,3) + g(0,2)*g(1,3)*g(3,1) + g(0,3)*g(1,1)*g(3,2)
           - g(0,1)*g(1,3)*g(3,2) - g(0,2)*g(1,1)*g(3,3) - g(0,3)*g(1,2)*g(3,1)) / D;
  C[0][3] = (g(0,1)*g(1,3)*g(2,2) + g(0,2)*g(1,1)*g(2,3) + g(0,3)*g(1,2)*g(2,1)
           - g(0,1)*g(1,2)*g(2,3) - g(0,2)*g(1,3)*g(2,1) - g(0,3)*g(1,1)*g(2,2)) / D;
  C[1][0] = C[0][1];
  C[1][1] = (g(0,0)*g(2,2)*g(3,3) + g(0,2)*g(2,3)*g(3,0) + g(0,3)*g(2,0)*g(3,2)
           - g(0,0)*g(2,3)*g(3,2) - g(0,2)*g(2,0)*g(3,3) - g(0,3)*g(2,2)*g(3,0)) / D;
  C[1][2] = (g(0,0)*g(1,3)*g(3,2) + g(0,2)*g(1,0)*g(3,3) + g(0,3)*g(1,2)*g(3,0)
           - g(0,0)*g(1,2)*g(3,3) - g(0,2)*g(1,3)*g(3,0) - g(0,3)*g(1,0)*g(3,2)) / D;
  C[1][3] = (g(0,0)*g(1,2)*g(2,3) + g(0,2)*g(1,3)*g(2,0) + g(0,3)*g(1,0)*g(2,2)
           - g(0,0)*g(1,3)*g(2,2) - g(0,2)*g(1,0)*g(2,3) - g(0,3)*g(1,2)*g(2,0)) / D;
  C[2][0] = C[0][2];
  C[2][1] = C[1][2];
  C[2][2] = (g(0,0)*g(1,1)*g(3,3) + g(0,1)*g(1,3)*g(3,0) + g(0,3)*g(1,0)*g(3,1)
           - g(0,0)*g(1,3)*g(3,1) - g(0,1)*g(1,0)*g(3,3) - g(0,3)*g(1,1)*g(3,0)) / D;
  C[2][3] = (g(0,0)*g(1,3)*g(2,1) + g(0,1)*g(1,0)*g(2,3) + g(0,3)*g(1,1)*g(2,0)
           - g(0,0)*g(1,1)*g(2,3) - g(0,1)*g(1,3)*g(2,0) - g(0,3)*g(1,0)*g(2,1)) / D;
  C[3][0] = C[0][3];
  C[3][1] = C[1][3];
  C[3][2] = C[2][3];
  C[3][3] = (g(0,0)*g(1,1)*g(2,2) + g(0,1)*g(1,2)*g(2,0) + g(0,2)*g(1,0)*g(2,1)
           - g(0,0)*g(1,2)*g(2,1) - g(0,1)*g(1,0)*g(2,2) - g(0,2)*g(1,1)*g(2,0)) / D;
#undef g
}

// coordinatesGrid::setXCoords (grid.cpp:168-249) offsets per location
__global__ void k_geometry(DevCfg c, GeoParams p, double o1, double o2, double* __restrict__ out,
                           double* __restrict__ gamma) {
  // one (i, j) plane: the maps and the metric do not depend on X3
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.GZ) return;
  const int i = (int)(z % c.N1T), j = (int)(z / c.N1T), k = c.g3;
  const long long Z = c.GZ;
  double X[3];
  X[0] = c.X1Start + ((double)(i - c.g1) + o1) * c.dX[0];
  X[1] = c.X2Start + ((double)(j - c.g2) + o2) * c.dX[1];
  X[2] = c.X3Start + ((double)(k - c.g3) + 0.5) * c.dX[2];
  double x[3];
  XtoX(p, X, x);
  double G[4][4], C[4][4], D;
  gcov_at(p, X, G);
  det_inverse(G, D, C);
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) {
      out[(long long)(m * 4 + n) * Z + z] = G[m][n];
      out[(long long)(16 + m * 4 + n) * Z + z] = C[m][n];
    }
  out[32LL * Z + z] = sqrt(-D);
  out[33LL * Z + z] = 1. / sqrt(-C[0][0]);
  out[34LL * Z + z] = x[0];
  out[35LL * Z + z] = x[1];
  // torus/problem.cpp:7-13 (dynamical time) and :547-548 (floors)
  out[36LL * Z + z] = pow(x[0], 1.5);
  out[37LL * Z + z] = pow(x[0], p.rhoFloorSlope) * p.rhoFloorAmpl;
  out[38LL * Z + z] = pow(x[0], p.uFloorSlope) * p.uFloorAmpl;
  if (gamma) {
    // computeConnectionCoeffs (geometry.cpp:61-119, 631-680), eps = 1e-5
    const double eps = 1.e-5;
    double Gp[3][4][4], Gm[3][4][4];
    for (int d = 0; d < 3; d++) {
      double Xp[3] = {X[0], X[1], X[2]}, Xm[3] = {X[0], X[1], X[2]};
      Xp[d] += eps;
      Xm[d] -= eps;
      gcov_at(p, Xp, Gp[d]);
      gcov_at(p, Xm, Gm[d]);
    }
    for (int mu = 0; mu < 4; mu++)
      for (int nu = 0; nu < 4; nu++)
        for (int la = 0; la < 4; la++) {
          double s = 0.;
          for (int eta = 0; eta < 4; eta++) {
            double o = 0.;
            if (la > 0) { o += 0.5 * Gp[la - 1][eta][nu] / (2. * eps); o -= 0.5 * Gm[la - 1][eta][nu] / (2. * eps); }
            if (nu > 0) { o += 0.5 * Gp[nu - 1][eta][la] / (2. * eps); o -= 0.5 * Gm[nu - 1][eta][la] / (2. * eps); }
            if (eta > 0) { o -= 0.5 * Gp[eta - 1][nu][la] / (2. * eps); o += 0.5 * Gm[eta - 1][nu][la] / (2. * eps); }
            s += C[mu][eta] * o;
          }
          gamma[(long long)(mu * 16 + nu * 4 + la) * Z + z] = s;
        }
  }
}

void launch_geometry(const DevCfg& c, const grim_config& cfg, int location, double* out, double* gamma,
                     cudaStream_t s) {
  GeoParams p;
  p.metric = cfg.metric;
  p.derefine = cfg.DerefineThetaHorizon;
  p.cylindrify = cfg.DoCylindrify;
  p.a = cfg.blackHoleSpin;
  p.hSlope = cfg.hSlope;
  p.X1Start = cfg.X1Start;
  p.X1cyl = cfg.X1cyl;
  p.X2cyl = cfg.X2cyl;
  p.rhoFloorAmpl = cfg.RhoFloorAmpl;
  p.rhoFloorSlope = cfg.RhoFloorSlope;
  p.uFloorAmpl = cfg.UFloorAmpl;
  p.uFloorSlope = cfg.UFloorSlope;
  double o1 = 0.5, o2 = 0.5;
  if (location == GRIM_LEFT) o1 = 0.;
  else if (location == GRIM_RIGHT) o1 = 1.;
  else if (location == GRIM_BOTTOM) o2 = 0.;
  else if (location == GRIM_TOP) o2 = 1.;
  const int t = 64;
  k_geometry<<<(unsigned)((c.GZ + t - 1) / t), t, 0, s>>>(c, p, o1, o2, out, gamma);
}

}  // namespace grim
