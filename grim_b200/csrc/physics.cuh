// physics.cuh -- per-zone GRMHD/EMHD physics as device functions.
//
// One fluid element is evaluated in registers for one zone; nothing is
// materialised in HBM (the reference keeps ~80 full-grid temporaries per
// element, src/physics/physics.cpp:53-183).  Templated on the scalar type of
// the unknown-dependent quantities (double for the residual, float or
// Dual<.,nf> for the Jacobian) and on the real type R of constants.
// Operation order follows the reference expression by expression so the
// FP64 build without FMA contraction reproduces the oracle bit for bit.
#pragma once
#include "common.cuh"

namespace grim {

template <class R>
struct ZoneGeo {
  R gcov[4][4];
  R gcon[4][4];
  R g, alpha;
  R ialpha;  // 1 / alpha, formed once per load (the fast path multiplies by it)
  R x1, x2;  // physical coordinates (closures)
  R dyn;     // x1^1.5 (torus closure)
};

// Minkowski at compile time; MKS from the stored per-location arrays
// (layout, SoA: 16 gCov, 16 gCon, g, alpha, then the auxiliary fields
// x1, x2, x1^1.5, rhoFloor(x1), uFloor(x1) -> 39 words per zone).  The last
// three depend on the geometry only and are evaluated once: the torus
// closure's dynamical time r^1.5 and the radial floors of applyFloor.
enum { GEO_WORDS = 39, GEO_AUX = 34, GEO_AUX_WORDS = 5 };

template <class R>
GRIM_D void geo_minkowski(ZoneGeo<R>& G, R x1, R x2) {
#pragma unroll
  for (int m = 0; m < 4; m++)
#pragma unroll
    for (int n = 0; n < 4; n++) { G.gcov[m][n] = R(0); G.gcon[m][n] = R(0); }
  G.gcov[0][0] = R(-1); G.gcov[1][1] = R(1); G.gcov[2][2] = R(1); G.gcov[3][3] = R(1);
  G.gcon[0][0] = R(-1); G.gcon[1][1] = R(1); G.gcon[2][2] = R(1); G.gcon[3][3] = R(1);
  G.g = R(1); G.alpha = R(1); G.ialpha = R(1);
  G.x1 = x1; G.x2 = x2;
  G.dyn = R(0);
}

template <class R>
GRIM_D void geo_load(ZoneGeo<R>& G, const double* __restrict__ geo, long long Z, long long z) {
#ifdef GRIM_FAST_MATH
  // the metric and its inverse are symmetric: the fast path loads the upper
  // triangles (10 + 10 words) and mirrors them, which also keeps 12 fewer
  // values in registers; the stored lower triangles can differ from them in
  // the last bit, so the parity path reads every word as the reference does
#pragma unroll
  for (int m = 0; m < 4; m++)
#pragma unroll
    for (int n = m; n < 4; n++) {
      G.gcov[m][n] = G.gcov[n][m] = (R)__ldg(geo + (long long)(m * 4 + n) * Z + z);
      G.gcon[m][n] = G.gcon[n][m] = (R)__ldg(geo + (long long)(16 + m * 4 + n) * Z + z);
    }
#else
#pragma unroll
  for (int m = 0; m < 4; m++)
#pragma unroll
    for (int n = 0; n < 4; n++) {
      G.gcov[m][n] = (R)__ldg(geo + (long long)(m * 4 + n) * Z + z);
      G.gcon[m][n] = (R)__ldg(geo + (long long)(16 + m * 4 + n) * Z + z);
    }
#endif
  G.g = (R)__ldg(geo + 32LL * Z + z);
  G.alpha = (R)__ldg(geo + 33LL * Z + z);
  G.ialpha = R(1) / G.alpha;
  G.x1 = (R)__ldg(geo + 34LL * Z + z);
  G.x2 = (R)__ldg(geo + 35LL * Z + z);
  G.dyn = (R)__ldg(geo + 36LL * Z + z);
}

GRIM_D double zone_x1(const DevCfg& c, int i, double o) { return c.X1Start + ((double)(i - c.g1) + o) * c.dX[0]; }
GRIM_D double zone_x2(const DevCfg& c, int j, double o) { return c.X2Start + ((double)(j - c.g2) + o) * c.dX[1]; }

// the geometry of zone (i, j) (any k) at offsets (o1, o2) in zone widths:
// Minkowski when geo is null, else the stored plane of that location
template <class R>
GRIM_D void load_geo(ZoneGeo<R>& G, const DevCfg& c, const double* geo, long long z, int i, int j, double o1,
                     double o2) {
  (void)z;
  if (geo == nullptr)
    geo_minkowski<R>(G, (R)zone_x1(c, i, o1), (R)zone_x2(c, j, o2));
  else
    geo_load<R>(G, geo, c.GZ, gidx(c, i, j));
}

template <class S, class R>
struct ElemT {
  S rho, u, u1, u2, u3, pressure, temperature, soundSpeed, gam;
  R B1, B2, B3;
  S uCon[4], uCov[4], bCon[4], bCov[4], bSqr, bNorm;
  S qTilde, deltaPTilde, q, deltaP, tau, chi, nu;
};

// --- scalar helpers for the torus closure ---------------------------------
GRIM_HD double dexp(double x) { return exp(x); }
GRIM_HD float dexp(float x) { return expf(x); }
template <class T, int N>
GRIM_HD Dual<T, N> dexp(const Dual<T, N>& a) {
  Dual<T, N> r; r.v = dexp(a.v);
#pragma unroll
  for (int k = 0; k < N; k++) r.d[k] = a.d[k] * r.v;
  return r;
}
GRIM_HD double dfabs(double x) { return fabs(x); }
GRIM_HD float dfabs(float x) { return fabsf(x); }
template <class T, int N>
GRIM_HD Dual<T, N> dfabs(const Dual<T, N>& a) { return a.v < T(0) ? -a : a; }
GRIM_HD double dmin2(double a, double b) { return fmin(a, b); }
GRIM_HD float dmin2(float a, float b) { return fminf(a, b); }
template <class T, int N>
GRIM_HD Dual<T, N> dmin2(const Dual<T, N>& a, const Dual<T, N>& b) { return (b.v < a.v) ? b : a; }
GRIM_HD double dmax2(double a, double b) { return fmax(a, b); }
GRIM_HD float dmax2(float a, float b) { return fmaxf(a, b); }
template <class T, int N>
GRIM_HD Dual<T, N> dmax2(const Dual<T, N>& a, const Dual<T, N>& b) { return (b.v > a.v) ? b : a; }
GRIM_HD double dcube(double x) { return pow(x, 3.); }
GRIM_HD float dcube(float x) { return x * x * x; }
template <class T, int N>
GRIM_HD Dual<T, N> dcube(const Dual<T, N>& a) { return a * a * a; }

// setFluidElementParameters (problem hook) -- closures
template <class S, class R>
GRIM_D void closure(ElemT<S, R>& e, const ZoneGeo<R>& G, const DevCfg& c) {
  const S cs = e.soundSpeed;
  if (c.closure == GRIM_CLOSURE_CONST_TAU) {
    // linear_modes/problem.cpp:3-8
    e.tau = Lift<S>::of(c.tau0);
    e.chi = cs * cs * e.tau;
    e.nu = cs * cs * e.tau;
  } else if (c.closure == GRIM_CLOSURE_TAU_PROFILE) {
    R s = (G.x2 - (R)c.X2Start) / ((R)c.X2End - (R)c.X2Start);
    e.tau = Lift<S>::of((double)val_of((R)c.tau0 + ((R)c.tau1 - (R)c.tau0) * s));
    e.chi = cs * cs * e.tau;
    e.nu = cs * cs * e.tau;
  } else {
    // torus/problem.cpp:7-55
    typedef typename Real<S>::type T;
    const T Dyn = (T)val_of(G.dyn);
    S t = Lift<S>::of((double)Dyn);
    if (c.conduction) {
      S Qmax = (T)c.CondClosure * e.rho * dcube(cs);
      const T lambda = (T)0.01;
      S yCon = dfabs(e.q) / Qmax;
      yCon = dexp(-(yCon - T(1.)) / lambda);
      S fdCon = yCon / (yCon + T(1.)) + T(1.e-5);
      t = dmin2(t, Dyn * fdCon);
    }
    if (c.viscosity) {
      const T fl = (T)c.bSqrFloor;
      const S p = e.pressure, dP = e.deltaP;
      S dPmod = dmaxc(p - T(2. / 3.) * dP, fl) / dmaxc(p + T(1. / 3.) * dP, fl);
      S dPmaxPlus = dmin2((T)c.ViscClosure * e.bSqr * T(0.5) * dPmod, T(1.49) * p / T(1.07));
      S dPmaxMinus = dmax2(-(T)c.ViscClosure * e.bSqr, -T(2.99) * p / T(1.07));
      S dPmax = (val(dP) > T(0.)) ? dPmaxPlus : dPmaxMinus;
      const T lambda = (T)0.01;
      S yVis = dfabs(dP) / (dfabs(dPmax) + fl);
      yVis = dexp(-(yVis - T(1.)) / lambda);
      S fdVis = yVis / (yVis + T(1.)) + T(1.e-5);
      t = dmin2(t, Dyn * fdVis);
    }
    e.tau = t;
    S maxAlpha = (T(1.) - cs * cs) / (T(2.) * cs * cs + T(1.e-12));
    e.chi = dmin2(maxAlpha, Lift<S>::of(c.CondAlpha)) * cs * cs * t;
    e.nu = dmin2(maxAlpha, Lift<S>::of(c.ViscAlpha)) * cs * cs * t;
  }
}

// fluidElement::set (physics.cpp:53-183) minus T^mu_nu, which callers take
// row by row with tmunu().
template <int COND, int VISC, class S, class R>
GRIM_D void elem_set(ElemT<S, R>& e, const S& rho_in, const S& u_in, const S& v1, const S& v2,
                     const S& v3, R B1, R B2, R B3, const S& qT, const S& dPT,
                     const ZoneGeo<R>& G, const DevCfg& c) {
  typedef typename Real<S>::type T;
  const T Gam = (T)c.Gam;
  e.rho = dmaxc(rho_in, (T)c.rhoFloor);
  e.u = dmaxc(u_in, (T)c.uFloor);
  e.u1 = v1; e.u2 = v2; e.u3 = v3;
  e.B1 = B1; e.B2 = B2; e.B3 = B3;
  e.pressure = (Gam - T(1.)) * e.u;
  e.temperature = dmaxc(e.pressure / e.rho, (T)c.TFloor);
  e.soundSpeed = dsqrt(Gam * e.pressure / (e.rho + Gam * e.u));
#ifdef GRIM_FAST_MATH
  // gamma and 1 / gamma from one reciprocal square root: u^0 = gamma / alpha
  // and 1 / u^0 = alpha / gamma without divisions
  const S gsq = T(1) + G.gcov[1][1] * v1 * v1 + G.gcov[2][2] * v2 * v2 + G.gcov[3][3] * v3 * v3 +
                T(2) * (G.gcov[1][2] * v1 * v2 + G.gcov[1][3] * v1 * v3 + G.gcov[2][3] * v2 * v3);
  const S rgam = drsqrt(gsq);
  e.gam = gsq * rgam;
  e.uCon[0] = e.gam * G.ialpha;
#else
  e.gam = dsqrt(T(1) + G.gcov[1][1] * v1 * v1 + G.gcov[2][2] * v2 * v2 + G.gcov[3][3] * v3 * v3 +
                T(2) * (G.gcov[1][2] * v1 * v2 + G.gcov[1][3] * v1 * v3 + G.gcov[2][3] * v2 * v3));
  e.uCon[0] = e.gam / G.alpha;
#endif
  e.uCon[1] = v1 - e.gam * G.gcon[0][1] * G.alpha;
  e.uCon[2] = v2 - e.gam * G.gcon[0][2] * G.alpha;
  e.uCon[3] = v3 - e.gam * G.gcon[0][3] * G.alpha;
#pragma unroll
  for (int mu = 0; mu < 4; mu++)
    e.uCov[mu] = G.gcov[mu][0] * e.uCon[0] + G.gcov[mu][1] * e.uCon[1] + G.gcov[mu][2] * e.uCon[2] +
                 G.gcov[mu][3] * e.uCon[3];
  e.bCon[0] = B1 * e.uCov[1] + B2 * e.uCov[2] + B3 * e.uCov[3];
#ifdef GRIM_FAST_MATH
  {
    const S iu0 = G.alpha * rgam;  // 1 / u^0
    e.bCon[1] = (B1 + e.bCon[0] * e.uCon[1]) * iu0;
    e.bCon[2] = (B2 + e.bCon[0] * e.uCon[2]) * iu0;
    e.bCon[3] = (B3 + e.bCon[0] * e.uCon[3]) * iu0;
  }
#else
  e.bCon[1] = (B1 + e.bCon[0] * e.uCon[1]) / e.uCon[0];
  e.bCon[2] = (B2 + e.bCon[0] * e.uCon[2]) / e.uCon[0];
  e.bCon[3] = (B3 + e.bCon[0] * e.uCon[3]) / e.uCon[0];
#endif
#pragma unroll
  for (int mu = 0; mu < 4; mu++)
    e.bCov[mu] = G.gcov[mu][0] * e.bCon[0] + G.gcov[mu][1] * e.bCon[1] + G.gcov[mu][2] * e.bCon[2] +
                 G.gcov[mu][3] * e.bCon[3];
  e.bSqr = e.bCon[0] * e.bCov[0] + e.bCon[1] * e.bCov[1] + e.bCon[2] * e.bCov[2] +
           e.bCon[3] * e.bCov[3] + (T)c.bSqrFloor;
  e.bNorm = dsqrt(e.bSqr);
  const S cs = e.soundSpeed;
  if (COND) {
    e.qTilde = qT;
    if (c.hoCond == 1)
      e.q = qT * e.temperature * dsqrt(e.rho * (T)c.CondAlpha * cs * cs);
    else
      e.q = qT;
  }
  if (VISC) {
    e.deltaPTilde = dPT;
    if (c.hoVisc == 1)
      e.deltaP = dPT * dsqrt(e.temperature * e.rho * (T)c.ViscAlpha * cs * cs);
    else
      e.deltaP = dPT;
  }
  if constexpr (COND || VISC) closure(e, G, c);
}

// T^mu_nu (physics.cpp:153-178)
template <int COND, int VISC, class S, class R>
GRIM_D S tmunu(const ElemT<S, R>& e, int mu, int nu) {
  typedef typename Real<S>::type T;
  const T d = (mu == nu) ? T(1.) : T(0.);
  S w = e.rho + e.u + e.pressure + e.bSqr;
  S pt = e.pressure + T(0.5) * e.bSqr;
  S r = w * e.uCon[mu] * e.uCov[nu] + pt * d - e.bCon[mu] * e.bCov[nu];
  if (COND) r += e.q / e.bNorm * (e.uCon[mu] * e.bCov[nu] + e.bCon[mu] * e.uCov[nu]);
  if (VISC) r += (-e.deltaP) * (e.bCon[mu] * e.bCov[nu] / e.bSqr - T(1. / 3.) * (d + e.uCon[mu] * e.uCov[nu]));
  return r;
}

// computeFluxes(dir) for the fluid rows (physics.cpp:185-217): out[0..nf)
template <int COND, int VISC, class S, class R>
GRIM_D void fluxes_fluid(const ElemT<S, R>& e, int dir, R g, S* out, int Q, int DP) {
  S fr = g * (e.rho * e.uCon[dir]);
  out[0] = fr;
  out[1] = g * tmunu<COND, VISC>(e, dir, 0) + fr;
  out[2] = g * tmunu<COND, VISC>(e, dir, 1);
  out[3] = g * tmunu<COND, VISC>(e, dir, 2);
  out[4] = g * tmunu<COND, VISC>(e, dir, 3);
  if (COND) out[Q] = g * (e.uCon[dir] * e.qTilde);
  if (VISC) out[DP] = g * (e.uCon[dir] * e.deltaPTilde);
}
// induction rows of computeFluxes
template <class S, class R>
GRIM_D void fluxes_B(const ElemT<S, R>& e, int dir, R g, S* out3) {
  out3[0] = g * (e.bCon[1] * e.uCon[dir] - e.bCon[dir] * e.uCon[1]);
  out3[1] = g * (e.bCon[2] * e.uCon[dir] - e.bCon[dir] * e.uCon[2]);
  out3[2] = g * (e.bCon[3] * e.uCon[dir] - e.bCon[dir] * e.uCon[3]);
}

// computeMinMaxCharSpeeds (riemannsolver.cpp:54-200), dir = 0,1,2
// (templated on the scalar for the op-counting build; double in the kernels)
template <int COND, int VISC, class S, class R>
GRIM_D void char_speeds(const ElemT<S, R>& e, const ZoneGeo<R>& G, int dir, const DevCfg& c, S& minSpeed,
                        S& maxSpeed) {
  const S Gam = S(c.Gam);
#ifdef GRIM_FAST_MATH
  // without conduction or viscosity: c_s^2 itself (the element's c_s, a
  // square root, is then dead code) and c_A^2 over one reciprocal of the
  // product of their denominators
  S cAlvenSqr, csSqr;
  if constexpr (COND || VISC) {
    cAlvenSqr = e.bSqr / (e.rho + Gam * e.u + e.bSqr);
    csSqr = e.soundSpeed * e.soundSpeed;
  } else {
    const S w1 = e.rho + Gam * e.u, w2 = w1 + e.bSqr;
    const S r = S(1.) / (w1 * w2);
    cAlvenSqr = e.bSqr * w1 * r;
    csSqr = Gam * e.pressure * w2 * r;
  }
#else
  S cAlvenSqr = e.bSqr / (e.rho + Gam * e.u + e.bSqr);
  S csSqr = e.soundSpeed * e.soundSpeed;
#endif
  S cVisSqr = S(0.);
  if (VISC) cVisSqr = S(4.) / S(3.) / (e.rho + Gam * e.u) * e.rho * e.nu / e.tau;
  S cConSqr = S(0.);
  if (COND) cConSqr = (Gam - S(1.)) * e.chi / e.tau;
#ifdef GRIM_FAST_MATH
  // with no conduction the combination is (cs^2 + |cs^2|) / 2 = cs^2
  // (cs^2 >= 0: a square root of a square is the magnitude exactly)
  if constexpr (COND)
    cConSqr = S(0.5) * (csSqr + cConSqr + dsqrt(csSqr * csSqr + cConSqr * cConSqr));
  else
    cConSqr = csSqr;
#else
  cConSqr = S(0.5) * (csSqr + cConSqr + dsqrt(csSqr * csSqr + cConSqr * cConSqr));
#endif
  csSqr = cConSqr + cVisSqr;
  csSqr = csSqr + cAlvenSqr - csSqr * cAlvenSqr;
  if (csSqr > S(1.)) csSqr = S(1.);
  const int s = dir + 1;
  const S ASqr = G.gcon[s][s];
  const S BSqr = G.gcon[0][0];
  const S ADotU = e.uCon[s];
  const S BDotU = e.uCon[0];
  const S ADotB = G.gcon[s][0];
  S A = (BDotU * BDotU) - (BSqr + BDotU * BDotU) * csSqr;
  S B = S(2.) * (ADotU * BDotU - (ADotB + ADotU * BDotU) * csSqr);
  S C = ADotU * ADotU - (ASqr + ADotU * ADotU) * csSqr;
  S discr = dsqrt(dmax2(B * B - S(4.) * A * C, S(1.e-16)));
#ifdef GRIM_FAST_MATH
  const S i2a = S(0.5) / A;
  S mn = (B - discr) * i2a;
  S mx = (B + discr) * i2a;
#else
  S mn = -(-B + discr) / S(2.) / A;
  S mx = -(-B - discr) / S(2.) / A;
#endif
  if (mn > S(-1.e-15)) mn = S(-1.e-15);
  if (mx < S(1.e-15)) mx = S(1.e-15);
  minSpeed = mn;
  maxSpeed = mx;
}

// ---------------------------------------------------------------------------
// Analytic Jacobian of the ideal-MHD zone residual.  With no conduction or
// viscosity the only unknown-dependent part of the residual is the
// conserved vector U(P) (the fluid rows of computeFluxes along X0,
// physics.cpp:185-217; residual.cpp:3-60), so J = (dU/dP) / dt' with B
// held fixed.  The columns follow fluidElement::set (physics.cpp:53-183)
// by the chain rule:
//   gamma = sqrt(1 + g_ij v^i v^j)        d gamma / d v^j = g_jk v^k / gamma
//   u^0 = gamma / alpha,  u^i = v^i - gamma alpha g^0i
//   b^0 = B^i u_i,  b^i = (B^i + b^0 u^i) / u^0,  d b^2 = 2 b_mu d b^mu
//   T^0_nu = w u^0 u_nu + (p + b^2/2) delta^0_nu - b^0 b_nu,  w = rho+u+p+b^2
// and a floored rho or u (af::max with the floor) has a zero column, as in
// the forward tangent.  About a third of the flops of the 5-lane tangent.
// ---------------------------------------------------------------------------
template <class T, class KC>
GRIM_D void ideal_jacobian(const double* P, const KC& K, const ZoneGeo<T>& G, const DevCfg& c, T J[5][5]) {
  const T Gam = (T)c.Gam;
  const T rhoIn = (T)P[0], uIn = (T)P[1];
  const T rhoF = (T)c.rhoFloor, uF = (T)c.uFloor;
  const bool fr = rhoIn >= rhoF, fu = uIn >= uF;
  const T rho = fr ? rhoIn : rhoF;
  const T u = fu ? uIn : uF;
  const T p = (Gam - T(1.)) * u;
  const T v[3] = {(T)P[2], (T)P[3], (T)P[4]};
  const T B[3] = {(T)K.B[0], (T)K.B[1], (T)K.B[2]};
  T gv[3];
#pragma unroll
  for (int j = 0; j < 3; j++) gv[j] = G.gcov[j + 1][1] * v[0] + G.gcov[j + 1][2] * v[1] + G.gcov[j + 1][3] * v[2];
  // gamma and 1 / gamma from one reciprocal square root
  const T gsq = T(1.) + v[0] * gv[0] + v[1] * gv[1] + v[2] * gv[2];
  const T rgam = drsqrt(gsq);
  const T gam = gsq * rgam;
  T uCon[4], uCov[4], bCon[4], bCov[4];
  uCon[0] = gam * G.ialpha;
#pragma unroll
  for (int i = 1; i < 4; i++) uCon[i] = v[i - 1] - gam * G.gcon[0][i] * G.alpha;
#pragma unroll
  for (int m = 0; m < 4; m++)
    uCov[m] = G.gcov[m][0] * uCon[0] + G.gcov[m][1] * uCon[1] + G.gcov[m][2] * uCon[2] + G.gcov[m][3] * uCon[3];
  const T iu0 = G.alpha * rgam;  // 1 / u^0
  bCon[0] = B[0] * uCov[1] + B[1] * uCov[2] + B[2] * uCov[3];
#pragma unroll
  for (int i = 1; i < 4; i++) bCon[i] = (B[i - 1] + bCon[0] * uCon[i]) * iu0;
#pragma unroll
  for (int m = 0; m < 4; m++)
    bCov[m] = G.gcov[m][0] * bCon[0] + G.gcov[m][1] * bCon[1] + G.gcov[m][2] * bCon[2] + G.gcov[m][3] * bCon[3];
  const T bsq = bCon[0] * bCov[0] + bCon[1] * bCov[1] + bCon[2] * bCov[2] + bCon[3] * bCov[3] + (T)c.bSqrFloor;
  const T w = rho + u + p + bsq;
  const T gi = G.g / (T)K.dtp;  // sqrt(-g) / dt'
  // rho column
  {
    const T s = fr ? gi * uCon[0] : T(0.);
    J[0][0] = s;
    J[1][0] = s * uCov[0] + s;
#pragma unroll
    for (int n = 1; n < 4; n++) J[1 + n][0] = s * uCov[n];
  }
  // u column
  {
    const T s = fu ? gi : T(0.);
    J[0][1] = T(0.);
    J[1][1] = s * (Gam * uCon[0] * uCov[0] + (Gam - T(1.)));
#pragma unroll
    for (int n = 1; n < 4; n++) J[1 + n][1] = s * (Gam * uCon[0] * uCov[n]);
  }
  // velocity columns
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const T dg = gv[j] * rgam;
    T du[4], duCov[4], db[4];
    du[0] = dg * G.ialpha;
#pragma unroll
    for (int i = 1; i < 4; i++) du[i] = ((i == j + 1) ? T(1.) : T(0.)) - dg * G.gcon[0][i] * G.alpha;
#pragma unroll
    for (int m = 0; m < 4; m++)
      duCov[m] = G.gcov[m][0] * du[0] + G.gcov[m][1] * du[1] + G.gcov[m][2] * du[2] + G.gcov[m][3] * du[3];
    db[0] = B[0] * duCov[1] + B[1] * duCov[2] + B[2] * duCov[3];
#pragma unroll
    for (int i = 1; i < 4; i++) db[i] = (db[0] * uCon[i] + bCon[0] * du[i] - bCon[i] * du[0]) * iu0;
    const T dbsq = T(2.) * (bCov[0] * db[0] + bCov[1] * db[1] + bCov[2] * db[2] + bCov[3] * db[3]);
    T dT[4];
#pragma unroll
    for (int n = 0; n < 4; n++) {
      const T dbCov = G.gcov[n][0] * db[0] + G.gcov[n][1] * db[1] + G.gcov[n][2] * db[2] + G.gcov[n][3] * db[3];
      dT[n] = dbsq * uCon[0] * uCov[n] + w * (du[0] * uCov[n] + uCon[0] * duCov[n]) -
              (db[0] * bCov[n] + bCon[0] * dbCov);
    }
    dT[0] = dT[0] + T(0.5) * dbsq;
    const T d0 = gi * rho * du[0];
    J[0][2 + j] = d0;
    J[1][2 + j] = gi * dT[0] + d0;
#pragma unroll
    for (int n = 1; n < 4; n++) J[1 + n][2 + j] = gi * dT[n];
  }
}

// ---------------------------------------------------------------------------
// Zone residual (residual.cpp:3-180) for the Newton kernels.
//
// Stage constants of one zone: Uold (consOld rows), divF and the explicit
// sources (stored by the stencil kernel), and the reference elements of the
// stage -- elemOld (half stage) or elemHalfStep (full stage) -- recomputed
// here from their primitives since they are pointwise.
// ---------------------------------------------------------------------------
template <int NF>
struct StageConst {
  double Uold[NF];
  double divF[NF];
  double Sexp[NF];
  double B[3];
  // EMHD: elemOld uCov / temperature, reference-element quantities
  double uCovOld[4], TOld;
  double refRho, refNu, refChi, refTau, refT, refBCon[4], refBSqr, refBNorm, refUCon0;
  double refQTilde, refDPTilde;
  double sImpOldQ, sImpOldDP;  // 0.5*(...) partner of the implicit source
  double normQ, normDP;        // EMHD row normalisation
  double dtp;                  // dt' (dt/2 or dt)
  // fast path, ideal MHD: R = U / dt' + Kc, Kc = divF + Sexp - Uold / dt'
  double idtp;
  double Kc[NF];
  // square of the Newton test's rounding floor: (tolUlps eps max_v |Kc_v|)^2
  // over the conserved rows (|Kc_v| = |U_v| / dt' at the solution, the
  // residual's largest term), 0 when tolUlps = 0
  double tolFloor2;
};

// the per-zone Newton test: converged once sum R^2 <= this (solve.cpp:36-41
// with atol; rtol relative to the first residual; the rounding floor)
template <class K_>
GRIM_D double newton_tol(const DevCfg& c, double l2first, const K_& K) {
  return fmax(fmax(c.atol, c.rtol * c.rtol * l2first), K.tolFloor2);
}

template <int COND, int VISC, class S, class R>
GRIM_D void zone_residual(const S* P, const StageConst<5 + COND + VISC>& K, const ZoneGeo<R>& G,
                          const DevCfg& c, S* Rout) {
  typedef typename Real<S>::type T;
  constexpr int NF = 5 + COND + VISC;
  constexpr int Q = 5, DP = 5 + COND;
  ElemT<S, R> e;
  S qT = COND ? P[Q] : S(T(0));
  S dPT = VISC ? P[DP] : S(T(0));
  elem_set<COND, VISC>(e, P[0], P[1], P[2], P[3], P[4], (R)K.B[0], (R)K.B[1], (R)K.B[2], qT, dPT, G, c);
  S U[NF];
  fluxes_fluid<COND, VISC>(e, 0, G.g, U, Q, DP);
#ifdef GRIM_FAST_MATH
  if constexpr (COND == 0 && VISC == 0) {
    // the unknown-independent terms folded into one constant per row
    const T idtp = (T)K.idtp;
#pragma unroll
    for (int v = 0; v < NF; v++) Rout[v] = U[v] * idtp + (T)K.Kc[v];
    return;
  }
#endif
  const T dtp = (T)K.dtp;
#pragma unroll
  for (int v = 0; v < NF; v++) {
    S r = (U[v] - (T)K.Uold[v]) / dtp + (T)K.divF[v];
    if (c.metric != GRIM_MINKOWSKI || COND || VISC) r = r + (T)K.Sexp[v];
    Rout[v] = r;
  }
  if (COND || VISC) {
    // time-derivative sources (physics.cpp:219-317) with `this` = the
    // stage's reference element, elemOld / elemNew = old / trial
    S dtuCov[4];
#pragma unroll
    for (int mu = 0; mu < 4; mu++) dtuCov[mu] = (e.uCov[mu] - (T)K.uCovOld[mu]) / dtp;
    S div = S(T(0.));
#pragma unroll
    for (int mu = 0; mu < 4; mu++) div = div + G.gcon[0][mu] * dtuCov[mu];
    const T rr = (T)K.refRho, rnu = (T)K.refNu, rchi = (T)K.refChi, rtau = (T)K.refTau, rT = (T)K.refT;
    const T rbn = (T)K.refBNorm, rbs = (T)K.refBSqr;
    if (VISC) {
      S d0 = -div * rr * rnu;
#pragma unroll
      for (int mu = 0; mu < 4; mu++) d0 += T(3.) * rr * rnu * (T)K.refBCon[0] * (T)K.refBCon[mu] / rbs * dtuCov[mu];
      if (c.hoVisc == 1) d0 = d0 * (T)sqrt((double)(rtau / rr / rnu / rT));
      S sdt = -G.g * (d0) / rtau;
      if (c.hoVisc == 1) sdt = sdt - T(0.5) * G.g * div * (T)K.refDPTilde;
      // implicit source of the trial with the reference tau (physics.cpp:343)
      S simp = G.g * (P[DP]) / rtau;
      S r = Rout[DP] + T(0.5) * ((T)K.sImpOldDP + simp) + sdt;
      Rout[DP] = r * (T)K.normDP;
    }
    if (COND) {
      S qq = -rr * rchi * (T)K.refBCon[0] / rbn * (e.temperature - (T)K.TOld) / dtp;
#pragma unroll
      for (int nu = 0; nu < 4; nu++) qq -= rr * rchi * rT * (T)K.refBCon[nu] / rbn * (T)K.refUCon0 * dtuCov[nu];
      if (c.hoCond == 1) qq = qq * ((T)sqrt((double)(rtau / rr / rchi)) / rT);
      S sdt = -G.g * (qq) / rtau;
      if (c.hoCond == 1) sdt = sdt - T(0.5) * G.g * div * (T)K.refQTilde;
      S simp = G.g * (P[Q]) / rtau;
      S r = Rout[Q] + T(0.5) * ((T)K.sImpOldQ + simp) + sdt;
      Rout[Q] = r * (T)K.normQ;
    }
  }
}

}  // namespace grim
