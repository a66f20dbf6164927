// torus.cuh -- the torus problem's hooks on the hot path
// (src/problem/torus/problem.cpp): floors applied after each stage
// (applyFloor, :542-712, with the NaN reset of fullStepDiagnostics,
// :719-746), the radial inflow check and the polar fix applied at the start
// of each stage (setProblemSpecificBCs, :941-1241).  The flux filter
// (:1243-1285) is applied inside the stage epilogue.  One thread per zone;
// each is a direct restatement of the reference's array expressions.
#pragma once
#include <type_traits>

#include "physics.cuh"

namespace grim {
namespace GRIM_KNS {

struct TorusCfg {
  double MaxLorentzFactor, RhoFloorAmpl, UFloorAmpl, RhoFloorSlope, UFloorSlope;
  double BsqrOverRhoMax, BsqrOverUMax;
};

template <int COND, int VISC>
GRIM_D void load_elem(ElemT<double, double>& e, const DevCfg& c, const double* p, long long z,
                      const ZoneGeo<double>& G) {
  const long long Z = c.Z;
  elem_set<COND, VISC>(e, p[z], p[Z + z], p[2 * Z + z], p[3 * Z + z], p[4 * Z + z], p[(long long)c.B1 * Z + z],
                       p[(long long)(c.B1 + 1) * Z + z], p[(long long)(c.B1 + 2) * Z + z],
                       COND ? p[(long long)c.Q * Z + z] : 0., VISC ? p[(long long)c.DP * Z + z] : 0., G, c);
}

// the element of one zone's primitives q (rows: fluid, then B1..B3); S is
// double, or the forward-tangent scalar of the adjoint's local Jacobians
template <int COND, int VISC, class S>
GRIM_D void elem_of(ElemT<S, S>& e, const DevCfg& c, const S* q, const ZoneGeo<S>& G) {
  constexpr int NFT = 5 + COND + VISC;
  elem_set<COND, VISC>(e, q[RHO], q[UU], q[U1], q[U2], q[U3], q[NFT], q[NFT + 1], q[NFT + 2], COND ? q[5] : S(0.),
                       VISC ? q[5 + COND] : S(0.), G, c);
}

// applyFloor (problem.cpp:542-712) on one zone's primitives q, held in
// registers, after the NaN reset of fullStepDiagnostics when nanReset;
// minRho, minU are the zone's floor values (geometry words 37, 38)
// Returns true when the element left in eOut (if given) is the element of
// the final q (no change after its last evaluation), so a caller needing
// that element can use it as is.
// S is double on the hot path, or the forward-tangent scalar when the
// adjoint takes the floors' local Jacobian (branches then follow the values;
// the zero-weight drift-frame fix is skipped as in the fast path, which
// leaves the derivative unchanged and keeps a non-finite correction out of
// it).
template <int COND, int VISC, class S>
GRIM_D bool torus_floor_zone(const DevCfg& c, const TorusCfg& t, S* q, const ZoneGeo<S>& G, double minRho,
                             double minU, bool nanReset, ElemT<S, S>* eOut = nullptr) {
  constexpr int NFT = 5 + COND + VISC, DOFT = NFT + 3;
#ifdef GRIM_FAST_MATH
  constexpr bool kSkipNoFix = true;
#else
  constexpr bool kSkipNoFix = !std::is_same<S, double>::value;
#endif
  if (nanReset) {
    bool bad = false;
#pragma unroll
    for (int v = 0; v < DOFT; v++) bad |= isnan(val_of(q[v]));
    if (bad)
#pragma unroll
      for (int v = 0; v < DOFT; v++) q[v] = S(0.);
  }
  const S rho_pre = q[RHO] * 1., u_pre = q[UU] * 1.;
  bool usefloor = false;
  {
    bool cd = val_of(q[RHO]) < minRho;
    usefloor = cd;
    if (cd) q[RHO] = S(minRho);
    cd = val_of(q[UU]) < minU;
    usefloor = usefloor || cd;
    if (cd) q[UU] = S(minU);
  }
  ElemT<S, S> e;
  elem_of<COND, VISC>(e, c, q, G);
  const S bSqr1 = e.bSqr;
  {
    bool cd = val_of(bSqr1) > t.BsqrOverRhoMax * val_of(q[RHO]);
    usefloor = usefloor || cd;
    if (cd) q[RHO] = bSqr1 / t.BsqrOverRhoMax;
    cd = val_of(bSqr1) > t.BsqrOverUMax * val_of(q[UU]);
    usefloor = usefloor || cd;
    if (cd) q[UU] = bSqr1 / t.BsqrOverUMax;
  }
  const S rho = q[RHO], u = q[UU];
  S trans = fmax(fmin(S(1.), (bSqr1 - 0.1 * rho) / rho), S(0.)) * (usefloor ? 1. : 0.);
  // the fix below blends with weight trans: with trans = 0 it returns the
  // velocities unchanged (up to the sign of a zero, or a non-finite
  // correction, which it would propagate), so the fast path skips it
  if (!kSkipNoFix || val_of(trans) != 0.) {
  // drift-frame velocity fix
  const S betapar = -e.bCon[0] / bSqr1 / e.uCon[0];
  S betasqr = betapar * betapar * bSqr1;
  const double betasqrmax = 1. - 1. / t.MaxLorentzFactor / t.MaxLorentzFactor;
  betasqr = fmin(betasqr, S(betasqrmax));
  const S gamma = 1. / dsqrt(1. - betasqr);
  S ucondr[4];
#pragma unroll
  for (int m = 0; m < 4; m++) ucondr[m] = gamma * (e.uCon[m] + betapar * e.bCon[m]);
  const S Bcon[4] = {S(0.), q[NFT], q[NFT + 1], q[NFT + 2]};
  S Bcov[4];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    S s = S(0.);
#pragma unroll
    for (int n = 0; n < 4; n++) s += G.gcov[n][m] * Bcon[n];
    Bcov[m] = s;
  }
  S udotB = S(0.), bSqr_fl = S(0.);
#pragma unroll
  for (int n = 0; n < 4; n++) {
    udotB += Bcov[n] * e.uCon[n];
    bSqr_fl += Bcov[n] * Bcon[n];
  }
  S bNorm = fmax(dsqrt(bSqr_fl), S(sqrt(c.bSqrFloor)));
  const S wold = rho_pre + u_pre * c.Gam;
  const S QdotB = udotB * wold * e.uCon[0];
  const S wnew = rho + u * c.Gam;
  const S x = 2. * QdotB / (bNorm * wnew * ucondr[0]);
  const S vpar = x / (ucondr[0] * (1. + dsqrt(1. + x * x)));
  const S inv_ut = 1. / ucondr[0];
  S vcon[4];
  vcon[0] = S(0. + 1.);
#pragma unroll
  for (int m = 1; m < 4; m++) vcon[m] = vpar * Bcon[m] / bNorm + ucondr[m] * inv_ut;
  S vsqr = S(0.);
#pragma unroll
  for (int m = 0; m < 4; m++)
#pragma unroll
    for (int n = 0; n < 4; n++) vsqr += G.gcov[m][n] * vcon[m] * vcon[n];
  if (val_of(vsqr) >= 0. || val_of(vsqr) < val_of(1. / G.gcon[0][0])) vsqr = 1. / G.gcon[0][0];
  const S ut = dsqrt(-1. / vsqr);
#pragma unroll
  for (int m = 1; m < 4; m++) {
    S utcon = ut * (vcon[m] - G.gcon[0][m] / G.gcon[0][0]);
    q[UU + m] = q[UU + m] * (1. - trans) + trans * utcon;
  }
  }  // drift-frame fix
  // maximum Lorentz factor
  // (no floor applied: q is the state the element above was set from, trans
  // is 0 so the fix was skipped, and that element stands)
  if (!kSkipNoFix || usefloor) elem_of<COND, VISC>(e, c, q, G);
  bool current = true;
  {
    const S lf2 = e.gam * e.gam;
    const double gm2 = t.MaxLorentzFactor * t.MaxLorentzFactor;
    if (val_of(lf2) > gm2) {
      S mf = 1. / dsqrt(fmax((lf2 - 1.) / (gm2 - 1.), S(1.)));
      q[U1] *= mf;
      q[U2] *= mf;
      q[U3] *= mf;
      current = false;
    }
  }
  if constexpr (COND || VISC) {
    // the EMHD limiters, on the scalar type (the adjoint takes their local
    // Jacobian); on doubles the same operations in the same order
    elem_of<COND, VISC>(e, c, q, G);
    if (COND) {
      const S cs = e.soundSpeed;
      const S Qmax = 1.07 * c.CondClosure * q[RHO] * dcube(cs);
      const S lim = fmax(fabs(e.q) / Qmax, S(1.));
      q[5] = q[5] / lim;
    }
    if (VISC) {
      const S pr = e.pressure, dP = e.deltaP, bs = e.bSqr;
      const S dPmod = fmax(pr - 2. / 3. * dP, S(0.01 * c.bSqrFloor)) / fmax(pr + 1. / 3. * dP, S(c.bSqrFloor));
      const S dPmaxPlus = fmin(1.07 * c.ViscClosure * bs * 0.5 * dPmod, 1.49 * pr);
      const S dPmaxMinus = fmax(-1.07 * c.ViscClosure * bs, -2.99 * pr);
      const S f = (val_of(dP) > 0.) ? 1. / fmax(dP / dPmaxPlus, S(1.)) : 1. / fmax(dP / dPmaxMinus, S(1.));
      q[5 + COND] = q[5 + COND] * f;
    }
    current = false;
  }
  if (eOut && current) *eOut = e;
  return current;
}

// applyFloor on every zone of p in place, after the NaN reset when
// *nanFlag is set
template <int COND, int VISC>
__global__ void k_torus_floor(DevCfg c, TorusCfg t, double* __restrict__ p, const double* __restrict__ geoC,
                              const unsigned long long* nanFlag) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  const long long Z = c.Z;
  const long long gz = gidx(c, z);
  ZoneGeo<double> G;
  geo_load<double>(G, geoC, c.GZ, gz);
  constexpr int DOFT = 8 + COND + VISC;
  double q[DOFT];
#pragma unroll
  for (int v = 0; v < DOFT; v++) q[v] = p[(long long)v * Z + z];
  torus_floor_zone<COND, VISC>(c, t, q, G, __ldg(geoC + 37LL * c.GZ + gz), __ldg(geoC + 38LL * c.GZ + gz),
                               nanFlag && *nanFlag);
#pragma unroll
  for (int v = 0; v < DOFT; v++) p[(long long)v * Z + z] = q[v];
}

// NaN count over the interior (fullStepDiagnostics, problem.cpp:725-733)
static __global__ void k_nan_flag(DevCfg c, const double* __restrict__ p, unsigned long long* flag) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int bad = 0;
  if (n < c.Zint) {
    long long z = interior_to_z(c, n);
    for (int v = 0; v < c.dof; v++) bad |= isnan(p[(long long)v * c.Z + z]) ? 1 : 0;
  }
  bad = __syncthreads_count(bad);
  if (threadIdx.x == 0 && bad) atomicAdd(flag, (unsigned long long)bad);
}

// inflowCheck (problem.cpp:941-1044) on the X1 ghost zones
template <int COND, int VISC>
__global__ void k_torus_inflow(DevCfg c, TorusCfg t, double* __restrict__ p, const double* __restrict__ geoC) {
  // one thread per (ghost i, j, k); 2*ng columns of X1 ghosts
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long cols = (long long)2 * c.ng * c.N2T * c.N3T;
  if (n >= cols) return;
  const int gi = (int)(n % (2 * c.ng));
  const long long r = n / (2 * c.ng);
  const int j = (int)(r % c.N2T), k = (int)(r / c.N2T);
  const bool right = gi >= c.ng;
  const int i = right ? (c.N1 + c.ng + (gi - c.ng)) : gi;
  const long long Z = c.Z;
  const long long z = zidx(c, i, j, k);
  ZoneGeo<double> G;
  geo_load<double>(G, geoC, c.GZ, gidx(c, i, j));
  ElemT<double, double> e;
  load_elem<COND, VISC>(e, c, p, z, G);
  double* u1 = p + (long long)U1 * Z + z;
  double* u2 = p + (long long)U2 * Z + z;
  double* u3 = p + (long long)U3 * Z + z;
  *u1 = *u1 / e.gam;
  *u2 = *u2 / e.gam;
  *u3 = *u3 / e.gam;
  if (right) {
    // the last active zone's g^{01} alpha, copied into the ghost columns
    const long long ze = gidx(c, c.N1 + c.ng - 1, j);
    const double minUr = __ldg(geoC + 17LL * c.GZ + ze) * __ldg(geoC + 33LL * c.GZ + ze);
    *u1 = fmax(minUr, *u1);
  } else {
    *u1 = fmin(G.gcon[0][1] * G.alpha, *u1);
  }
  const double U[3] = {*u1, *u2, *u3};
  double vSqr = 0.;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) vSqr += G.gcov[a + 1][b + 1] * U[a] * U[b];
  const double vSqrMax = 1. - 1. / t.MaxLorentzFactor / t.MaxLorentzFactor;
  vSqr = fmax(fmin(vSqr, vSqrMax), 1.e-13);
  const double lf = 1. / sqrt(1. - vSqr);
  *u1 = *u1 * lf;
  *u2 = *u2 * lf;
  *u3 = *u3 * lf;
}

// fixPoles (problem.cpp:1046-1215): one thread per (i, k) column and pole.
// The two rows next to the pole are rebuilt from the third (idx2) and the
// ghost rows mirror those three rows (ghost g from row idx_g, with numGhost
// 3 the only width make_devcfg accepts), so every value a thread writes is a
// function of row idx2's fluid variables, the three rows' field components
// and their theta: all of them are loaded before the first store, and a
// thread waits on memory once instead of once per copied value.  The
// arithmetic is the reference's, value for value.
static __global__ void k_torus_poles(DevCfg c, double* __restrict__ p, const double* __restrict__ geoC) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long cols = (long long)c.N1T * c.N3T;
  if (n >= 2 * cols) return;
  const bool top = n >= cols;
  const long long m = top ? n - cols : n;
  const int i = (int)(m % c.N1T), k = (int)(m / c.N1T);
  const long long Z = c.Z;
  const int ng = c.ng;
  auto at = [&](int v, int j) -> double& { return p[(long long)v * Z + zidx(c, i, j, k)]; };
  auto theta = [&](int j) -> double {
    double th = __ldg(geoC + 35LL * c.GZ + gidx(c, i, j));
    return top ? th * (-1.) + M_PI : th;
  };
  const int idx0 = top ? c.N2 + ng - 1 : ng;
  const int row[3] = {idx0, top ? idx0 - 1 : ng + 1, top ? idx0 - 2 : ng + 2};
  // ---- loads
  double th[3], b1[3], b2[3], b3[3];
#pragma unroll
  for (int g = 0; g < 3; g++) {
    th[g] = theta(row[g]);
    b1[g] = at(c.B1, row[g]);
    b2[g] = at(c.B1 + 1, row[g]);
    b3[g] = at(c.B1 + 2, row[g]);
  }
  const double rho = at(RHO, row[2]), uu = at(UU, row[2]), u1 = at(U1, row[2]), u2 = at(U2, row[2]),
               u3 = at(U3, row[2]);
  const double q = c.conduction ? at(c.Q, row[2]) : 0., dp = c.viscosity ? at(c.DP, row[2]) : 0.;
  // ---- the rows next to the pole (U2, q, deltaP scaled by theta), then
  // the ghost rows
  double su2[3], sq[3], sdp[3];
#pragma unroll
  for (int g = 0; g < 3; g++) {
    su2[g] = g < 2 ? u2 * th[g] / th[2] : u2;
    sq[g] = g < 2 ? q * th[g] / th[2] : q;
    sdp[g] = g < 2 ? dp * th[g] / th[2] : dp;
  }
#pragma unroll
  for (int g = 0; g < 2; g++) {
    const int jj = row[g];
    at(RHO, jj) = rho;
    at(UU, jj) = uu;
    at(U1, jj) = u1;
    at(U2, jj) = su2[g];
    at(U3, jj) = u3;
    if (c.conduction) at(c.Q, jj) = sq[g];
    if (c.viscosity) at(c.DP, jj) = sdp[g];
  }
#pragma unroll
  for (int g = 0; g < 3; g++) {
    const int dst = top ? c.N2 + ng + g : ng - 1 - g;
    at(RHO, dst) = rho;
    at(UU, dst) = uu;
    at(U1, dst) = u1;
    at(U3, dst) = u3;
    at(U2, dst) = su2[g] * (-1.0);
    at(c.B1, dst) = b1[g];
    at(c.B1 + 2, dst) = b3[g];
    at(c.B1 + 1, dst) = b2[g] * (-1.0);
    if (c.conduction) at(c.Q, dst) = sq[g] * (-1.0);
    if (c.viscosity) at(c.DP, dst) = sdp[g] * (-1.0);
  }
}

}  // namespace GRIM_KNS
}  // namespace grim
