// opcount.cuh -- algorithmic flop counts of the Newton kernels' building
// blocks, taken from the code itself: the templated zone physics is
// instantiated on a counting scalar (Cnt<double> / Cnt<float>) and run for
// one zone by one thread.  Every add/subtract, multiply, divide, square root
// and exponential on the counting type is tallied per precision; signs,
// comparisons, min/max and conversions are not flops and are not counted.
// The counts feed the FP64/FP32 pipe rooflines of the Newton and stencil
// kernels.
//
// Included by kernels_fast.cu only (one definition of the tally).
#pragma once

namespace grim {

// [precision: 0 fp64, 1 fp32][op: add, mul, div, sqrt, exp]
__device__ unsigned long long g_op_tally[2][5];

template <class B>
struct Cnt {
  B v;
  static constexpr int P = sizeof(B) == 8 ? 0 : 1;
  GRIM_HD Cnt() : v(0) {}
  GRIM_HD Cnt(double x) : v((B)x) {}
  GRIM_HD Cnt(float x) : v((B)x) {}
  GRIM_HD Cnt(int x) : v((B)x) {}
  GRIM_HD explicit operator double() const { return (double)v; }
  GRIM_HD explicit operator float() const { return (float)v; }
  static GRIM_D void tick(int op) { g_op_tally[P][op]++; }

  friend GRIM_D Cnt operator+(Cnt a, Cnt b) { tick(0); return Cnt(a.v + b.v); }
  friend GRIM_D Cnt operator-(Cnt a, Cnt b) { tick(0); return Cnt(a.v - b.v); }
  friend GRIM_D Cnt operator*(Cnt a, Cnt b) { tick(1); return Cnt(a.v * b.v); }
  friend GRIM_D Cnt operator/(Cnt a, Cnt b) { tick(2); return Cnt(a.v / b.v); }
  friend GRIM_D Cnt operator-(Cnt a) { return Cnt(-a.v); }
  friend GRIM_D Cnt& operator+=(Cnt& a, Cnt b) { a = a + b; return a; }
  friend GRIM_D Cnt& operator-=(Cnt& a, Cnt b) { a = a - b; return a; }
  friend GRIM_D Cnt& operator*=(Cnt& a, Cnt b) { a = a * b; return a; }
  friend GRIM_D Cnt& operator/=(Cnt& a, Cnt b) { a = a / b; return a; }
  friend GRIM_D bool operator<(Cnt a, Cnt b) { return a.v < b.v; }
  friend GRIM_D bool operator>(Cnt a, Cnt b) { return a.v > b.v; }
  friend GRIM_D bool operator<=(Cnt a, Cnt b) { return a.v <= b.v; }
  friend GRIM_D bool operator>=(Cnt a, Cnt b) { return a.v >= b.v; }
  friend GRIM_D bool operator==(Cnt a, Cnt b) { return a.v == b.v; }
  friend GRIM_D bool operator!=(Cnt a, Cnt b) { return a.v != b.v; }

  // the scalar helpers the physics calls (found by argument lookup)
  friend GRIM_D Cnt val(Cnt a) { return a; }
  friend GRIM_D Cnt dsqrt(Cnt a) { tick(3); return Cnt(sqrt((double)a.v)); }
  friend GRIM_D Cnt drsqrt(Cnt a) { tick(3); return Cnt(1. / sqrt((double)a.v)); }
  friend GRIM_D Cnt dexp(Cnt a) { tick(4); return Cnt(exp((double)a.v)); }
  friend GRIM_D Cnt dfabs(Cnt a) { return Cnt(a.v < B(0) ? -a.v : a.v); }
  friend GRIM_D Cnt fabs(Cnt a) { return dfabs(a); }
  friend GRIM_D Cnt dmaxc(Cnt a, Cnt b) { return a.v >= b.v ? a : b; }
  friend GRIM_D Cnt dmin2(Cnt a, Cnt b) { return a.v <= b.v ? a : b; }
  friend GRIM_D Cnt dmax2(Cnt a, Cnt b) { return a.v >= b.v ? a : b; }
  friend GRIM_D Cnt dcube(Cnt a) { return a * a * a; }
  friend GRIM_D Cnt fmin(Cnt a, Cnt b) { return a.v <= b.v ? a : b; }
  friend GRIM_D Cnt fmax(Cnt a, Cnt b) { return a.v >= b.v ? a : b; }
  friend GRIM_D Cnt copysign(Cnt a, Cnt b) { return Cnt(::copysign((double)a.v, (double)b.v)); }
  friend GRIM_D bool isfinite(Cnt a) { return ::isfinite((double)a.v); }
};

// the value of a counted scalar (the closures read the geometry's values)
template <class B>
GRIM_HD double val_of(const Cnt<B>& x) { return (double)x.v; }

template <class B>
struct Lift<Cnt<B>> {
  GRIM_HD static Cnt<B> of(double x) { return Cnt<B>(x); }
};

namespace GRIM_KNS {

// One thread, one zone z of the stage buffers b (filled by a stage set-up):
// out = {residual fp64, Jacobian(fp32) fp32, Jacobian(fp64) fp64,
//        solve fp32, solve fp64, residual divides, residual sqrt+exp,
//        generic forward-tangent pass fp32, reconstruction of one zone
//        along one direction (all dof), Riemann solve of one face,
//        epilogue centre work of one zone (element, conserved vector,
//        geometric source contraction; CT and divergence not counted)};
// the Jacobian is the closed form for ideal MHD and the forward tangent
// otherwise
template <int COND, int VISC>
__global__ void k_count_ops(DevCfg c, int stage, StageBufs b, long long z, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  constexpr int NF = 5 + COND + VISC;
  const long long Z = c.Z;
  int i, j, k;
  zijk(c, z, i, j, k);
  ZoneGeo<double> G;
  load_geo(G, c, b.geoC, z, i, j, 0.5, 0.5);
  StageConst<NF> K;
  load_stage_const<COND, VISC>(K, c, stage, b, z, G);
  auto clear = [] {
    for (int p = 0; p < 2; p++)
      for (int o = 0; o < 5; o++) g_op_tally[p][o] = 0;
  };
  auto flops = [](int p) {
    return (double)(g_op_tally[p][0] + g_op_tally[p][1] + g_op_tally[p][2] + g_op_tally[p][3] +
                    g_op_tally[p][4]);
  };
  double Pd[NF];
  for (int v = 0; v < NF; v++) Pd[v] = b.prim[(long long)v * Z + z];
  // residual, FP64
  {
    typedef Cnt<double> C8;
    ZoneGeo<C8> Gc;
    for (int m = 0; m < 4; m++)
      for (int q = 0; q < 4; q++) { Gc.gcov[m][q] = C8(G.gcov[m][q]); Gc.gcon[m][q] = C8(G.gcon[m][q]); }
    Gc.g = C8(G.g); Gc.alpha = C8(G.alpha); Gc.ialpha = C8(G.ialpha); Gc.x1 = C8(G.x1); Gc.x2 = C8(G.x2); Gc.dyn = C8(G.dyn);
    C8 P[NF], R[NF];
    for (int v = 0; v < NF; v++) P[v] = C8(Pd[v]);
    clear();
    zone_residual<COND, VISC, C8, C8>(P, K, Gc, c, R);
    out[0] = flops(0);
    out[5] = (double)g_op_tally[0][2];
    out[6] = (double)(g_op_tally[0][3] + g_op_tally[0][4]);
  }
  // tangent pass in FP32 and in FP64
  {
    typedef Cnt<float> C4;
    ZoneGeo<C4> Gt;
    for (int m = 0; m < 4; m++)
      for (int q = 0; q < 4; q++) { Gt.gcov[m][q] = C4(G.gcov[m][q]); Gt.gcon[m][q] = C4(G.gcon[m][q]); }
    Gt.g = C4(G.g); Gt.alpha = C4(G.alpha); Gt.ialpha = C4(G.ialpha); Gt.x1 = C4(G.x1); Gt.x2 = C4(G.x2); Gt.dyn = C4(G.dyn);
    C4 J[NF][NF];
    clear();
    tangent_jacobian<COND, VISC, C4, true>(Pd, K, Gt, c, J);
    out[7] = flops(1);  // the generic forward-tangent pass
    clear();
    tangent_jacobian<COND, VISC, C4>(Pd, K, Gt, c, J);
    out[1] = flops(1);
    C4 bv[NF], xv[NF];
    for (int v = 0; v < NF; v++) bv[v] = C4(1.0);
    clear();
    gauss_solve<C4, NF>(J, bv, xv);
    out[3] = flops(1);
  }
  {
    typedef Cnt<double> C8;
    ZoneGeo<C8> Gt;
    for (int m = 0; m < 4; m++)
      for (int q = 0; q < 4; q++) { Gt.gcov[m][q] = C8(G.gcov[m][q]); Gt.gcon[m][q] = C8(G.gcon[m][q]); }
    Gt.g = C8(G.g); Gt.alpha = C8(G.alpha); Gt.ialpha = C8(G.ialpha); Gt.x1 = C8(G.x1); Gt.x2 = C8(G.x2); Gt.dyn = C8(G.dyn);
    C8 J[NF][NF];
    clear();
    tangent_jacobian<COND, VISC, C8>(Pd, K, Gt, c, J);
    out[2] = flops(0);
    C8 bv[NF], xv[NF];
    for (int v = 0; v < NF; v++) bv[v] = C8(1.0);
    clear();
    gauss_solve<C8, NF>(J, bv, xv);
    out[4] = flops(0);
  }
  // stencil work, FP64
  {
    typedef Cnt<double> C8;
    constexpr int DOF = NF + 3;
    ZoneGeo<C8> Gc;
    for (int m = 0; m < 4; m++)
      for (int q = 0; q < 4; q++) { Gc.gcov[m][q] = C8(G.gcov[m][q]); Gc.gcon[m][q] = C8(G.gcon[m][q]); }
    Gc.g = C8(G.g); Gc.alpha = C8(G.alpha); Gc.ialpha = C8(G.ialpha); Gc.x1 = C8(G.x1); Gc.x2 = C8(G.x2); Gc.dyn = C8(G.dyn);
    const double* ps = b.ps;
    // reconstruction of every dof of the zone along X1
    clear();
    C8 lo[DOF], ro[DOF];
    for (int v = 0; v < DOF; v++) {
      const double* a = ps + (long long)v * Z + z;
      recon_faces_fast<C8>(c.reconstruction, c.theta, C8(a[-2]), C8(a[-1]), C8(a[0]), C8(a[1]), C8(a[2]), lo[v],
                           ro[v]);
    }
    out[8] = flops(0);
    // one face: both states through the element, fluxes along X1 and X0,
    // characteristic speeds, then the HLL / LLF combination
    clear();
    C8 F[2][DOF], U[2][DOF], mn[2], mx[2];
    for (int side = 0; side < 2; side++) {
      const C8* q = side ? lo : ro;
      ElemT<C8, C8> e;
      elem_set<COND, VISC>(e, q[0], q[1], q[2], q[3], q[4], q[NF], q[NF + 1], q[NF + 2], COND ? q[5] : C8(0.),
                           VISC ? q[5 + COND] : C8(0.), Gc, c);
      fluxes_fluid<COND, VISC>(e, 1, Gc.g, F[side], 5, 5 + COND);
      fluxes_B(e, 1, Gc.g, F[side] + NF);
      fluxes_fluid<COND, VISC>(e, 0, Gc.g, U[side], 5, 5 + COND);
      fluxes_B(e, 0, Gc.g, U[side] + NF);
      char_speeds<COND, VISC>(e, Gc, 0, c, mn[side], mx[side]);
    }
    const C8 cmin = mn[0] <= mn[1] ? mn[0] : mn[1], cmax = mx[0] >= mx[1] ? mx[0] : mx[1];
    C8 fl[DOF];
    if (c.riemann == GRIM_HLL) {
      const C8 id = C8(1.) / (cmax - cmin);
      for (int v = 0; v < DOF; v++)
        fl[v] = (cmax * F[0][v] - cmin * F[1][v] + cmin * cmax * (U[1][v] - U[0][v])) * id;
    } else {
      const C8 cm = cmax >= -cmin ? cmax : -cmin;
      for (int v = 0; v < DOF; v++) fl[v] = C8(0.5) * (F[0][v] + F[1][v] - cm * (U[1][v] - U[0][v]));
    }
    out[9] = flops(0);
    // epilogue centre: element, conserved vector, -g T^k_l Gamma^l_kn
    clear();
    {
      ElemT<C8, C8> e;
      elem_set<COND, VISC>(e, C8(ps[z]), C8(ps[Z + z]), C8(ps[2 * Z + z]), C8(ps[3 * Z + z]), C8(ps[4 * Z + z]),
                           C8(ps[(long long)c.B1 * Z + z]), C8(ps[(long long)(c.B1 + 1) * Z + z]),
                           C8(ps[(long long)(c.B1 + 2) * Z + z]), C8(0.), C8(0.), Gc, c);
      C8 Uc[NF], UB[3];
      fluxes_fluid<COND, VISC>(e, 0, Gc.g, Uc, 5, 5 + COND);
      fluxes_B(e, 0, Gc.g, UB);
      if (c.metric != GRIM_MINKOWSKI) {
        C8 T[4][4];
        for (int ka = 0; ka < 4; ka++)
          for (int la = 0; la < 4; la++) T[ka][la] = tmunu<COND, VISC>(e, ka, la);
        C8 S[4];
        for (int nu = 0; nu < 4; nu++) {
          S[nu] = C8(0.);
          for (int ka = 0; ka < 4; ka++)
            for (int la = 0; la < 4; la++) S[nu] = S[nu] - Gc.g * T[ka][la] * C8(1.);
        }
        (void)S;
      }
    }
    out[10] = flops(0);
  }
}

template <int C, int V>
static void count_ops_t(const DevCfg& c, int stage, const StageBufs& b, long long z, double* out,
                        cudaStream_t s) {
  k_count_ops<C, V><<<1, 32, 0, s>>>(c, stage, b, z, out);
}
void count_ops(const DevCfg& c, int stage, const StageBufs& b, long long z, double* out, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, count_ops_t, c, stage, b, z, out, s);
}

}  // namespace GRIM_KNS
}  // namespace grim
