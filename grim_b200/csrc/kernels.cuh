// kernels.cuh -- the CUDA kernels of one implicit timestep.
//
// Included by two translation units: kernels_exact.cu (--fmad=false, the
// FP64 operation order of the reference, used by the parity path) and
// kernels_fast.cu (FMA contraction on, used by the tangent / mixed paths).
// Each defines GRIM_KNS to put its instantiations in its own namespace.
//
// Per stage:
//   k_ghost_fill       ghost zones <- interior (periodic wrap, outflow,
//                      mirror; boundary.cpp:5-241 + grid.cpp:306-315)
//   k_emhd_prepass     u_mu and T of the stage element per zone (EMHD only)
//   k_face_flux(dir)   reconstruction + two face elements + HLL/LLF, one
//                      thread per face (fvmfluxes.cpp, riemannsolver.cpp)
//   k_stage_epilogue   EMFs + flux-CT + divergence + induction + explicit
//                      sources + consOld, per interior zone
//   k_dt_speeds        max over zones of sum_d c_max,d / dX_d (computeDt)
//   k_newton_*         per-zone Newton (solve.cpp / residual.cpp)
#pragma once
#include <algorithm>

#include "physics.cuh"
#include "recon.cuh"
#include "stage.cuh"
#include "torus.cuh"

namespace grim {
namespace GRIM_KNS {

#ifdef GRIM_FAST_MATH
constexpr bool kFastMath = true;   // reassociated arithmetic allowed (fast path)
#else
constexpr bool kFastMath = false;  // the reference's operation order (parity path)
#endif


// ---------------------------------------------------------------------------
// ghost fill: composite gather (every ghost zone reads the interior zone
// that the wrap / outflow / mirror maps of each direction select)
// ---------------------------------------------------------------------------
GRIM_D int bc_map(int x, int g, int N, int lo, int hi) {
  if (x >= g && x < N + g) return x;
  if ((x < g && lo == GRIM_EXCHANGE) || (x >= N + g && hi == GRIM_EXCHANGE)) return x;  // the caller's halo
  if (x < g) {
    if (lo == GRIM_PERIODIC) return g + ((x - g) % N + N) % N;
    if (lo == GRIM_MIRROR) return 2 * g - 1 - x;
    return g;  // outflow
  }
  if (hi == GRIM_PERIODIC) return g + ((x - g) % N + N) % N;
  if (hi == GRIM_MIRROR) return 2 * (N + g) - 1 - x;
  return N + g - 1;
}

// boundaries::applyBoundaryConditions (boundary.cpp:5-241): outflow and
// mirror only; periodic directions are left as they are (the reference fills
// them in grid::communicate at the end of each stage).  Applied direction by
// direction over full spans, its result is the gather below.
// the n-th ghost zone: the X1 ghost columns (all j, k), then the X2 ghost
// rows of the X1 interior (all k), then the X3 ghost planes of the X1 / X2
// interior; n < Z - Zint
GRIM_D void ghost_ijk(const DevCfg& c, long long n, int& i, int& j, int& k) {
  const long long a = 2LL * c.g1 * c.N2T * c.N3T, b = (long long)c.N1 * 2 * c.g2 * c.N3T;
  if (n < a) {
    const int gi = (int)(n % (2 * c.g1));
    const long long r = n / (2 * c.g1);
    i = gi < c.g1 ? gi : c.N1 + gi;
    j = (int)(r % c.N2T);
    k = (int)(r / c.N2T);
  } else if (n < a + b) {
    const long long m = n - a;
    i = c.g1 + (int)(m % c.N1);
    const long long r = m / c.N1;
    const int gj = (int)(r % (2 * c.g2));
    j = gj < c.g2 ? gj : c.N2 + gj;
    k = (int)(r / (2 * c.g2));
  } else {
    const long long m = n - a - b;
    i = c.g1 + (int)(m % c.N1);
    const long long r = m / c.N1;
    j = c.g2 + (int)(r % c.N2);
    const int gk = (int)(r / c.N2);
    k = gk < c.g3 ? gk : c.N3 + gk;
  }
}

// one thread per ghost zone
static __global__ void k_ghost_fill(DevCfg c, double* __restrict__ prim, int nv) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Z - c.Zint) return;
  int i, j, k;
  ghost_ijk(c, n, i, j, k);
  const long long z = zidx(c, i, j, k);
  const bool p1 = c.bc[0] == GRIM_PERIODIC || c.bc[1] == GRIM_PERIODIC;
  const bool p2 = c.bc[2] == GRIM_PERIODIC || c.bc[3] == GRIM_PERIODIC;
  const bool p3 = c.bc[4] == GRIM_PERIODIC || c.bc[5] == GRIM_PERIODIC;
  int si = p1 ? i : bc_map(i, c.g1, c.N1, c.bc[0], c.bc[1]);
  int sj = (c.dim >= 2 && !p2) ? bc_map(j, c.g2, c.N2, c.bc[2], c.bc[3]) : j;
  int sk = (c.dim >= 3 && !p3) ? bc_map(k, c.g3, c.N3, c.bc[4], c.bc[5]) : k;
  if (si == i && sj == j && sk == k) return;
  long long s = zidx(c, si, sj, sk);
  for (int v = 0; v < nv; v++) prim[(long long)v * c.Z + z] = prim[(long long)v * c.Z + s];
}

// grid::communicate (grid.cpp:306-360) with PETSc DMDA semantics: periodic
// ghost zones (corners included) take the wrapped interior value; ghost
// zones on a non-periodic edge come back from the never-written local
// vector, i.e. as zero.
// the zone communicate reads for zone (i, j, k): itself inside, the wrapped
// interior zone across a periodic edge; zero is set on a non-periodic edge.
// A GRIM_EXCHANGE side keeps its own ghost value (the caller's halo).
GRIM_D long long comm_source(const DevCfg& c, int i, int j, int k, bool& zero) {
  const bool p1 = c.bc[0] == GRIM_PERIODIC || c.bc[1] == GRIM_PERIODIC;
  const bool p2 = c.bc[2] == GRIM_PERIODIC || c.bc[3] == GRIM_PERIODIC;
  const bool p3 = c.bc[4] == GRIM_PERIODIC || c.bc[5] == GRIM_PERIODIC;
  zero = false;
  auto m = [&](int x, int g, int N, bool per, int lo, int hi) -> int {
    if (x >= g && x < N + g) return x;
    if ((x < g && lo == GRIM_EXCHANGE) || (x >= N + g && hi == GRIM_EXCHANGE)) return x;
    if (!per) { zero = true; return x; }
    return g + ((x - g) % N + N) % N;
  };
  const int si = m(i, c.g1, c.N1, p1, c.bc[0], c.bc[1]);
  const int sj = (c.dim >= 2) ? m(j, c.g2, c.N2, p2, c.bc[2], c.bc[3]) : j;
  const int sk = (c.dim >= 3) ? m(k, c.g3, c.N3, p3, c.bc[4], c.bc[5]) : k;
  return zidx(c, si, sj, sk);
}
// a ghost zone on a GRIM_EXCHANGE side: it repeats a neighbouring slab's
// interior, which that slab's own reductions count
GRIM_D bool in_exchange_ghost(const DevCfg& c, int i, int j, int k) {
  const bool x1 = (i < c.g1 && c.bc[0] == GRIM_EXCHANGE) || (i >= c.N1 + c.g1 && c.bc[1] == GRIM_EXCHANGE);
  const bool x2 = c.dim >= 2 && ((j < c.g2 && c.bc[2] == GRIM_EXCHANGE) || (j >= c.N2 + c.g2 && c.bc[3] == GRIM_EXCHANGE));
  const bool x3 = c.dim >= 3 && ((k < c.g3 && c.bc[4] == GRIM_EXCHANGE) || (k >= c.N3 + c.g3 && c.bc[5] == GRIM_EXCHANGE));
  return x1 || x2 || x3;
}

static __global__ void k_communicate(DevCfg c, double* __restrict__ prim, int nv) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  bool zero;
  const long long s = comm_source(c, i, j, k, zero);
  if (!zero && s == z) return;
  for (int v = 0; v < nv; v++) prim[(long long)v * c.Z + z] = zero ? 0. : prim[(long long)v * c.Z + s];
}

// ---------------------------------------------------------------------------
// computeDivB (constrainedtransport.cpp:85-110): corner divergence of
// sqrt(-g) B in 2D from ArrayFire's circular shifts over the whole array,
// ghosts included; zero in 1D and 3D, where the reference writes nothing
// ---------------------------------------------------------------------------
static __global__ void k_divb(DevCfg c, const double* __restrict__ p, const double* __restrict__ geoC,
                              double* __restrict__ out) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  if (c.dim != 2) { out[z] = 0.; return; }
  int i, j, k;
  zijk(c, z, i, j, k);
  auto gB = [&](int v, int ii, int jj) -> double {
    ii = (ii + c.N1T) % c.N1T;
    jj = (jj + c.N2T) % c.N2T;
    const double g = geoC ? __ldg(geoC + 32LL * c.GZ + gidx(c, ii, jj)) : 1.;
    return g * p[(long long)(c.B1 + v) * c.Z + zidx(c, ii, jj, k)];
  };
  const double a = gB(0, i, j), a01 = gB(0, i, j - 1), a10 = gB(0, i - 1, j), a11 = gB(0, i - 1, j - 1);
  const double b = gB(1, i, j), b10 = gB(1, i - 1, j), b01 = gB(1, i, j - 1), b11 = gB(1, i - 1, j - 1);
  out[z] = (a + a01 - a10 - a11) / (2. * c.dX[0]) + (b + b10 - b01 - b11) / (2. * c.dX[1]);
}

// ---------------------------------------------------------------------------
// EMHD pre-pass: u_mu and T of the stage element at every zone
// ---------------------------------------------------------------------------
template <int COND, int VISC>
__global__ void k_emhd_prepass(DevCfg c, const double* __restrict__ ps, const double* __restrict__ geoC,
                                        double* __restrict__ uT) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  ZoneGeo<double> G;
  load_geo(G, c, geoC, z, i, j, 0.5, 0.5);
  const long long Z = c.Z;
  ElemT<double, double> e;
  elem_set<COND, VISC>(e, ps[z], ps[Z + z], ps[2 * Z + z], ps[3 * Z + z], ps[4 * Z + z],
                       ps[(long long)c.B1 * Z + z], ps[(long long)(c.B1 + 1) * Z + z],
                       ps[(long long)(c.B1 + 2) * Z + z], COND ? ps[(long long)c.Q * Z + z] : 0.,
                       VISC ? ps[(long long)c.DP * Z + z] : 0., G, c);
#pragma unroll
  for (int m = 0; m < 4; m++) uT[(long long)m * Z + z] = e.uCov[m];
  uT[4 * Z + z] = e.temperature;
}

// ---------------------------------------------------------------------------
// face fluxes (riemannsolver.cpp:202-328 after its shift): the flux through
// the face z - 1/2 along `dir` from the left state (right face value of zone
// z - s) and the right state (left face value of zone z).  Every zone is
// reconstructed once per direction and handed to its neighbour by a warp
// shuffle: X1 faces take 31 faces per warp along i, X2 / X3 faces 7 faces
// along the direction for each of 4 consecutive i.
// ---------------------------------------------------------------------------
template <int DOF, int RS>
GRIM_D void recon_zone_rs(const DevCfg& c, const double* __restrict__ ps, long long z, long long s, double* lo,
                          double* ro) {
#pragma unroll
  for (int v = 0; v < DOF; v++) {
    const double* a = ps + (long long)v * c.Z + z;
    const double y0 = __ldg(a - 2 * s), y1 = __ldg(a - s), y2 = __ldg(a), y3 = __ldg(a + s), y4 = __ldg(a + 2 * s);
    recon_faces_rs<RS, kFastMath>(c.reconstruction, c.theta, y0, y1, y2, y3, y4, lo[v], ro[v]);
  }
}
// the scheme is chosen once, outside the loop over the variables, so the
// path a warp executes is one scheme's contiguous code
template <int DOF>
GRIM_D void recon_zone(const DevCfg& c, const double* __restrict__ ps, long long z, long long s, int scheme,
                       double* lo, double* ro) {
  switch (scheme) {
    case GRIM_WENO5: recon_zone_rs<DOF, GRIM_WENO5>(c, ps, z, s, lo, ro); break;
    case GRIM_PPM: recon_zone_rs<DOF, GRIM_PPM>(c, ps, z, s, lo, ro); break;
    case GRIM_MP5: recon_zone_rs<DOF, GRIM_MP5>(c, ps, z, s, lo, ro); break;
    default: recon_zone_rs<DOF, GRIM_MINMOD>(c, ps, z, s, lo, ro); break;
  }
}

// Shared memory holds what waits: the right face state (slot 2, put there
// by the caller) while the left element is evaluated, then the left
// state's fluxes (slots 0, 1) while the right element is; slot [v][thread],
// 3 x DOF doubles per thread.  Neither holds registers across an element.
template <int COND, int VISC>
GRIM_D void riemann_face(const DevCfg& c, int dir, const double* pl, const ZoneGeo<double>& G,
                         double* __restrict__ flux, long long z, double* __restrict__ park) {
  constexpr int NF = 5 + COND + VISC;
  constexpr int DOF = NF + 3;
  const long long Z = c.Z;
  const int fd = dir + 1;
  const int nt = blockDim.x, t = threadIdx.x;
  double minL, maxL;
  {
    double F[DOF], U[DOF];
    ElemT<double, double> e;
    elem_set<COND, VISC>(e, pl[0], pl[1], pl[2], pl[3], pl[4], pl[NF], pl[NF + 1], pl[NF + 2],
                         COND ? pl[5] : 0., VISC ? pl[5 + COND] : 0., G, c);
    fluxes_fluid<COND, VISC>(e, fd, G.g, F, 5, 5 + COND);
    fluxes_B(e, fd, G.g, F + NF);
    fluxes_fluid<COND, VISC>(e, 0, G.g, U, 5, 5 + COND);
    fluxes_B(e, 0, G.g, U + NF);
    char_speeds<COND, VISC>(e, G, dir, c, minL, maxL);
#pragma unroll
    for (int v = 0; v < DOF; v++) {
      park[v * nt + t] = F[v];
      park[(DOF + v) * nt + t] = U[v];
    }
  }
  double F[DOF], U[DOF], minR, maxR;
  {
    double pr[DOF];
#pragma unroll
    for (int v = 0; v < DOF; v++) pr[v] = park[(2 * DOF + v) * nt + t];
    ElemT<double, double> e;
    elem_set<COND, VISC>(e, pr[0], pr[1], pr[2], pr[3], pr[4], pr[NF], pr[NF + 1], pr[NF + 2],
                         COND ? pr[5] : 0., VISC ? pr[5 + COND] : 0., G, c);
    fluxes_fluid<COND, VISC>(e, fd, G.g, F, 5, 5 + COND);
    fluxes_B(e, fd, G.g, F + NF);
    fluxes_fluid<COND, VISC>(e, 0, G.g, U, 5, 5 + COND);
    fluxes_B(e, 0, G.g, U + NF);
    char_speeds<COND, VISC>(e, G, dir, c, minR, maxR);
  }
  const double cmin = fmin(minL, minR);
  const double cmax = fmax(maxL, maxR);
  if (c.riemann == GRIM_HLL) {
    const double id = 1. / (cmax - cmin);
#pragma unroll
    for (int v = 0; v < DOF; v++) {
      const double FL = park[v * nt + t], UL = park[(DOF + v) * nt + t];
      const double num = cmax * FL - cmin * F[v] + cmin * cmax * (U[v] - UL);
      flux[(long long)v * Z + z] = kFastMath ? num * id : num / (cmax - cmin);
    }
  } else {
    const double cm = fmax(cmax, -cmin);
#pragma unroll
    for (int v = 0; v < DOF; v++) {
      const double FL = park[v * nt + t], UL = park[(DOF + v) * nt + t];
      flux[(long long)v * Z + z] = 0.5 * (FL + F[v] - cm * (U[v] - UL));
    }
  }
}

// The same face flux with both states' elements evaluated side by side
// (no shared-memory parking): twice the independent arithmetic per thread
// for more registers, which the autotuner weighs against occupancy.
template <int COND, int VISC>
GRIM_D void riemann_face_pair(const DevCfg& c, int dir, const double* pl, const double* pr,
                              const ZoneGeo<double>& G, double* __restrict__ flux, long long z) {
  constexpr int NF = 5 + COND + VISC;
  constexpr int DOF = NF + 3;
  const long long Z = c.Z;
  const int fd = dir + 1;
  double F[2][DOF], U[2][DOF], mn[2], mx[2];
  ElemT<double, double> e[2];
#pragma unroll
  for (int sd = 0; sd < 2; sd++) {
    const double* q = sd ? pr : pl;
    elem_set<COND, VISC>(e[sd], q[0], q[1], q[2], q[3], q[4], q[NF], q[NF + 1], q[NF + 2], COND ? q[5] : 0.,
                         VISC ? q[5 + COND] : 0., G, c);
  }
#pragma unroll
  for (int sd = 0; sd < 2; sd++) {
    fluxes_fluid<COND, VISC>(e[sd], fd, G.g, F[sd], 5, 5 + COND);
    fluxes_B(e[sd], fd, G.g, F[sd] + NF);
    fluxes_fluid<COND, VISC>(e[sd], 0, G.g, U[sd], 5, 5 + COND);
    fluxes_B(e[sd], 0, G.g, U[sd] + NF);
    char_speeds<COND, VISC>(e[sd], G, dir, c, mn[sd], mx[sd]);
  }
  const double cmin = fmin(mn[0], mn[1]);
  const double cmax = fmax(mx[0], mx[1]);
  if (c.riemann == GRIM_HLL) {
    const double id = 1. / (cmax - cmin);
#pragma unroll
    for (int v = 0; v < DOF; v++) {
      const double num = cmax * F[0][v] - cmin * F[1][v] + cmin * cmax * (U[1][v] - U[0][v]);
      flux[(long long)v * Z + z] = kFastMath ? num * id : num / (cmax - cmin);
    }
  } else {
    const double cm = fmax(cmax, -cmin);
#pragma unroll
    for (int v = 0; v < DOF; v++) flux[(long long)v * Z + z] = 0.5 * (F[0][v] + F[1][v] - cm * (U[1][v] - U[0][v]));
  }
}

// X1 faces: warp w of a row covers faces i0 .. i0+30; lane l reconstructs
// zone i0 - 1 + l and, for l >= 1, computes the face between zones
// i0 - 2 + l and i0 - 1 + l with the left state shuffled from lane l - 1.
template <int COND, int VISC, int MINB, bool PAIR, int RS>
__global__ void __launch_bounds__(128, MINB) k_face_flux_x1(DevCfg c, const double* __restrict__ ps,
                                                      const double* __restrict__ geoF, double* __restrict__ flux) {
  constexpr int DOF = 8 + COND + VISC;
  const int lane = threadIdx.x & 31;
  const long long wg = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nfaces = c.N1T - 5;  // faces i = 3 .. N1T-3
  const int wpr = (nfaces + 30) / 31;
  const long long rows = (long long)c.nfj * c.nfk;
  if (wg >= rows * wpr) return;  // whole warps exit together
  const unsigned wgu = (unsigned)wg, row = wgu / (unsigned)wpr;
  const int i0 = 3 + (int)(wgu - row * (unsigned)wpr) * 31;
  const int iz = i0 - 1 + lane;
  const unsigned rk = row / (unsigned)c.nfj;
  const int k = c.fk0 + (int)rk, j = c.fj0 + (int)(row - rk * (unsigned)c.nfj);
  const bool reconOK = iz >= 2 && iz <= c.N1T - 3;
  double lo[DOF], ro[DOF];
  const long long z = zidx(c, reconOK ? iz : 2, j, k);
  recon_zone_rs<DOF, RS>(c, ps, z, 1, lo, ro);
  double pl[DOF];
#pragma unroll
  for (int v = 0; v < DOF; v++) pl[v] = __shfl_up_sync(0xffffffffu, ro[v], 1);
  if (lane == 0 || iz > c.N1T - 3) return;
  ZoneGeo<double> G;
  load_geo(G, c, geoF, z, iz, j, 0., 0.5);
  if constexpr (PAIR) {
    riemann_face_pair<COND, VISC>(c, 0, pl, lo, G, flux, z);
  } else {
    extern __shared__ double park_x1[];
#pragma unroll
    for (int v = 0; v < DOF; v++) park_x1[(2 * DOF + v) * blockDim.x + threadIdx.x] = lo[v];
    riemann_face<COND, VISC>(c, 0, pl, G, flux, z, park_x1);
  }
}

// ---------------------------------------------------------------------------
// X1 faces with TMA-staged rows.  Persistent warps walk over the 31-face row
// segments; while a warp computes one segment, the tensor-memory accelerator
// copies the next segment's primitives (all dof, 40 zones along i) into the
// warp's other shared-memory buffer, so the stencil loads come from shared
// memory.  The tensor map covers the prim array as (i, j, k, var).  Waits
// on the copy barrier are bounded in time (kCopyWaitNs): a wait that gives up
// counts in DevState::waitTimeouts, raises the handle's host-visible error
// word, and the warp stops once every copy it issued has landed (itself a
// bounded wait; one that gives up too counts in DevState::drainTimeouts).
// ---------------------------------------------------------------------------
constexpr int kX1Box = 40;  // zones per TMA row box (x rounded down to even)

GRIM_D unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
GRIM_D void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
GRIM_D void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
GRIM_D void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
GRIM_D bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
GRIM_D unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// A copy of one row box lands within microseconds; a wait that lasts this
// long means the copy will not complete.
constexpr unsigned long long kCopyWaitNs = 1000000000ull;  // 1 s
// bounded wait: false when the barrier did not complete within kCopyWaitNs
// (or, should the global timer not advance, 2^26 polls)
GRIM_D bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (int spin = 0; spin < (1 << 26); spin++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kCopyWaitNs) break;
  }
  return false;
}
// The give-up path of a warp whose copy wait ran out (lane 0): count it,
// raise the host-visible error word, then wait (bounded) for each copy the
// warp still has in flight so none lands after the warp has stopped.
GRIM_D void copy_wait_gave_up(DevState* st, unsigned long long* bars, const bool inflight[2],
                              const unsigned phase[2]) {
  atomicAdd(&st->waitTimeouts, 1ULL);
  for (int b = 0; b < 2; b++)
    if (inflight[b] && !mbar_wait_bounded(&bars[b], phase[b])) atomicAdd(&st->drainTimeouts, 1ULL);
  if (st->hostError) {
    *(volatile unsigned*)st->hostError = 1u;
    __threadfence_system();
  }
}
GRIM_D void tma_load_4d(void* dst, const CUtensorMap* map, unsigned long long* bar, int x, int y, int z, int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}

template <int COND, int VISC, int MINB, int RS, bool PAIR>
__global__ void __launch_bounds__(128, MINB) k_face_flux_x1_tma(const __grid_constant__ CUtensorMap tmap, DevCfg c,
                                                                 const double* __restrict__ geoF,
                                                                 double* __restrict__ flux, DevState* st) {
  constexpr int DOF = 8 + COND + VISC;
  constexpr int ROW = DOF * kX1Box;  // doubles per row buffer (a multiple of 128 bytes)
  extern __shared__ __align__(128) double smem_x1[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double* rows = smem_x1 + (size_t)w * 2 * ROW;
  double* park = smem_x1 + (size_t)nw * 2 * ROW;
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(park + 3 * DOF * blockDim.x) + 2 * w;
  const int nfaces = c.N1T - 5;  // faces i = 3 .. N1T-3
  const int wpr = (nfaces + 30) / 31;
  const long long nitems = (long long)c.nfj * c.nfk * wpr;
  const long long stride = (long long)gridDim.x * nw;
  long long item = (long long)blockIdx.x * nw + w;
  if (lane == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncwarp();
  auto decompose = [&](long long it, int& i0, int& j, int& k) {
    const unsigned itu = (unsigned)it, row = itu / (unsigned)wpr;
    i0 = 3 + (int)(itu - row * (unsigned)wpr) * 31;
    const unsigned rk = row / (unsigned)c.nfj;
    k = c.fk0 + (int)rk;
    j = c.fj0 + (int)(row - rk * (unsigned)c.nfj);
  };
  // lane 0's record of the copies it issued and not yet seen land (the
  // debug setting dbgSkipCopies issues none, so the waits run out)
  bool inflight[2] = {false, false};
  unsigned phase[2] = {0u, 0u};
  auto issue = [&](long long it, int buf) {
    if (c.dbgSkipCopies) return;
    int i0, j, k;
    decompose(it, i0, j, k);
    mbar_expect_tx(&bars[buf], ROW * (unsigned)sizeof(double));
    tma_load_4d(rows + buf * ROW, &tmap, &bars[buf], (i0 - 3) & ~1, j, k, 0);
    inflight[buf] = true;
  };
  if (lane == 0 && item < nitems) issue(item, 0);
  int buf = 0;
  for (; item < nitems; item += stride, buf ^= 1) {
    const long long next = item + stride;
    if (lane == 0 && next < nitems) issue(next, buf ^ 1);
    const bool arrived = mbar_wait_bounded(&bars[buf], phase[buf]);
    if (!__all_sync(0xffffffffu, arrived)) {
      if (lane == 0) copy_wait_gave_up(st, bars, inflight, phase);
      __syncwarp();
      return;
    }
    phase[buf] ^= 1u;
    inflight[buf] = false;
    int i0, j, k;
    decompose(item, i0, j, k);
    const int x0 = (i0 - 3) & ~1;
    const int iz = i0 - 1 + lane;
    const bool reconOK = iz >= 2 && iz <= c.N1T - 3;
    const int iu = reconOK ? iz : i0 - 1;  // a zone inside the buffer
    const double* rb = rows + buf * ROW;
    double lo[DOF], ro[DOF];
#pragma unroll
    for (int v = 0; v < DOF; v++) {
      const double* a = rb + v * kX1Box + (iu - x0);
      recon_faces_rs<RS, kFastMath>(c.reconstruction, c.theta, a[-2], a[-1], a[0], a[1], a[2], lo[v], ro[v]);
    }
    __syncwarp();  // the buffer is read; it may be refilled two items on
    double pl[DOF];
#pragma unroll
    for (int v = 0; v < DOF; v++) pl[v] = __shfl_up_sync(0xffffffffu, ro[v], 1);
    if (lane > 0 && reconOK) {
      const long long z = zidx(c, iz, j, k);
      ZoneGeo<double> G;
      load_geo(G, c, geoF, z, iz, j, 0., 0.5);
      if constexpr (PAIR) {
        riemann_face_pair<COND, VISC>(c, 0, pl, lo, G, flux, z);
      } else {
#pragma unroll
        for (int v = 0; v < DOF; v++) park[(2 * DOF + v) * blockDim.x + threadIdx.x] = lo[v];
        riemann_face<COND, VISC>(c, 0, pl, G, flux, z, park);
      }
    }
  }
}

// X2 / X3 faces, TMA-staged: the strip scheme below (4 consecutive i by 8
// zones along the direction per warp, 7 faces) with persistent warps that
// stage each chunk's stencil -- a box of 4 i x 12 zones along DIR x all dof
// -- in shared memory while computing the previous chunk.  The tensor map's
// box is (4, 12, 1, dof) for X2 and (4, 1, 12, dof) for X3; x starts at 4q
// (32-byte aligned) and the box along DIR at 7 x chunk (never negative).
constexpr int kStripRows = 12;
template <int COND, int VISC, int MINB, int DIR, int RS, bool PAIR>
__global__ void __launch_bounds__(128, MINB) k_face_flux_strip_tma(const __grid_constant__ CUtensorMap tmap, DevCfg c,
                                                                    const double* __restrict__ geoF,
                                                                    const double* __restrict__ geoC,
                                                                    double* __restrict__ flux, DevState* st) {
  constexpr int DOF = 8 + COND + VISC;
  constexpr int QI = 4, FPW = 7;
  constexpr int BOX = QI * kStripRows * DOF;  // doubles per buffer (a multiple of 128 bytes)
  constexpr int dir = DIR;
  extern __shared__ __align__(128) double smem_st[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double* bufs = smem_st + (size_t)w * 2 * BOX;
  double* park = smem_st + (size_t)nw * 2 * BOX;
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(park + 3 * DOF * blockDim.x) + 2 * w;
  const int NT = (DIR == 1) ? c.N2T : c.N3T;
  const unsigned nq = (unsigned)(c.N1T + QI - 1) / QI;
  const unsigned nch = (unsigned)(NT - 5 + FPW - 1) / FPW;  // faces 3 .. NT-3
  const unsigned nother = (unsigned)((DIR == 1) ? c.nfk : c.nfj);  // rows across the direction
  const int other0 = (DIR == 1) ? c.fk0 : c.fj0;
  const long long nitems = (long long)nq * nch * nother;
  const long long stride = (long long)gridDim.x * nw;
  long long item = (long long)blockIdx.x * nw + w;
  if (lane == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncwarp();
  auto decompose = [&](long long it, int& iq, int& ch, int& other) {
    const unsigned itu = (unsigned)it, r = itu / nq;
    iq = (int)(itu - r * nq);
    const unsigned o = r / nch;
    ch = (int)(r - o * nch);
    other = other0 + (int)o;
  };
  bool inflight[2] = {false, false};  // lane 0: copies issued, not yet seen land
  unsigned phase[2] = {0u, 0u};
  auto issue = [&](long long it, int buf) {
    if (c.dbgSkipCopies) return;
    int iq, ch, other;
    decompose(it, iq, ch, other);
    mbar_expect_tx(&bars[buf], BOX * (unsigned)sizeof(double));
    if (DIR == 1)
      tma_load_4d(bufs + buf * BOX, &tmap, &bars[buf], iq * QI, ch * FPW, other, 0);
    else
      tma_load_4d(bufs + buf * BOX, &tmap, &bars[buf], iq * QI, other, ch * FPW, 0);
    inflight[buf] = true;
  };
  if (lane == 0 && item < nitems) issue(item, 0);
  int buf = 0;
  const int ii = lane % QI, jj = lane / QI;
  for (; item < nitems; item += stride, buf ^= 1) {
    const long long next = item + stride;
    if (lane == 0 && next < nitems) issue(next, buf ^ 1);
    const bool arrived = mbar_wait_bounded(&bars[buf], phase[buf]);
    if (!__all_sync(0xffffffffu, arrived)) {
      if (lane == 0) copy_wait_gave_up(st, bars, inflight, phase);
      __syncwarp();
      return;
    }
    phase[buf] ^= 1u;
    inflight[buf] = false;
    int iq, ch, other;
    decompose(item, iq, ch, other);
    const int i = iq * QI + ii;
    const int x = 2 + ch * FPW + jj;  // zone along DIR; face x sits at its left
    const bool reconOK = i < c.N1T && x <= NT - 3;
    const double* rb = bufs + buf * BOX;
    double lo[DOF], ro[DOF];
#pragma unroll
    for (int v = 0; v < DOF; v++) {
      const double* a = rb + (v * kStripRows + jj) * QI + ii;  // rows jj .. jj+4 hold x-2 .. x+2
      recon_faces_rs<RS, kFastMath>(c.reconstruction, c.theta, a[0], a[QI], a[2 * QI], a[3 * QI], a[4 * QI], lo[v],
                                    ro[v]);
    }
    __syncwarp();  // the buffer is read; it may be refilled two items on
    double pl[DOF];
#pragma unroll
    for (int v = 0; v < DOF; v++) pl[v] = __shfl_up_sync(0xffffffffu, ro[v], QI);
    if (lane >= QI && reconOK) {
      const long long z = (DIR == 1) ? zidx(c, i, x, other) : zidx(c, i, other, x);
      ZoneGeo<double> G;
      // X3 faces use the centre geometry of each side (fvmfluxes.cpp:150-151),
      // one and the same: the metric does not depend on X3
      if (DIR == 2)
        load_geo(G, c, geoC, z, i, other, 0.5, 0.5);
      else
        load_geo(G, c, geoF, z, i, x, 0.5, 0.);
      if constexpr (PAIR) {
        riemann_face_pair<COND, VISC>(c, dir, pl, lo, G, flux, z);
      } else {
#pragma unroll
        for (int v = 0; v < DOF; v++) park[(2 * DOF + v) * blockDim.x + threadIdx.x] = lo[v];
        riemann_face<COND, VISC>(c, dir, pl, G, flux, z, park);
      }
    }
  }
}

// X2 / X3 faces: the X1 scheme turned sideways.  A warp holds QI
// consecutive i (lane % QI) by 32/QI consecutive zones along dir
// (lane / QI); every lane reconstructs its zone once and the right-face
// state moves QI lanes up by shuffle, giving (32/QI - 1) x QI faces per
// warp.  With QI = 4 each warp-wide load still covers whole 32-byte
// sectors (4 consecutive doubles along i), as in the X1 kernel.
template <int COND, int VISC, int QI, int MINB, bool PAIR, int DIR, int RS>
__global__ void __launch_bounds__(128, MINB) k_face_flux_strip(DevCfg c, const double* __restrict__ ps,
                                                         const double* __restrict__ geoF,
                                                         const double* __restrict__ geoC, double* __restrict__ flux) {
  constexpr int DOF = 8 + COND + VISC;
  constexpr int dir = DIR;  // a compile-time direction keeps the element in registers
  constexpr int JR = 32 / QI;       // zones along dir per warp
  constexpr int FPW = JR - 1;       // faces along dir per warp
  const int lane = threadIdx.x & 31;
  const long long wg = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int NT = (dir == 1) ? c.N2T : c.N3T;
  const int nq = (c.N1T + QI - 1) / QI;
  const int nch = (NT - 5 + FPW - 1) / FPW;  // faces 3 .. NT-3
  const long long nother = (dir == 1) ? c.nfk : c.nfj;  // rows across the direction
  if (wg >= (long long)nq * nch * nother) return;  // whole warps exit together
  const unsigned wgu = (unsigned)wg, r = wgu / (unsigned)nq;
  const int iq = (int)(wgu - r * (unsigned)nq);
  const unsigned oth = r / (unsigned)nch;
  const int ch = (int)(r - oth * (unsigned)nch);
  const int other = ((dir == 1) ? c.fk0 : c.fj0) + (int)oth;  // k for X2 faces, j for X3 faces
  const int i = iq * QI + (lane % QI);
  const int x = 2 + ch * FPW + lane / QI;  // zone along dir; face x sits at its left
  const bool reconOK = i < c.N1T && x <= NT - 3;
  const int ic = reconOK ? i : min(i, c.N1T - 1);
  const int xc = reconOK ? x : 2;
  const long long s = stride_of(c, dir);
  const long long z = dir == 1 ? zidx(c, ic, xc, other) : zidx(c, ic, other, xc);
  double lo[DOF], ro[DOF];
  recon_zone_rs<DOF, RS>(c, ps, z, s, lo, ro);
  double pl[DOF];
#pragma unroll
  for (int v = 0; v < DOF; v++) pl[v] = __shfl_up_sync(0xffffffffu, ro[v], QI);
  if (lane < QI || !reconOK) return;
  ZoneGeo<double> G;
  // X3 faces use the centre geometry of each side (fvmfluxes.cpp:150-151),
  // which is one and the same: the metric does not depend on X3
  if (dir == 2)
    load_geo(G, c, geoC, z, i, other, 0.5, 0.5);
  else
    load_geo(G, c, geoF, z, i, x, 0.5, 0.);
  if constexpr (PAIR) {
    riemann_face_pair<COND, VISC>(c, dir, pl, lo, G, flux, z);
  } else {
    extern __shared__ double park_strip[];
#pragma unroll
    for (int v = 0; v < DOF; v++) park_strip[(2 * DOF + v) * blockDim.x + threadIdx.x] = lo[v];
    riemann_face<COND, VISC>(c, dir, pl, G, flux, z, park_strip);
  }
}

// ---------------------------------------------------------------------------
// stage epilogue: EMF / CT (constrainedtransport.cpp:3-83), divergence
// (fvmfluxes.cpp), induction (timestep.cpp:80-89, 226-237), consOld
// (timestep.cpp:33-36), explicit sources (physics.cpp:360-586)
// ---------------------------------------------------------------------------
struct FluxView {
  const double* F[3];
  long long Z;
  int B1;
  GRIM_D double at(int d, int v, long long z) const { return __ldg(F[d] + (long long)v * Z + z); }
};

// EMF3 at edge (i-1/2, j-1/2) of zone z
GRIM_D double emf3(const FluxView& f, long long z, long long s1, long long s2) {
  return 0.25 * (f.at(0, f.B1 + 1, z) + f.at(0, f.B1 + 1, z - s2) - f.at(1, f.B1, z) - f.at(1, f.B1, z - s1));
}
GRIM_D double emf1(const FluxView& f, long long z, long long s2, long long s3) {
  return 0.25 * (f.at(1, f.B1 + 2, z) + f.at(1, f.B1 + 2, z - s3) - f.at(2, f.B1 + 1, z) - f.at(2, f.B1 + 1, z - s2));
}
GRIM_D double emf2(const FluxView& f, long long z, long long s1, long long s3) {
  return 0.25 * (f.at(2, f.B1, z) + f.at(2, f.B1, z - s1) - f.at(0, f.B1 + 2, z) - f.at(0, f.B1 + 2, z - s3));
}

// computeEMF (constrainedtransport.cpp:53-83) as arrays over the whole grid,
// neighbours by circular shift as in the reference: out = [emfX1 | emfX2 |
// emfX3] x Z (emfX1, emfX2 only in 3D, emfX3 from 2D on; zero otherwise)
static __global__ void k_emf(DevCfg c, const double* __restrict__ F1, const double* __restrict__ F2,
                             const double* __restrict__ F3, double* __restrict__ out) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  const long long Z = c.Z;
  const long long zi = zidx(c, (i - 1 + c.N1T) % c.N1T, j, k);
  const long long zj = zidx(c, i, (j - 1 + c.N2T) % c.N2T, k);
  const long long zk = zidx(c, i, j, (k - 1 + c.N3T) % c.N3T);
  const long long b1 = (long long)c.B1 * Z, b2 = b1 + Z, b3 = b2 + Z;
  double e1 = 0., e2 = 0., e3 = 0.;
  if (c.dim >= 2) e3 = 0.25 * (F1[b2 + z] + F1[b2 + zj] - F2[b1 + z] - F2[b1 + zi]);
  if (c.dim == 3) {
    e1 = 0.25 * (F2[b3 + z] + F2[b3 + zk] - F3[b2 + z] - F3[b2 + zj]);
    e2 = 0.25 * (F3[b1 + z] + F3[b1 + zi] - F1[b3 + z] - F1[b3 + zk]);
  }
  out[z] = e1;
  out[Z + z] = e2;
  out[2 * Z + z] = e3;
}

// PART 0 does all of the epilogue; the split launches PART 1 (centre: the
// stage element, consOld on the half stage, explicit sources) and then
// PART 2 (fluxes: CT, divergence, induction, Newton guess), each with the
// registers of its own half (the flux half is a memory stream).
// blocks per SM each part is compiled for: the flux half is a memory
// stream that wants warps in flight more than registers (measured on the
// 3D torus: 64 registers with a few spills beat 85 and 98 without)
constexpr int kEpiMinBlocks[3] = {4, 5, 8};
template <int COND, int VISC, int PART>
__global__ void __launch_bounds__(128, kEpiMinBlocks[PART]) k_stage_epilogue(DevCfg c, int stage, StageBufs b) {
  constexpr int NF = 5 + COND + VISC;
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  const long long Z = c.Z;
  const long long z = interior_to_z(c, n);
  int i, j, k;
  zijk(c, z, i, j, k);
  const long long s1 = 1, s2 = (long long)c.N1T, s3 = (long long)c.N1T * c.N2T;
  FluxView f;
  f.F[0] = b.flux[0]; f.F[1] = b.flux[1]; f.F[2] = b.flux[2]; f.Z = Z; f.B1 = c.B1;
  const double dt = b.st->dt;

  constexpr int DOF = NF + 3;
  double div[DOF];
  if constexpr (PART != 1) {
  // ---- fluxes on the zone's two faces of each direction: Riemann fluxes
  // for the fluid rows, flux-CT values for the field rows
  // (constrainedtransport.cpp:3-51); the divergence (fvmfluxes.cpp) adds
  // one direction at a time, so only that direction's faces are live:
  // zero-padded convolution Fr*(1/dX) + Fl*(-1/dX) in 1D/2D, shifted
  // difference (Fr - Fl)/dX in 3D, summed in direction order
  const long long sd[3] = {s1, s2, s3};
  // corner EMFs (constrainedtransport.cpp:53-83), each formed here from the
  // face fluxes around its edge as computeEMF forms it: a corner's fluxes
  // are L1/L2 hits shared with the neighbouring zones' threads, cheaper
  // than a separate pass that writes the corners out and reads them back
  double e[12];  // EMF3 (i|i+1, j|j+1), EMF2 (i|i+1, k|k+1), EMF1 (j|j+1, k|k+1)
  if (c.dim >= 2) {
    e[0] = emf3(f, z, s1, s2); e[1] = emf3(f, z + s1, s1, s2);
    e[2] = emf3(f, z + s2, s1, s2); e[3] = emf3(f, z + s1 + s2, s1, s2);
  }
  if (c.dim == 3) {
    e[4] = emf2(f, z, s1, s3); e[5] = emf2(f, z + s1, s1, s3);
    e[6] = emf2(f, z + s3, s1, s3); e[7] = emf2(f, z + s1 + s3, s1, s3);
    e[8] = emf1(f, z, s2, s3); e[9] = emf1(f, z + s2, s2, s3);
    e[10] = emf1(f, z + s3, s2, s3); e[11] = emf1(f, z + s2 + s3, s2, s3);
  }
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (d >= c.dim) break;
    double Fl[DOF], Fr[DOF];
#pragma unroll
    for (int v = 0; v < NF; v++) { Fl[v] = f.at(d, v, z); Fr[v] = f.at(d, v, z + sd[d]); }
#pragma unroll
    for (int v = NF; v < DOF; v++) { Fl[v] = 0.; Fr[v] = 0.; }
    if (c.dim == 1) {
#pragma unroll
      for (int b3 = 0; b3 < 3; b3++) { Fl[NF + b3] = f.at(0, c.B1 + b3, z); Fr[NF + b3] = f.at(0, c.B1 + b3, z + s1); }
    } else if (c.dim == 2) {
      // F1: B1 -> 0, B2 -> 0.5 (emf3 + emf3[j+1]); F2: B1 -> -0.5 (emf3 + emf3[i+1]), B2 -> 0
      if (d == 0) {
        Fl[NF + 1] = 0.5 * (e[0] + e[2]);
        Fr[NF + 1] = 0.5 * (e[1] + e[3]);
      } else {
        Fl[NF + 0] = -0.5 * (e[0] + e[1]);
        Fr[NF + 0] = -0.5 * (e[2] + e[3]);
      }
      Fl[NF + 2] = f.at(d, c.B1 + 2, z);
      Fr[NF + 2] = f.at(d, c.B1 + 2, z + sd[d]);
    } else if (d == 0) {
      Fl[NF + 1] = 0.5 * (e[0] + e[2]);  Fr[NF + 1] = 0.5 * (e[1] + e[3]);
      Fl[NF + 2] = -0.5 * (e[4] + e[6]); Fr[NF + 2] = -0.5 * (e[5] + e[7]);
    } else if (d == 1) {
      Fl[NF + 0] = -0.5 * (e[0] + e[1]); Fr[NF + 0] = -0.5 * (e[2] + e[3]);
      Fl[NF + 2] = 0.5 * (e[8] + e[10]); Fr[NF + 2] = 0.5 * (e[9] + e[11]);
    } else {
      Fl[NF + 0] = 0.5 * (e[4] + e[5]);  Fr[NF + 0] = 0.5 * (e[6] + e[7]);
      Fl[NF + 1] = -0.5 * (e[8] + e[9]); Fr[NF + 1] = -0.5 * (e[10] + e[11]);
    }
    if (c.problem == GRIM_PROBLEM_TORUS) {
      // applyProblemSpecificFluxFilter (torus/problem.cpp:1243-1285)
      if (d == 0) {
        if (i == c.g1) Fl[RHO] = fmin(Fl[RHO], 0.);
        if (i == c.N1 + c.g1 - 1) Fr[RHO] = fmax(Fr[RHO], 0.);
      } else if (d == 1) {
        if (j == c.g2)
#pragma unroll
          for (int v = 0; v < DOF; v++) Fl[v] = 0.;
        if (j == c.N2 + c.g2 - 1)
#pragma unroll
          for (int v = 0; v < DOF; v++) Fr[v] = 0.;
      }
    }
    if (c.dim <= 2) {
      const double id = 1. / c.dX[d];
#pragma unroll
      for (int v = 0; v < DOF; v++) {
        const double t = Fr[v] * id + Fl[v] * (-id);
        div[v] = (d == 0) ? t : div[v] + t;
      }
    } else {
      const double id = 1. / c.dX[d];
#pragma unroll
      for (int v = 0; v < DOF; v++) {
        const double t = kFastMath ? (Fr[v] - Fl[v]) * id : (Fr[v] - Fl[v]) / c.dX[d];
        div[v] = (d == 0) ? t : div[v] + t;
      }
    }
  }

  }  // PART != 1
  ZoneGeo<double> G;
  load_geo(G, c, b.geoC, z, i, j, 0.5, 0.5);
  if constexpr (PART != 2) {
  // ---- stage element at the centre (elemOld / elemHalfStep)
  const double* ps = b.ps;
  ElemT<double, double> e;
  elem_set<COND, VISC>(e, ps[z], ps[Z + z], ps[2 * Z + z], ps[3 * Z + z], ps[4 * Z + z],
                       ps[(long long)c.B1 * Z + z], ps[(long long)(c.B1 + 1) * Z + z],
                       ps[(long long)(c.B1 + 2) * Z + z], COND ? ps[(long long)c.Q * Z + z] : 0.,
                       VISC ? ps[(long long)c.DP * Z + z] : 0., G, c);
  if (stage == GRIM_HALF_STEP) {
    double U[NF], UB[3];
    fluxes_fluid<COND, VISC>(e, 0, G.g, U, 5, 5 + COND);
    fluxes_B(e, 0, G.g, UB);
#pragma unroll
    for (int v = 0; v < NF; v++) b.consOld[(long long)v * Z + z] = U[v];
#pragma unroll
    for (int v = 0; v < 3; v++) b.consOld[(long long)(NF + v) * Z + z] = UB[v];
  }
  // ---- explicit sources
  double S[NF];
#pragma unroll
  for (int v = 0; v < NF; v++) S[v] = 0.;
  const bool needS = (c.metric != GRIM_MINKOWSKI) || COND || VISC;
  if (c.metric != GRIM_MINKOWSKI) {
    double T[4][4];
#pragma unroll
    for (int ka = 0; ka < 4; ka++)
#pragma unroll
      for (int la = 0; la < 4; la++) T[ka][la] = tmunu<COND, VISC>(e, ka, la);
    const double* gam = b.gamma + gidx(c, i, j);
    if constexpr (kFastMath) {
      // Gamma^la_(ka nu) is symmetric in its lower pair: 40 loads, each
      // used for (ka, nu) and (nu, ka)
      double acc[4] = {S[UU], S[UU + 1], S[UU + 2], S[UU + 3]};
#pragma unroll
      for (int la = 0; la < 4; la++)
#pragma unroll
        for (int ka = 0; ka < 4; ka++)
#pragma unroll
          for (int nu = ka; nu < 4; nu++) {
            const double gv = G.g * __ldg(gam + (long long)(la * 16 + ka * 4 + nu) * c.GZ);
            acc[nu] -= T[ka][la] * gv;
            if (nu != ka) acc[ka] -= T[nu][la] * gv;
          }
#pragma unroll
      for (int nu = 0; nu < 4; nu++) S[UU + nu] = acc[nu];
    } else {
#pragma unroll
      for (int nu = 0; nu < 4; nu++) {
        double s = S[UU + nu];
#pragma unroll
        for (int ka = 0; ka < 4; ka++)
#pragma unroll
          for (int la = 0; la < 4; la++)
            s -= G.g * T[ka][la] * __ldg(gam + (long long)(la * 16 + ka * 4 + nu) * c.GZ);
        S[UU + nu] = s;
      }
    }
  }
  if (COND || VISC) {
    // computeEMHDGradients (physics.cpp:502-586) from the pre-pass u_mu, T
    double gu[4][4], gT[4];
    const double* uT = b.uT;
    auto st = [&](int m, int dir, double dx) -> double {
      const long long sd = stride_of(c, dir);
      const double* a = uT + (long long)m * Z + z;
      return recon_slope(c.reconstruction, c.theta, a[-2 * sd], a[-sd], a[0], a[sd], a[2 * sd], dx);
    };
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
      gu[0][mu] = 0.;
      gu[1][mu] = st(mu, 0, c.dX[0]);
      gu[2][mu] = (c.dim > 1) ? st(mu, 1, c.dX[1]) : 0.;
      gu[3][mu] = (c.dim > 2) ? st(mu, 2, c.dX[2]) : 0.;
      if (c.metric != GRIM_MINKOWSKI) {
#pragma unroll
        for (int nu = 0; nu < 4; nu++)
#pragma unroll
          for (int la = 0; la < 4; la++)
            gu[nu][mu] -= __ldg(b.gamma + (long long)(la * 16 + nu * 4 + mu) * c.GZ + gidx(c, i, j)) * e.uCov[la];
      }
    }
    if (COND) {
      gT[0] = 0.;
      gT[1] = st(4, 0, c.dX[0]);
      gT[2] = (c.dim > 1) ? st(4, 1, c.dX[1]) : 0.;
      gT[3] = (c.dim > 2) ? st(4, 2, c.dX[2]) : 0.;
    }
    double dv = 0.;
#pragma unroll
    for (int mu = 0; mu < 4; mu++)
#pragma unroll
      for (int nu = 0; nu < 4; nu++) dv += G.gcon[mu][nu] * gu[mu][nu];
    if (VISC) {
      double d0 = -dv * e.rho * e.nu;
#pragma unroll
      for (int mu = 0; mu < 4; mu++)
#pragma unroll
        for (int nu = 0; nu < 4; nu++) d0 += 3. * e.rho * e.nu * e.bCon[mu] * e.bCon[nu] / e.bSqr * gu[mu][nu];
      double d0t = (c.hoVisc == 1) ? d0 * sqrt(e.tau / e.rho / e.nu / e.temperature) : d0;
      double s = -G.g * (d0t) / e.tau;
      if (c.hoVisc == 1) s -= 0.5 * G.g * dv * e.deltaPTilde;
      S[c.DP] = s;
    }
    if (COND) {
      double qq = 0.;
#pragma unroll
      for (int mu = 0; mu < 4; mu++) {
        qq -= e.rho * e.chi * e.bCon[mu] / e.bNorm * gT[mu];
#pragma unroll
        for (int nu = 0; nu < 4; nu++) qq -= e.rho * e.chi * e.temperature * e.bCon[nu] / e.bNorm * e.uCon[mu] * gu[mu][nu];
      }
      double qt = (c.hoCond == 1) ? qq * sqrt(e.tau / e.rho / e.chi) / e.temperature : qq;
      double s = -G.g * (qt) / e.tau;
      if (c.hoCond == 1) s -= 0.5 * G.g * dv * e.qTilde;
      S[c.Q] = s;
    }
  }
  // ---- outputs: stage constants for the Newton kernels
  if (needS)
#pragma unroll
    for (int v = 0; v < NF; v++) b.Sexp[(long long)v * Z + z] = S[v];
  }  // PART != 2
  if constexpr (PART != 1) {
#pragma unroll
  for (int v = 0; v < NF; v++) b.divF[(long long)v * Z + z] = div[v];
  if (b.divFB)
#pragma unroll
    for (int v = NF; v < DOF; v++) b.divF[(long long)v * Z + z] = div[v];
  // ---- induction and the Newton guess
  const double fac = (stage == GRIM_HALF_STEP) ? 0.5 * dt : dt;
#pragma unroll
  for (int b3 = 0; b3 < 3; b3++) {
    double cons = b.consOld[(long long)(NF + b3) * Z + z] - fac * div[NF + b3];
    b.prim[(long long)(c.B1 + b3) * Z + z] = cons / G.g;
  }
  if (stage == GRIM_HALF_STEP && !b.guessOld)
#pragma unroll
    for (int v = 0; v < NF; v++) b.prim[(long long)v * Z + z] = b.pold[(long long)v * Z + z];
  }  // PART != 1
}

// ---------------------------------------------------------------------------
// computeDt (timestep.cpp:336-400): max over all zones (ghosts included) of
// sum_d max(c_max/dX_d, |c_min/dX_d|) of the element state `mode` selects:
//   0: prims as stored, 1: grid::communicate semantics (periodic ghosts
//   wrapped, ghosts on a non-periodic edge read as zero), 2: all-zero prims
//   (the grids the reference's elements are first set on)
// ---------------------------------------------------------------------------
GRIM_D void atomic_max_pos(double* addr, double v) {
  if (!(v >= 0.)) v = 0.;
  atomicMax((unsigned long long*)addr, (unsigned long long)__double_as_longlong(v));
}

// one zone's sum over directions of max(c_max/dX_d, |c_min/dX_d|)
template <int COND, int VISC>
GRIM_D double elem_inv_dt(const DevCfg& c, const ElemT<double, double>& e, const ZoneGeo<double>& G) {
  double acc = 0.;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (d < c.dim) {
      double mn, mx;
      char_speeds<COND, VISC>(e, G, d, c, mn, mx);
      double m2;
      if constexpr (kFastMath) {
        // one product for two divisions: scaling by 1/dX > 0 commutes with
        // the max (rounding is monotonic)
        m2 = fmax(mx, fabs(mn)) * c.invdX[d];
      } else {
        double a = mn / c.dX[d], bb = mx / c.dX[d];
        m2 = fmax(bb, fabs(a));
      }
      acc = (d == 0) ? m2 : acc + m2;
    }
  }
  return acc;
}
template <int COND, int VISC>
GRIM_D double zone_inv_dt(const DevCfg& c, const double* pv, const ZoneGeo<double>& G) {
  ElemT<double, double> e;
  elem_of<COND, VISC>(e, c, pv, G);
  return elem_inv_dt<COND, VISC>(c, e, G);
}

// block reduction of the threads' values, then one atomic max per block
// (every thread of the block calls it)
GRIM_D void block_max_to(double best, double* out) {
  __shared__ double sm[32];
  for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sm[w] = best;
  __syncthreads();
  if (w == 0) {
    best = (lane < (int)(blockDim.x >> 5)) ? sm[lane] : 0.;
    for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) atomic_max_pos(out, best);
  }
}

template <int COND, int VISC>
__global__ void k_dt_speeds(DevCfg c, const double* __restrict__ p, const double* __restrict__ geoC,
                                     int mode, DevState* st) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double best = 0.;
  if (z < c.Z) {
    int i, j, k;
    zijk(c, z, i, j, k);
    long long src = z;
    bool zero = (mode == 2);
    if (mode == 1) src = comm_source(c, i, j, k, zero);
    const long long Z = c.Z;
    constexpr int NF = 5 + COND + VISC, DOF = NF + 3;
    double pv[DOF];
#pragma unroll
    for (int v = 0; v < DOF; v++) pv[v] = zero ? 0. : p[(long long)v * Z + src];
    ZoneGeo<double> G;
    load_geo(G, c, geoC, z, i, j, 0.5, 0.5);
    if (!in_exchange_ghost(c, i, j, k)) best = zone_inv_dt<COND, VISC>(c, pv, G);
  }
  block_max_to(best, &st->maxInvDt);
}

// The end of a stage in one pass over the grid: the Newton result src is
// copied into the stage's array dst with grid::communicate's ghost values
// (timestep.cpp: primHalfStep / primOld = prim, then communicate;
// grid.cpp:306-360), then per zone
//   FLOOR: the torus floors (halfStepDiagnostics / fullStepDiagnostics,
//          torus/problem.cpp:714-746; with POST the NaN reset first),
//   POST:  after the full step, the zone's term of the next computeDt from
//          the stored result (all zones, as k_dt_speeds mode 0; when
//          dtOn) and the non-finite count over the interior.
// Every step of the reference's sequence acts on one zone at a time, so the
// fused pass gives the same values (the NaN flag is counted beforehand over
// the interior of src, which the copy leaves unchanged).
template <int COND, int VISC, bool FLOOR, bool POST>
__global__ void __launch_bounds__(128) k_stage_finish(DevCfg c, TorusCfg t, const double* __restrict__ src,
                                                      double* __restrict__ dst, const double* __restrict__ geoC,
                                                      const unsigned long long* nanFlag, int dtOn, DevState* st) {
  constexpr int DOF = 8 + COND + VISC;
  const long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long Z = c.Z;
  double best = 0.;
  int bad = 0;
  if (z < Z) {
    int i, j, k;
    zijk(c, z, i, j, k);
    bool zero;
    const long long s = comm_source(c, i, j, k, zero);
    double q[DOF];
#pragma unroll
    for (int v = 0; v < DOF; v++) q[v] = zero ? 0. : src[(long long)v * Z + s];
    ZoneGeo<double> G;
    load_geo(G, c, geoC, z, i, j, 0.5, 0.5);
    // the floors' last element, when it is that of the final state, serves
    // the dt speeds below (the same function of the same values)
    ElemT<double, double> ef;
    bool haveElem = false;
    if constexpr (FLOOR) {
      const long long gz = gidx(c, i, j);
      haveElem = torus_floor_zone<COND, VISC>(c, t, q, G, __ldg(geoC + 37LL * c.GZ + gz),
                                              __ldg(geoC + 38LL * c.GZ + gz), POST && *nanFlag != 0,
                                              POST ? &ef : nullptr);
    }
#pragma unroll
    for (int v = 0; v < DOF; v++) dst[(long long)v * Z + z] = q[v];
    if constexpr (POST) {
      if (dtOn && !in_exchange_ghost(c, i, j, k))
        best = haveElem ? elem_inv_dt<COND, VISC>(c, ef, G) : zone_inv_dt<COND, VISC>(c, q, G);
      const bool inside = i >= c.g1 && i < c.N1 + c.g1 && j >= c.g2 && j < c.N2 + c.g2 && k >= c.g3 &&
                          k < c.N3 + c.g3;
      if (inside)
#pragma unroll
        for (int v = 0; v < DOF; v++)
          if (!isfinite(q[v])) bad = 1;
    }
  }
  if constexpr (POST) {
    block_max_to(best, &st->maxInvDt);
    bad = __syncthreads_count(bad);
    if (threadIdx.x == 0 && bad) atomicAdd(&st->nonFinite, (unsigned long long)bad);
  }
}

// ---------------------------------------------------------------------------
// Torus observers (ObserversTorus.hpp:6-253, called by fullStepDiagnostics,
// torus/problem.cpp:754-778): integrals and extrema over the interior of
// primOld with the element of its final state at the zone centres, each
// integrand in the reference's operation order.  Two launches: fixed-size
// per-block partials (grid-stride over the interior, shuffle trees), then
// one thread combines them in block order, so the sums are reproducible.
// ---------------------------------------------------------------------------
// ObserveData (problem.cpp:754): this step's time crossed a multiple of
// every (every <= 0: always)
GRIM_D bool obs_due(const DevState* st, double every) {
  if (every <= 0.) return true;
  return floor(st->time / every) != floor((st->time - st->dt) / every);
}
GRIM_D double obs_join(int v, double a, double b) {
  return v == OBS_RHOMAX ? fmax(a, b) : (v == OBS_BETAMIN ? fmin(a, b) : a + b);
}

template <int COND, int VISC>
__global__ void __launch_bounds__(128, 5) k_torus_obs_partial(DevCfg c, const double* __restrict__ p,
                                                           const double* __restrict__ geoC, double volElem,
                                                           double every, const DevState* st,
                                                           double* __restrict__ partials) {
  if (!obs_due(st, every)) return;
  constexpr int DOF = 8 + COND + VISC;
  double acc[OBS_N];
#pragma unroll
  for (int v = 0; v < OBS_N; v++) acc[v] = 0.;
  acc[OBS_RHOMAX] = -INFINITY;
  acc[OBS_BETAMIN] = INFINITY;
  const long long Z = c.Z;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < c.Zint;
       n += (long long)gridDim.x * blockDim.x) {
    const long long z = interior_to_z(c, n);
    int i, j, k;
    zijk(c, z, i, j, k);
    double q[DOF];
#pragma unroll
    for (int v = 0; v < DOF; v++) q[v] = p[(long long)v * Z + z];
    ZoneGeo<double> G;
    load_geo(G, c, geoC, z, i, j, 0.5, 0.5);
    ElemT<double, double> e;
    elem_of<COND, VISC>(e, c, q, G);
    const double rho = q[RHO], u = q[UU];
    acc[OBS_MASS] += rho * volElem * G.g * e.gam / G.alpha;
    acc[OBS_EMAG] += volElem * e.bSqr * G.g * e.gam / G.alpha;
    acc[OBS_ETH] += volElem * u * G.g * e.gam / G.alpha;
    acc[OBS_RHOMAX] = fmax(acc[OBS_RHOMAX], rho);
    acc[OBS_BETAMIN] = fmin(acc[OBS_BETAMIN], 2. * (e.pressure + 1.e-13) / (e.bSqr + 1.e-18));
    // boundary fluxes at the first and last interior X1 columns
    const double mi = rho * volElem * G.g * e.uCon[1];
    if (i == 3) acc[OBS_MDOT_IN] += mi;
    if (i == c.N1 + 2) {
      acc[OBS_MDOT_OUT] += mi;
      const double bern = (1. + u / rho * c.Gam) * e.uCov[0];
      const double unb = mi * ((bern < -1.) ? 1. : 0.);
      acc[OBS_UNBOUND_OUT] += unb;
      acc[OBS_REL_UNBOUND_OUT] += unb * ((e.gam > 2.) ? 1. : 0.);
    }
  }
  __shared__ double sm[8][OBS_N];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < OBS_N; v++) {
    double a = acc[v];
    for (int o = 16; o > 0; o >>= 1) a = obs_join(v, a, __shfl_xor_sync(0xffffffffu, a, o));
    if (lane == 0) sm[w][v] = a;
  }
  __syncthreads();
  if (threadIdx.x < OBS_N) {
    const int v = threadIdx.x;
    double a = sm[0][v];
    for (int ww = 1; ww < (int)(blockDim.x >> 5); ww++) a = obs_join(v, a, sm[ww][v]);
    partials[(long long)blockIdx.x * OBS_N + v] = a;
  }
}

// combines the partials in block order; writes out (OBS_N values) and, with
// a history, appends the record {time, values} at ring slot obsCount % cap
static __global__ void k_torus_obs_final(const double* __restrict__ partials, int nblocks, double every,
                                         DevState* st, double* out, double* hist, int cap) {
  // one thread per observable folds the partials in block order; launched
  // as one warp
  const int v = threadIdx.x;
  if (blockIdx.x != 0 || !obs_due(st, every)) return;
  double* rec = (hist && cap > 0) ? hist + (st->obsCount % (unsigned long long)cap) * (OBS_N + 1) : nullptr;
  if (v < OBS_N) {
    // 16 loads in flight per chunk, joined in block order
    double r = partials[v];
    for (int b0 = 1; b0 < nblocks; b0 += 16) {
      double t[16];
#pragma unroll
      for (int q = 0; q < 16; q++) t[q] = (b0 + q < nblocks) ? partials[(long long)(b0 + q) * OBS_N + v] : 0.;
#pragma unroll
      for (int q = 0; q < 16; q++)
        if (b0 + q < nblocks) r = obs_join(v, r, t[q]);
    }
    if (out) out[v] = r;
    if (rec) rec[1 + v] = r;
  }
  __syncwarp();
  if (v == 0 && rec) {
    rec[0] = st->time;
    st->obsCount += 1;
  }
}

// dt = Courant / maxInvDt, capped at maxDtIncrement * dt (timestep.cpp:393-399)
static __global__ void k_dt_update(DevState* st, double courant, double maxInc) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double newDt = courant / st->maxInvDt;
    if (newDt > maxInc * st->dt) newDt = maxInc * st->dt;
    st->dtOld = st->dt;
    st->dt = newDt;
  }
}

static __global__ void k_advance_time(DevState* st) {
  if (threadIdx.x == 0 && blockIdx.x == 0) st->time += st->dt;
}

// ---------------------------------------------------------------------------
// Newton
// ---------------------------------------------------------------------------
template <int COND, int VISC>
GRIM_D void load_stage_const(StageConst<5 + COND + VISC>& K, const DevCfg& c, int stage, const StageBufs& b,
                             long long z, const ZoneGeo<double>& G) {
  constexpr int NF = 5 + COND + VISC;
  const long long Z = c.Z;
  const bool needS = (c.metric != GRIM_MINKOWSKI) || COND || VISC;
  const double dt = b.st->dt;
  K.dtp = (stage == GRIM_HALF_STEP) ? dt / 2. : dt;
  K.idtp = 1. / K.dtp;
#pragma unroll
  for (int v = 0; v < NF; v++) {
    K.Uold[v] = b.consOld[(long long)v * Z + z];
    K.divF[v] = b.divF[(long long)v * Z + z];
    K.Sexp[v] = needS ? b.Sexp[(long long)v * Z + z] : 0.;
  }
#pragma unroll
  for (int v = 0; v < NF; v++) K.Kc[v] = K.divF[v] + K.Sexp[v] - K.Uold[v] * K.idtp;
#pragma unroll
  for (int v = 0; v < 3; v++) K.B[v] = b.prim[(long long)(c.B1 + v) * Z + z];
  // the rounding floor: the residual's largest term is U / dt', which at
  // the solution is -Kc (R = U / dt' + Kc = 0), over the conserved rows
  K.tolFloor2 = 0.;
  if (c.tolUlps > 0.) {
    double s = 0.;
#pragma unroll
    for (int v = 0; v < 5; v++) s = fmax(s, fabs(K.Kc[v]));
    const double f = c.tolUlps * 2.220446049250313e-16 * s;
    K.tolFloor2 = f * f;
  }
  if (COND || VISC) {
    const double* po = b.pold;
    ElemT<double, double> eo;
    elem_set<COND, VISC>(eo, po[z], po[Z + z], po[2 * Z + z], po[3 * Z + z], po[4 * Z + z],
                         po[(long long)c.B1 * Z + z], po[(long long)(c.B1 + 1) * Z + z],
                         po[(long long)(c.B1 + 2) * Z + z], COND ? po[(long long)c.Q * Z + z] : 0.,
                         VISC ? po[(long long)c.DP * Z + z] : 0., G, c);
#pragma unroll
    for (int m = 0; m < 4; m++) K.uCovOld[m] = eo.uCov[m];
    K.TOld = eo.temperature;
    ElemT<double, double> er;
    if (stage == GRIM_HALF_STEP) {
      er = eo;
    } else {
      const double* ph = b.ps;
      elem_set<COND, VISC>(er, ph[z], ph[Z + z], ph[2 * Z + z], ph[3 * Z + z], ph[4 * Z + z],
                           ph[(long long)c.B1 * Z + z], ph[(long long)(c.B1 + 1) * Z + z],
                           ph[(long long)(c.B1 + 2) * Z + z], COND ? ph[(long long)c.Q * Z + z] : 0.,
                           VISC ? ph[(long long)c.DP * Z + z] : 0., G, c);
    }
    K.refRho = er.rho; K.refNu = VISC ? er.nu : 0.; K.refChi = COND ? er.chi : 0.;
    K.refTau = er.tau; K.refT = er.temperature;
#pragma unroll
    for (int m = 0; m < 4; m++) K.refBCon[m] = er.bCon[m];
    K.refBSqr = er.bSqr; K.refBNorm = er.bNorm; K.refUCon0 = er.uCon[0];
    K.refQTilde = COND ? er.qTilde : 0.;
    K.refDPTilde = VISC ? er.deltaPTilde : 0.;
    // elemOld->computeImplicitSources(sourcesImplicitOld, ref.tau)
    K.sImpOldQ = COND ? G.g * (eo.qTilde) / er.tau : 0.;
    K.sImpOldDP = VISC ? G.g * (eo.deltaPTilde) / er.tau : 0.;
    // residual normalisation (residual.cpp:291-323, :366-399)
    if (COND) K.normQ = (c.hoCond) ? er.temperature * sqrt(er.rho * er.chi * er.tau) : er.tau;
    if (VISC) K.normDP = (c.hoVisc) ? sqrt(er.rho * er.nu * er.temperature * er.tau) : er.tau;
  }
}

// pivoted Gaussian elimination (the oracle's; af::solve at solve.cpp:220)
template <class T, int N>
GRIM_D void gauss_solve(T A[N][N], T b[N], T x[N]) {
#pragma unroll
  for (int kk = 0; kk < N; kk++) {
    int p = kk;
    T best = fabs(A[kk][kk]);
#pragma unroll
    for (int r = kk + 1; r < N; r++) {
      T v = fabs(A[r][kk]);
      if (v > best) { best = v; p = r; }
    }
    // row exchange as selects over compile-time indices, so the matrix
    // stays in registers (a conditional swap sends it to local memory);
    // columns left of kk are not read again
#pragma unroll
    for (int r = kk + 1; r < N; r++) {
      const bool sw = (r == p);
#pragma unroll
      for (int cc = kk; cc < N; cc++) {
        const T a0 = A[kk][cc], a1 = A[r][cc];
        A[kk][cc] = sw ? a1 : a0;
        A[r][cc] = sw ? a0 : a1;
      }
      const T b0 = b[kk], b1 = b[r];
      b[kk] = sw ? b1 : b0;
      b[r] = sw ? b0 : b1;
    }
    const T akk = A[kk][kk];
    if constexpr (kFastMath) {
      // one reciprocal per pivot, kept for the back substitution
      const T ia = T(1) / akk;
      A[kk][kk] = ia;
#pragma unroll
      for (int r = kk + 1; r < N; r++) {
        T l = A[r][kk] * ia;
#pragma unroll
        for (int cc = kk + 1; cc < N; cc++) A[r][cc] -= l * A[kk][cc];
        b[r] -= l * b[kk];
      }
    } else {
#pragma unroll
      for (int r = kk + 1; r < N; r++) {
        T l = A[r][kk] / akk;
#pragma unroll
        for (int cc = kk + 1; cc < N; cc++) A[r][cc] -= l * A[kk][cc];
        b[r] -= l * b[kk];
      }
    }
  }
#pragma unroll
  for (int r = N - 1; r >= 0; r--) {
    T s = b[r];
#pragma unroll
    for (int cc = r + 1; cc < N; cc++) s -= A[r][cc] * x[cc];
    if constexpr (kFastMath)
      x[r] = s * A[r][r];  // the stored reciprocal
    else
      x[r] = s / A[r][r];
  }
}

// histogram of per-zone iteration counts, one atomic per distinct value in
// a warp
GRIM_D void hist_add(unsigned long long* hist, int bin, bool active) {
  const unsigned act = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const unsigned peers = __match_any_sync(act, bin);
  if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[bin], (unsigned long long)__popc(peers));
}

template <int NF>
GRIM_D double l2sum(const double* R) {
  double s = 0.;
#pragma unroll
  for (int v = 0; v < NF; v++) s += R[v] * R[v];
  return s;
}

// Parity Newton, launch 0: floor, residual, per-zone l2 and the count of
// unconverged zones for iteration 0 (solve.cpp:17-41)
template <int COND, int VISC>
__global__ void __launch_bounds__(128) k_newton_fd_init(DevCfg c, int stage, StageBufs b) {
  constexpr int NF = 5 + COND + VISC;
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int unconv = 0;
  if (n < c.Zint) {
    const long long Z = c.Z;
    const long long z = interior_to_z(c, n);
    int i, j, k;
    zijk(c, z, i, j, k);
    ZoneGeo<double> G;
    load_geo(G, c, b.geoC, z, i, j, 0.5, 0.5);
    StageConst<NF> K;
    load_stage_const<COND, VISC>(K, c, stage, b, z, G);
    double P[NF], R[NF];
#pragma unroll
    for (int v = 0; v < NF; v++) P[v] = b.prim[(long long)v * Z + z];
    P[0] = fmax(P[0], c.rhoFloor);
    P[1] = fmax(P[1], c.uFloor);
    b.prim[z] = P[0];
    b.prim[Z + z] = P[1];
    zone_residual<COND, VISC, double, double>(P, K, G, c, R);
#pragma unroll
    for (int v = 0; v < NF; v++) b.R[(long long)v * Z + z] = R[v];
    double l2 = l2sum<NF>(R);
    b.l2[z] = l2;
    b.l2[Z + z] = l2;
    double tol = newton_tol(c, l2, K);
    unconv = (l2 > tol) ? 1 : 0;
  }
  unconv = __syncthreads_count(unconv);
  if (threadIdx.x == 0 && unconv) atomicAdd(&b.st->count[stage][0], (unsigned long long)unconv);
}

// Parity Newton, iteration `it` (solve.cpp:80-199): FD Jacobian, pivoted
// solve, quadratic backtracking, update; then the floor + residual + count
// of iteration it+1.  Returns at once when iteration `it` found every zone
// converged (the reference's global break).
template <int COND, int VISC>
__global__ void __launch_bounds__(128) k_newton_fd_iter(DevCfg c, int stage, int it, StageBufs b) {
  constexpr int NF = 5 + COND + VISC;
  if (b.st->count[stage][it] == 0ULL) return;
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int unconv = 0;
  if (n < c.Zint) {
    const long long Z = c.Z;
    const long long z = interior_to_z(c, n);
    int i, j, k;
    zijk(c, z, i, j, k);
    ZoneGeo<double> G;
    load_geo(G, c, b.geoC, z, i, j, 0.5, 0.5);
    StageConst<NF> K;
    load_stage_const<COND, VISC>(K, c, stage, b, z, G);
    double P[NF], R[NF];
#pragma unroll
    for (int v = 0; v < NF; v++) {
      P[v] = b.prim[(long long)v * Z + z];
      R[v] = b.R[(long long)v * Z + z];
    }
    const double l2 = b.l2[z];
    const double l2first = b.l2[Z + z];
    // FD Jacobian, J[col][row] = dR_col / dP_row
    double J[NF][NF];
    const double eps = c.jacEps;
#pragma unroll
    for (int row = 0; row < NF; row++) {
      double Pe[NF];
#pragma unroll
      for (int v = 0; v < NF; v++) Pe[v] = P[v];
      double small = (fabs(P[row]) < .5 * eps) ? 1. : 0.;
      Pe[row] = P[row] + eps * P[row] * (1. - small) + small * eps;
      double Rp[NF];
      zone_residual<COND, VISC, double, double>(Pe, K, G, c, Rp);
      const double dP = Pe[row] - P[row];
#pragma unroll
      for (int col = 0; col < NF; col++) J[col][row] = (Rp[col] - R[col]) / dP;
    }
    double bvec[NF], dPv[NF];
#pragma unroll
    for (int v = 0; v < NF; v++) bvec[v] = -R[v];
    gauss_solve<double, NF>(J, bvec, dPv);
    // line search
    const double f0 = 0.5 * l2;
    const double fPrime0 = -2. * f0;
    double lam = 1.;
    bool haveRt = false;
    double Rt[NF];
    for (int ls = 0; ls < c.maxLS; ls++) {
      double Pt[NF];
#pragma unroll
      for (int v = 0; v < NF; v++) Pt[v] = P[v] + lam * dPv[v];
      zone_residual<COND, VISC, double, double>(Pt, K, G, c, Rt);
      const double f1 = 0.5 * l2sum<NF>(Rt);
      const double alpha = 1e-4;
      if (!(f1 > (f0 * (1. - alpha * lam) + c.lsFloor))) { haveRt = true; break; }
      const double denom = (f1 - f0 - fPrime0 * lam);
      lam = -fPrime0 * lam * lam / denom / 2.;
    }
#pragma unroll
    for (int v = 0; v < NF; v++) P[v] = P[v] + lam * dPv[v];
    if (it + 1 < c.maxIter) {
      const bool floored = (P[0] < c.rhoFloor) || (P[1] < c.uFloor);
      P[0] = fmax(P[0], c.rhoFloor);
      P[1] = fmax(P[1], c.uFloor);
      if (!haveRt || floored) zone_residual<COND, VISC, double, double>(P, K, G, c, Rt);
      const double l2n = l2sum<NF>(Rt);
#pragma unroll
      for (int v = 0; v < NF; v++) b.R[(long long)v * Z + z] = Rt[v];
      b.l2[z] = l2n;
      double tol = newton_tol(c, l2first, K);
      unconv = (l2n > tol) ? 1 : 0;
    }
#pragma unroll
    for (int v = 0; v < NF; v++) b.prim[(long long)v * Z + z] = P[v];
  }
  unconv = __syncthreads_count(unconv);
  if (threadIdx.x == 0) {
    if (unconv) atomicAdd(&b.st->count[stage][it + 1], (unsigned long long)unconv);
    if (blockIdx.x == 0) atomicAdd(&b.st->itersDone[stage], 1ULL);
  }
}

// ---------------------------------------------------------------------------
// Fast Newton: per-zone convergence, exact Jacobian from one forward-tangent
// pass of the residual; T = double (TANGENT64) or float (MIXED32: Jacobian
// and solve in FP32, residual in FP64, i.e. FP32 inexact Newton refined by
// the FP64 residual).
// ---------------------------------------------------------------------------
template <int COND, int VISC, class T, bool GENERIC = false>
GRIM_D void tangent_jacobian(const double* P, const StageConst<5 + COND + VISC>& K, const ZoneGeo<T>& Gt,
                             const DevCfg& c, T J[5 + COND + VISC][5 + COND + VISC]) {
  constexpr int NF = 5 + COND + VISC;
  if constexpr (COND == 0 && VISC == 0 && !GENERIC) {
    // ideal MHD: the closed-form dU/dP
    ideal_jacobian<T>(P, K, Gt, c, J);
    return;
  }
  typedef Dual<T, NF> D;
  D Pd[NF], Rd[NF];
#pragma unroll
  for (int v = 0; v < NF; v++) Pd[v] = D::var((T)P[v], v);
  zone_residual<COND, VISC, D, T>(Pd, K, Gt, c, Rd);
#pragma unroll
  for (int r = 0; r < NF; r++)
#pragma unroll
    for (int cc = 0; cc < NF; cc++) J[r][cc] = Rd[r].d[cc];
}

// One zone's fast Newton from iteration `it` up to (not including) itEnd:
// at the top of each iteration the floors, the residual where the last
// line search did not leave one, and the per-zone test; then the Jacobian,
// the solve and the backtracking line search (solve.cpp:80-199 per zone).
// Returns with conv set when the test passed (`it` = the updates taken) or
// with it == itEnd.
template <int COND, int VISC, class T>
GRIM_D void fast_newton_iters(const DevCfg& c, const StageConst<5 + COND + VISC>& K, const ZoneGeo<double>& G,
                              double* P, double* R, bool& haveR, double& l2first, int& it, bool& conv,
                              int itEnd) {
  constexpr int NF = 5 + COND + VISC;
  for (; it < itEnd; it++) {
    const bool floored = (P[0] < c.rhoFloor) || (P[1] < c.uFloor);
    P[0] = fmax(P[0], c.rhoFloor);
    P[1] = fmax(P[1], c.uFloor);
    if (!haveR || floored) zone_residual<COND, VISC, double, double>(P, K, G, c, R);
    const double l2 = l2sum<NF>(R);
    if (it == 0) l2first = l2;
    if (l2 <= newton_tol(c, l2first, K)) { conv = true; return; }
    T J[NF][NF];
    {
      // the Jacobian's geometry, converted where it is used rather than
      // kept beside the FP64 copy across the iterations
      ZoneGeo<T> Gt;
#pragma unroll
      for (int m = 0; m < 4; m++)
#pragma unroll
        for (int q = 0; q < 4; q++) { Gt.gcov[m][q] = (T)G.gcov[m][q]; Gt.gcon[m][q] = (T)G.gcon[m][q]; }
      Gt.g = (T)G.g; Gt.alpha = (T)G.alpha; Gt.ialpha = (T)G.ialpha; Gt.x1 = (T)G.x1; Gt.x2 = (T)G.x2; Gt.dyn = (T)G.dyn;
      tangent_jacobian<COND, VISC, T>(P, K, Gt, c, J);
    }
    T bv[NF], xv[NF];
#pragma unroll
    for (int v = 0; v < NF; v++) bv[v] = (T)(-R[v]);
    gauss_solve<T, NF>(J, bv, xv);
    double dPv[NF];
#pragma unroll
    for (int v = 0; v < NF; v++) dPv[v] = (double)xv[v];
    const double f0 = 0.5 * l2, fPrime0 = -2. * f0;
    double lam = 1.;
    haveR = false;
    double Rt[NF];
    for (int ls = 0; ls < c.maxLS; ls++) {
      double Pt[NF];
#pragma unroll
      for (int v = 0; v < NF; v++) Pt[v] = P[v] + lam * dPv[v];
      zone_residual<COND, VISC, double, double>(Pt, K, G, c, Rt);
      const double f1 = 0.5 * l2sum<NF>(Rt);
      if (!(f1 > (f0 * (1. - 1e-4 * lam) + c.lsFloor))) { haveR = true; break; }
      const double denom = (f1 - f0 - fPrime0 * lam);
      lam = -fPrime0 * lam * lam / denom / 2.;
    }
#pragma unroll
    for (int v = 0; v < NF; v++) {
      P[v] = P[v] + lam * dPv[v];
      if (haveR) R[v] = Rt[v];
    }
  }
}

// The test of a zone that used every iteration, on the state it returns; a
// last step whose line search ran out was applied unevaluated: its residual
// is formed here, at the floored state the next iteration would see.
// Returns true when the zone is above tolerance.
template <int COND, int VISC>
GRIM_D bool fast_newton_final(const DevCfg& c, const StageConst<5 + COND + VISC>& K, const ZoneGeo<double>& G,
                              const double* P, double* R, bool haveR, double l2first) {
  constexpr int NF = 5 + COND + VISC;
  if (!haveR) {
    double Pf[NF];
#pragma unroll
    for (int v = 0; v < NF; v++) Pf[v] = P[v];
    Pf[0] = fmax(Pf[0], c.rhoFloor);
    Pf[1] = fmax(Pf[1], c.uFloor);
    zone_residual<COND, VISC, double, double>(Pf, K, G, c, R);
  }
  const double l2 = l2sum<NF>(R);
  return !(l2 >= 0. && l2 <= newton_tol(c, l2first, K));
}

constexpr int kNewtonMinBlocks = 3;  // blocks per SM of the ideal FP32-Jacobian Newton
template <int COND, int VISC, class T>
__global__ void __launch_bounds__(128, (COND || VISC || sizeof(T) == 8) ? 1 : kNewtonMinBlocks) k_newton_fast(DevCfg c, int stage, StageBufs b,
                                                              const int* __restrict__ list, long long nlist) {
  constexpr int NF = 5 + COND + VISC;
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int unconv = 0, itsMax = 0;
  bool nanZone = false;
  if (n < nlist) {
    const long long Z = c.Z;
    const long long z = list ? (long long)list[n] : interior_to_z(c, n);
    int i, j, k;
    zijk(c, z, i, j, k);
    ZoneGeo<double> G;
    load_geo(G, c, b.geoC, z, i, j, 0.5, 0.5);
    StageConst<NF> K;
    load_stage_const<COND, VISC>(K, c, stage, b, z, G);
    double P[NF], R[NF];
    const double* guess = (stage == GRIM_HALF_STEP && b.guessOld) ? b.pold : b.prim;
#pragma unroll
    for (int v = 0; v < NF; v++) P[v] = guess[(long long)v * Z + z];
    bool haveR = false, conv = false;
    double l2first = 0.;
    int it = 0;
    fast_newton_iters<COND, VISC, T>(c, K, G, P, R, haveR, l2first, it, conv, c.maxIter);
    if (!conv && it == c.maxIter) unconv = fast_newton_final<COND, VISC>(c, K, G, P, R, haveR, l2first) ? 1 : 0;
    itsMax = it;
#pragma unroll
    for (int v = 0; v < NF; v++) b.prim[(long long)v * Z + z] = P[v];
    if (b.nanCount) {
#pragma unroll
      for (int v = 0; v < NF; v++) nanZone |= isnan(P[v]);
#pragma unroll
      for (int v = 0; v < 3; v++) nanZone |= isnan(K.B[v]);
    }
  }
  hist_add(b.st->itHist[stage], min(itsMax, 15), n < nlist);
  // warp-level tallies: no block barrier, so a warp whose zones converged
  // early retires without waiting for the rest of its block
  const int nUnconv = __popc(__ballot_sync(0xffffffffu, unconv != 0));
  for (int o = 16; o > 0; o >>= 1) itsMax = max(itsMax, __shfl_xor_sync(0xffffffffu, itsMax, o));
  const int nNan = __popc(__ballot_sync(0xffffffffu, nanZone));
  if ((threadIdx.x & 31) == 0) {
    atomicMax((unsigned long long*)&b.st->itersDone[stage], (unsigned long long)itsMax);
    if (nUnconv) atomicAdd(&b.st->finalUnconv[stage], (unsigned long long)nUnconv);
    if (nNan) atomicAdd(b.nanCount, (unsigned long long)nNan);
  }
}

#ifdef GRIM_FAST_MATH
// ---------------------------------------------------------------------------
// Deferred-tail fast Newton, ideal MHD: a persistent kernel whose warps take
// batches of 32 consecutive zones and run each zone's first maxIter - 1
// updates together; a zone still above tolerance then goes, with its state,
// onto its warp's stash in shared memory, and whenever the stash holds 32
// zones the warp runs their last update as one full batch.  Most zones
// converge one update before the cap, so the per-zone kernel's warps nearly
// all run the last update for a few lanes; here it runs on full warps
// only.  The per-zone arithmetic is fast_newton_iters / fast_newton_final,
// as in k_newton_fast: the results are the same bits.  The stash keeps what
// the ideal residual and Jacobian read besides the geometry (reloaded, it
// is the same for every stage): B, Kc, the rounding floor; dt' comes from
// the step's dt as in load_stage_const.
// ---------------------------------------------------------------------------
constexpr int kDeferWarps = 4;  // warps per block
constexpr int kDeferCap = 64;   // stash slots per warp (< 32 left + 32 pushed)
struct DeferStash {
  double P[5][kDeferCap];
  double R[5][kDeferCap];
  double Kc[5][kDeferCap];
  double B[3][kDeferCap];
  double l2first[kDeferCap];
  double tolFloor2[kDeferCap];
  int z[kDeferCap];
  int haveR[kDeferCap];
};

template <class T>
__global__ void __launch_bounds__(32 * kDeferWarps, kNewtonMinBlocks) k_newton_defer(DevCfg c, int stage, StageBufs b,
                                                                                  long long nlist) {
  constexpr int NF = 5;
  __shared__ DeferStash stashes[kDeferWarps];
  const int lane = threadIdx.x & 31;
  DeferStash& S = stashes[threadIdx.x >> 5];
  const long long Z = c.Z;
  const int split = c.maxIter - 1;
  const double dt = b.st->dt;
  const double dtp = (stage == GRIM_HALF_STEP) ? dt / 2. : dt;
  const double* guess = (stage == GRIM_HALF_STEP && b.guessOld) ? b.pold : b.prim;
  const long long nbatch = (nlist + 31) / 32;
  const long long stride = (long long)gridDim.x * kDeferWarps;
  long long bt = (long long)blockIdx.x * kDeferWarps + (threadIdx.x >> 5);
  int held = 0;                           // warp-uniform stash fill
  int itsMax = 0, nUnconv = 0, nNan = 0;  // this lane's tallies
  // one task per pass, the same for the whole warp: the last update of 32
  // stashed zones when the stash holds 32, else the first maxIter - 1
  // updates of the next batch, else the last update of what is left
  for (;;) {
    bool tail;
    int from = 0, count = 32;
    if (held >= 32) {
      tail = true;
      held -= 32;
      from = held;
    } else if (bt < nbatch) {
      tail = false;
    } else if (held > 0) {
      tail = true;
      count = held;
      held = 0;
    } else {
      break;
    }
    const long long n = bt * 32 + lane;
    const bool act = tail ? lane < count : n < nlist;
    long long z = 0;
    StageConst<NF> K;
    double P[NF], R[NF], l2first = 0.;
    bool haveR = false, conv = false;
    int it = tail ? split : 0;
    if (act) {
      const int sl = from + lane;
      z = tail ? (long long)S.z[sl] : interior_to_z(c, n);
      int i, j, k;
      zijk(c, z, i, j, k);
      ZoneGeo<double> G;
      load_geo(G, c, b.geoC, z, i, j, 0.5, 0.5);
      if (tail) {
        K.dtp = dtp;
        K.idtp = 1. / dtp;
#pragma unroll
        for (int v = 0; v < NF; v++) { K.Kc[v] = S.Kc[v][sl]; P[v] = S.P[v][sl]; R[v] = S.R[v][sl]; }
#pragma unroll
        for (int v = 0; v < 3; v++) K.B[v] = S.B[v][sl];
        K.tolFloor2 = S.tolFloor2[sl];
        haveR = S.haveR[sl] != 0;
        l2first = S.l2first[sl];
      } else {
        load_stage_const<0, 0>(K, c, stage, b, z, G);
#pragma unroll
        for (int v = 0; v < NF; v++) P[v] = guess[(long long)v * Z + z];
      }
      fast_newton_iters<0, 0, T>(c, K, G, P, R, haveR, l2first, it, conv, tail ? c.maxIter : split);
      if (tail && !conv) nUnconv += fast_newton_final<0, 0>(c, K, G, P, R, haveR, l2first) ? 1 : 0;
      if (tail || conv) {
        itsMax = max(itsMax, it);
#pragma unroll
        for (int v = 0; v < NF; v++) b.prim[(long long)v * Z + z] = P[v];
        if (b.nanCount) {
          bool nz = false;
#pragma unroll
          for (int v = 0; v < NF; v++) nz |= isnan(P[v]);
#pragma unroll
          for (int v = 0; v < 3; v++) nz |= isnan(K.B[v]);
          nNan += nz ? 1 : 0;
        }
      }
    }
    hist_add(b.st->itHist[stage], min(it, 15), act && (tail || conv));
    if (!tail) {
      // the zones of the batch still above tolerance onto the stash
      const bool defer = act && !conv;
      const unsigned m = __ballot_sync(0xffffffffu, defer);
      if (defer) {
        const int sl = held + __popc(m & ((1u << lane) - 1u));
        S.z[sl] = (int)z;
#pragma unroll
        for (int v = 0; v < NF; v++) { S.P[v][sl] = P[v]; S.R[v][sl] = R[v]; S.Kc[v][sl] = K.Kc[v]; }
#pragma unroll
        for (int v = 0; v < 3; v++) S.B[v][sl] = K.B[v];
        S.l2first[sl] = l2first;
        S.tolFloor2[sl] = K.tolFloor2;
        S.haveR[sl] = haveR ? 1 : 0;
      }
      held += __popc(m);
      bt += stride;
    }
    __syncwarp();
  }
  // warp tallies
  for (int o = 16; o > 0; o >>= 1) {
    itsMax = max(itsMax, __shfl_xor_sync(0xffffffffu, itsMax, o));
    nUnconv += __shfl_xor_sync(0xffffffffu, nUnconv, o);
    nNan += __shfl_xor_sync(0xffffffffu, nNan, o);
  }
  if (lane == 0) {
    atomicMax((unsigned long long*)&b.st->itersDone[stage], (unsigned long long)itsMax);
    if (nUnconv) atomicAdd(&b.st->finalUnconv[stage], (unsigned long long)nUnconv);
    if (nNan) atomicAdd(b.nanCount, (unsigned long long)nNan);
  }
}
#endif  // GRIM_FAST_MATH

// ---------------------------------------------------------------------------
// Compacted fast Newton: one launch per iteration over a worklist of the
// zones still above tolerance, so no warp carries converged lanes.  The
// state between launches (P in prim, R, l2first) lives in HBM; worklists are
// appended with warp-aggregated atomics.  Launch 0 floors, evaluates the
// residual and lists the unconverged zones; launch it >= 1 does Newton
// iteration it-1 on list[(it-1)&1] and lists the zones still unconverged.
// ---------------------------------------------------------------------------
GRIM_D void list_append(int* list, unsigned long long* count, int zone, bool take) {
  const unsigned m = __ballot_sync(0xffffffffu, take);
  if (m == 0) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (take) list[base + __popc(m & ((1u << lane) - 1))] = zone;
}

// Launch 0, one zone: floors, residual, stored state; true when the zone
// is above tolerance (goes on the worklist).
template <int COND, int VISC>
GRIM_D bool list_init_zone(const DevCfg& c, int stage, const StageBufs& b, long long z) {
  constexpr int NF = 5 + COND + VISC;
  const long long Z = c.Z;
  int i, j, k;
  zijk(c, z, i, j, k);
  ZoneGeo<double> G;
  load_geo(G, c, b.geoC, z, i, j, 0.5, 0.5);
  StageConst<NF> K;
  load_stage_const<COND, VISC>(K, c, stage, b, z, G);
  double P[NF], R[NF];
#pragma unroll
  for (int v = 0; v < NF; v++) P[v] = b.prim[(long long)v * Z + z];
  P[0] = fmax(P[0], c.rhoFloor);
  P[1] = fmax(P[1], c.uFloor);
  b.prim[z] = P[0];
  b.prim[Z + z] = P[1];
  zone_residual<COND, VISC, double, double>(P, K, G, c, R);
  const double l2 = l2sum<NF>(R);
#pragma unroll
  for (int v = 0; v < NF; v++) b.R[(long long)v * Z + z] = R[v];
  b.l2[Z + z] = l2;
  return l2 > newton_tol(c, l2, K);
}

// Launch it >= 1, one zone on the worklist: one Newton update from the
// stored state; true when the zone stays above tolerance (and it is not
// the last iteration).
template <int COND, int VISC, class T>
GRIM_D bool list_iter_zone(const DevCfg& c, int stage, int it, const StageBufs& b, long long z) {
  constexpr int NF = 5 + COND + VISC;
  const long long Z = c.Z;
  const bool last = (it == c.maxIter);
  int i, j, k;
  zijk(c, z, i, j, k);
  ZoneGeo<double> G;
  load_geo(G, c, b.geoC, z, i, j, 0.5, 0.5);
  ZoneGeo<T> Gt;
#pragma unroll
  for (int m = 0; m < 4; m++)
#pragma unroll
    for (int q = 0; q < 4; q++) { Gt.gcov[m][q] = (T)G.gcov[m][q]; Gt.gcon[m][q] = (T)G.gcon[m][q]; }
  Gt.g = (T)G.g; Gt.alpha = (T)G.alpha; Gt.ialpha = (T)G.ialpha; Gt.x1 = (T)G.x1; Gt.x2 = (T)G.x2; Gt.dyn = (T)G.dyn;
  StageConst<NF> K;
  load_stage_const<COND, VISC>(K, c, stage, b, z, G);
  double P[NF], R[NF];
#pragma unroll
  for (int v = 0; v < NF; v++) {
    P[v] = b.prim[(long long)v * Z + z];
    R[v] = b.R[(long long)v * Z + z];
  }
  const double l2 = l2sum<NF>(R);
  const double l2first = b.l2[Z + z];
  T J[NF][NF];
  tangent_jacobian<COND, VISC, T>(P, K, Gt, c, J);
  T bv[NF], xv[NF];
#pragma unroll
  for (int v = 0; v < NF; v++) bv[v] = (T)(-R[v]);
  gauss_solve<T, NF>(J, bv, xv);
  double dPv[NF];
#pragma unroll
  for (int v = 0; v < NF; v++) dPv[v] = (double)xv[v];
  const double f0 = 0.5 * l2, fPrime0 = -2. * f0;
  double lam = 1.;
  bool haveR = false;
  double Rt[NF];
  for (int ls = 0; ls < c.maxLS; ls++) {
    double Pt[NF];
#pragma unroll
    for (int v = 0; v < NF; v++) Pt[v] = P[v] + lam * dPv[v];
    zone_residual<COND, VISC, double, double>(Pt, K, G, c, Rt);
    const double f1 = 0.5 * l2sum<NF>(Rt);
    if (!(f1 > (f0 * (1. - 1e-4 * lam) + c.lsFloor))) { haveR = true; break; }
    const double denom = (f1 - f0 - fPrime0 * lam);
    lam = -fPrime0 * lam * lam / denom / 2.;
  }
#pragma unroll
  for (int v = 0; v < NF; v++) P[v] = P[v] + lam * dPv[v];
  const bool floored = (P[0] < c.rhoFloor) || (P[1] < c.uFloor);
  if (!last) {
    P[0] = fmax(P[0], c.rhoFloor);
    P[1] = fmax(P[1], c.uFloor);
  }
  if (!haveR || floored) zone_residual<COND, VISC, double, double>(P, K, G, c, Rt);
  const double l2n = l2sum<NF>(Rt);
  const bool conv = l2n <= newton_tol(c, l2first, K);
  if (!conv && last) atomicAdd(&b.st->finalUnconv[stage], 1ULL);
#pragma unroll
  for (int v = 0; v < NF; v++) {
    b.prim[(long long)v * Z + z] = P[v];
    b.R[(long long)v * Z + z] = Rt[v];
  }
  return !conv && !last;
}

template <int COND, int VISC>
__global__ void __launch_bounds__(128) k_newton_list_init(DevCfg c, int stage, StageBufs b) {
  for (long long n0 = (long long)blockIdx.x * blockDim.x; n0 < c.Zint; n0 += (long long)gridDim.x * blockDim.x) {
    const long long n = n0 + threadIdx.x;
    bool take = false;
    long long z = 0;
    if (n < c.Zint) {
      z = interior_to_z(c, n);
      take = list_init_zone<COND, VISC>(c, stage, b, z);
    }
    hist_add(b.st->itHist[stage], 0, n < c.Zint && !take);
    list_append(b.list[0], &b.st->listCount[0], (int)z, take);
  }
}

template <int COND, int VISC, class T>
__global__ void __launch_bounds__(128) k_newton_list_iter(DevCfg c, int stage, int it, StageBufs b) {
  const int in = (it - 1) & 1, out = it & 1;
  const long long count = (long long)b.st->listCount[in];
  const bool last = (it == c.maxIter);
  for (long long n0 = (long long)blockIdx.x * blockDim.x; n0 < count; n0 += (long long)gridDim.x * blockDim.x) {
    const long long n = n0 + threadIdx.x;
    bool take = false;
    int zone = 0;
    if (n < count) {
      zone = b.list[in][n];
      take = list_iter_zone<COND, VISC, T>(c, stage, it, b, zone);
    }
    hist_add(b.st->itHist[stage], min(it, 15), n < count && !take);
    if (!last) list_append(b.list[out], &b.st->listCount[out], zone, take);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && count > 0) atomicMax(&b.st->itersDone[stage], (unsigned long long)it);
}

// ---------------------------------------------------------------------------
// Ragged batch: the compacted Newton of several independent problems (grid
// sizes may differ) in one launch per iteration.  Worklist entries are
// global interior indices over the concatenated problems; each lane finds
// its problem in the offset table and runs the same per-zone code with that
// problem's configuration and buffers.
// ---------------------------------------------------------------------------
GRIM_D int batch_problem(const BatchEntry* tbl, int nprob, long long g) {
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tbl[mid].offset <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
// histogram add keyed by (problem, bin): one atomic per distinct key in a warp
GRIM_D void batch_hist_add(const BatchEntry* tbl, int stage, int p, int bin, bool active) {
  const unsigned act = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const unsigned peers = __match_any_sync(act, p * 16 + bin);
  if ((threadIdx.x & 31) == __ffs(peers) - 1)
    atomicAdd(&tbl[p].b[stage].st->itHist[stage][bin], (unsigned long long)__popc(peers));
}

template <int COND, int VISC>
__global__ void __launch_bounds__(128) k_batch_list_init(const BatchEntry* __restrict__ tbl, int nprob,
                                                         long long total, int stage, BatchState* bs) {
  for (long long n0 = (long long)blockIdx.x * blockDim.x; n0 < total; n0 += (long long)gridDim.x * blockDim.x) {
    const long long gidx_ = n0 + threadIdx.x;
    bool take = false;
    int p = 0;
    if (gidx_ < total) {
      p = batch_problem(tbl, nprob, gidx_);
      const DevCfg& c = tbl[p].c;
      const long long z = interior_to_z(c, gidx_ - tbl[p].offset);
      take = list_init_zone<COND, VISC>(c, stage, tbl[p].b[stage], z);
    }
    batch_hist_add(tbl, stage, p, 0, gidx_ < total && !take);
    list_append(bs->list[0], &bs->listCount[0], (int)gidx_, take);
  }
}

template <int COND, int VISC, class T>
__global__ void __launch_bounds__(128) k_batch_list_iter(const BatchEntry* __restrict__ tbl, int nprob, int stage,
                                                         int it, int lastIt, BatchState* bs) {
  const int in = (it - 1) & 1, out = it & 1;
  const long long count = (long long)bs->listCount[in];
  for (long long n0 = (long long)blockIdx.x * blockDim.x; n0 < count; n0 += (long long)gridDim.x * blockDim.x) {
    const long long n = n0 + threadIdx.x;
    bool take = false;
    int gidx_ = 0, p = 0;
    if (n < count) {
      gidx_ = bs->list[in][n];
      p = batch_problem(tbl, nprob, gidx_);
      const DevCfg& c = tbl[p].c;
      const long long z = interior_to_z(c, gidx_ - tbl[p].offset);
      // a problem past its own maxIter leaves the list (its last update
      // was counted there)
      if (it <= c.maxIter) take = list_iter_zone<COND, VISC, T>(c, stage, it, tbl[p].b[stage], z);
    }
    batch_hist_add(tbl, stage, p, min(it, 15), n < count && !take);
    {
      // iterations done, per problem: one atomic per problem in the warp
      const unsigned act = __ballot_sync(0xffffffffu, n < count);
      if (n < count) {
        const unsigned peers = __match_any_sync(act, p);
        if ((threadIdx.x & 31) == __ffs(peers) - 1)
          atomicMax(&tbl[p].b[stage].st->itersDone[stage], (unsigned long long)it);
      }
    }
    if (it < lastIt) list_append(bs->list[out], &bs->listCount[out], gidx_, take);
  }
}

// ---------------------------------------------------------------------------
// kernels behind the test entry points
// ---------------------------------------------------------------------------
template <int COND, int VISC>
__global__ void k_residual(DevCfg c, int stage, StageBufs b, const double* __restrict__ pg,
                                    double* __restrict__ out) {
  constexpr int NF = 5 + COND + VISC;
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  const long long Z = c.Z;
  int i, j, k;
  zijk(c, z, i, j, k);
  bool inner = i >= c.g1 && i < c.N1 + c.g1 && j >= c.g2 && j < c.N2 + c.g2 && k >= c.g3 && k < c.N3 + c.g3;
  if (!inner) {
#pragma unroll
    for (int v = 0; v < NF; v++) out[(long long)v * Z + z] = 0.;
    return;
  }
  ZoneGeo<double> G;
  load_geo(G, c, b.geoC, z, i, j, 0.5, 0.5);
  StageConst<NF> K;
  load_stage_const<COND, VISC>(K, c, stage, b, z, G);
#pragma unroll
  for (int v = 0; v < 3; v++) K.B[v] = pg[(long long)(c.B1 + v) * Z + z];
  double P[NF], R[NF];
#pragma unroll
  for (int v = 0; v < NF; v++) P[v] = pg[(long long)v * Z + z];
  zone_residual<COND, VISC, double, double>(P, K, G, c, R);
#pragma unroll
  for (int v = 0; v < NF; v++) out[(long long)v * Z + z] = R[v];
}

template <int COND, int VISC>
__global__ void k_jacobian(DevCfg c, int stage, StageBufs b, const double* __restrict__ pg,
                                    double* __restrict__ jac, int tangent) {
  constexpr int NF = 5 + COND + VISC;
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  const long long Z = c.Z;
  int i, j, k;
  zijk(c, z, i, j, k);
  bool inner = i >= c.g1 && i < c.N1 + c.g1 && j >= c.g2 && j < c.N2 + c.g2 && k >= c.g3 && k < c.N3 + c.g3;
  double J[NF][NF];
#pragma unroll
  for (int a = 0; a < NF; a++)
#pragma unroll
    for (int q = 0; q < NF; q++) J[a][q] = 0.;
  if (inner) {
    ZoneGeo<double> G;
    load_geo(G, c, b.geoC, z, i, j, 0.5, 0.5);
    StageConst<NF> K;
    load_stage_const<COND, VISC>(K, c, stage, b, z, G);
#pragma unroll
    for (int v = 0; v < 3; v++) K.B[v] = pg[(long long)(c.B1 + v) * Z + z];
    double P[NF], R[NF];
#pragma unroll
    for (int v = 0; v < NF; v++) P[v] = pg[(long long)v * Z + z];
    if (tangent == 1) {
      tangent_jacobian<COND, VISC, double>(P, K, G, c, J);
    } else if (tangent == 2) {
      tangent_jacobian<COND, VISC, double, true>(P, K, G, c, J);
    } else if (tangent == 3) {
      // the form and precision the mixed Newton uses: geometry rounded to
      // FP32, the Jacobian in FP32
      ZoneGeo<float> Gt;
#pragma unroll
      for (int m = 0; m < 4; m++)
#pragma unroll
        for (int q = 0; q < 4; q++) { Gt.gcov[m][q] = (float)G.gcov[m][q]; Gt.gcon[m][q] = (float)G.gcon[m][q]; }
      Gt.g = (float)G.g; Gt.alpha = (float)G.alpha; Gt.ialpha = (float)G.ialpha; Gt.x1 = (float)G.x1;
      Gt.x2 = (float)G.x2; Gt.dyn = (float)G.dyn;
      float Jf[NF][NF];
      tangent_jacobian<COND, VISC, float>(P, K, Gt, c, Jf);
#pragma unroll
      for (int a = 0; a < NF; a++)
#pragma unroll
        for (int q = 0; q < NF; q++) J[a][q] = (double)Jf[a][q];
    } else {
      zone_residual<COND, VISC, double, double>(P, K, G, c, R);
      const double eps = c.jacEps;
#pragma unroll
      for (int row = 0; row < NF; row++) {
        double Pe[NF];
#pragma unroll
        for (int v = 0; v < NF; v++) Pe[v] = P[v];
        double small = (fabs(P[row]) < .5 * eps) ? 1. : 0.;
        Pe[row] = P[row] + eps * P[row] * (1. - small) + small * eps;
        double Rp[NF];
        zone_residual<COND, VISC, double, double>(Pe, K, G, c, Rp);
#pragma unroll
        for (int col = 0; col < NF; col++) J[col][row] = (Rp[col] - R[col]) / (Pe[row] - P[row]);
      }
    }
  }
#pragma unroll
  for (int a = 0; a < NF; a++)
#pragma unroll
    for (int q = 0; q < NF; q++) jac[(z * NF + a) * NF + q] = J[a][q];
}

// the centre element of a prim array: its fluxes along X^fdir into out
// (fluidElement::computeFluxes, physics.cpp:185-217; fdir 0 gives the
// conserved variables) and / or its characteristic speeds along the
// spatial direction dir into mn, mx
template <int COND, int VISC>
__global__ void k_conserved(DevCfg c, const double* __restrict__ p, const double* __restrict__ geoC,
                                     double* __restrict__ out, int fdir, int dir, double* mn, double* mx) {
  constexpr int NF = 5 + COND + VISC;
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  const long long Z = c.Z;
  int i, j, k;
  zijk(c, z, i, j, k);
  ZoneGeo<double> G;
  load_geo(G, c, geoC, z, i, j, 0.5, 0.5);
  ElemT<double, double> e;
  elem_set<COND, VISC>(e, p[z], p[Z + z], p[2 * Z + z], p[3 * Z + z], p[4 * Z + z], p[(long long)c.B1 * Z + z],
                       p[(long long)(c.B1 + 1) * Z + z], p[(long long)(c.B1 + 2) * Z + z],
                       COND ? p[(long long)c.Q * Z + z] : 0., VISC ? p[(long long)c.DP * Z + z] : 0., G, c);
  if (out) {
    double U[NF], UB[3];
    fluxes_fluid<COND, VISC>(e, fdir, G.g, U, 5, 5 + COND);
    fluxes_B(e, fdir, G.g, UB);
#pragma unroll
    for (int v = 0; v < NF; v++) out[(long long)v * Z + z] = U[v];
#pragma unroll
    for (int v = 0; v < 3; v++) out[(long long)(NF + v) * Z + z] = UB[v];
  }
  if (mn) {
    double a, bb;
    char_speeds<COND, VISC>(e, G, dir, c, a, bb);
    mn[z] = a;
    mx[z] = bb;
  }
}

// reconstruction of one direction for every zone (test entry point)
static __global__ void k_reconstruct(DevCfg c, int dir, const double* __restrict__ p, double* __restrict__ pl,
                                       double* __restrict__ pr) {
  long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  int i, j, k;
  zijk(c, z, i, j, k);
  const int NT = (dir == 0) ? c.N1T : (dir == 1 ? c.N2T : c.N3T);
  const int x = (dir == 0) ? i : (dir == 1 ? j : k);
  const long long s = stride_of(c, dir);
  for (int v = 0; v < c.dof; v++) {
    const double* a = p + (long long)v * c.Z;
    double y[5];
#pragma unroll
    for (int m = 0; m < 5; m++) {
      int xx = x + m - 2;
      xx = ((xx % NT) + NT) % NT;  // circular, af::shift semantics
      y[m] = a[z + (long long)(xx - x) * s];
    }
    double lo, ro;
    recon_faces(c.reconstruction, c.theta, y[0], y[1], y[2], y[3], y[4], lo, ro);
    pl[(long long)v * c.Z + z] = lo;
    pr[(long long)v * c.Z + z] = ro;
  }
}

// batched dense solve (test entry point), one system per thread
template <int N>
__global__ void k_batch_solve(int batch, const double* __restrict__ A, const double* __restrict__ b,
                                       double* __restrict__ x) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= batch) return;
  double a[N][N], bb[N], xx[N];
#pragma unroll
  for (int r = 0; r < N; r++) {
    bb[r] = b[n * N + r];
#pragma unroll
    for (int q = 0; q < N; q++) a[r][q] = A[(n * N + r) * N + q];
  }
  gauss_solve<double, N>(a, bb, xx);
#pragma unroll
  for (int r = 0; r < N; r++) x[n * N + r] = xx[r];
}

// non-finite primitives count (diagnostic after each step)
static __global__ void k_count_nonfinite(DevCfg c, const double* __restrict__ p, DevState* st) {
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int bad = 0;
  if (n < c.Zint) {
    long long z = interior_to_z(c, n);
    for (int v = 0; v < c.dof; v++) {
      double a = p[(long long)v * c.Z + z];
      if (!isfinite(a)) bad = 1;
    }
  }
  bad = __syncthreads_count(bad);
  if (threadIdx.x == 0 && bad) atomicAdd(&st->nonFinite, (unsigned long long)bad);
}

}  // namespace GRIM_KNS
}  // namespace grim

// ---------------------------------------------------------------------------
// launchers (declared in launch.h)
// ---------------------------------------------------------------------------
namespace grim {
namespace GRIM_KNS {

static inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

#define GRIM_EMHD_DISPATCH(c, KERNEL, ...)                              \
  do {                                                                  \
    if ((c).conduction && (c).viscosity) KERNEL<1, 1>(__VA_ARGS__);     \
    else if ((c).conduction) KERNEL<1, 0>(__VA_ARGS__);                 \
    else if ((c).viscosity) KERNEL<0, 1>(__VA_ARGS__);                  \
    else KERNEL<0, 0>(__VA_ARGS__);                                     \
  } while (0)

#if !defined(GRIM_ONLY_FACES)
void ghost_fill(const DevCfg& c, double* prim, int nv, cudaStream_t s) {
  if (c.Z > c.Zint) k_ghost_fill<<<nblk(c.Z - c.Zint, 256), 256, 0, s>>>(c, prim, nv);
}
void communicate(const DevCfg& c, double* prim, int nv, cudaStream_t s) {
  k_communicate<<<nblk(c.Z, 256), 256, 0, s>>>(c, prim, nv);
}

template <int C, int V>
static void emhd_prepass_t(const DevCfg& c, const double* ps, const double* geoC, double* uT, cudaStream_t s) {
  k_emhd_prepass<C, V><<<nblk(c.Z, 128), 128, 0, s>>>(c, ps, geoC, uT);
}
void emhd_prepass(const DevCfg& c, const double* ps, const double* geoC, double* uT, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, emhd_prepass_t, c, ps, geoC, uT, s);
}

#endif  // !GRIM_ONLY_FACES

#if !defined(GRIM_SKIP_FACES)
// Launch-shape variants of the face kernels, chosen per direction by the
// autotuner (grim_autotune): X1 faces by the register budget (3 or 4
// resident 128-thread blocks per SM), X2 / X3 faces by that budget and by
// the lane split QI (i per warp).  EMHD has one shape (2 resident blocks).
// the reconstruction scheme is a compile-time constant of the X1 kernels
// as of the TMA ones: one scheme's code per kernel keeps the instruction
// footprint small
template <int C, int V, int MINB, bool PAIR = false>
static void face_x1_launch(const DevCfg& c, const double* ps, const double* geoF, double* flux, cudaStream_t s) {
  const long long warps = (long long)c.nfj * c.nfk * ((c.N1T - 5 + 30) / 31);
  const size_t park = PAIR ? 0 : 3 * (8 + C + V) * 128 * sizeof(double);
  const unsigned nb = nblk(warps * 32, 128);
  switch (c.reconstruction) {
    case GRIM_WENO5: k_face_flux_x1<C, V, MINB, PAIR, GRIM_WENO5><<<nb, 128, park, s>>>(c, ps, geoF, flux); break;
    case GRIM_PPM: k_face_flux_x1<C, V, MINB, PAIR, GRIM_PPM><<<nb, 128, park, s>>>(c, ps, geoF, flux); break;
    case GRIM_MP5: k_face_flux_x1<C, V, MINB, PAIR, GRIM_MP5><<<nb, 128, park, s>>>(c, ps, geoF, flux); break;
    default: k_face_flux_x1<C, V, MINB, PAIR, GRIM_MINMOD><<<nb, 128, park, s>>>(c, ps, geoF, flux); break;
  }
}
template <int C, int V, int QI, int MINB, bool PAIR = false>
static void face_strip_launch(const DevCfg& c, int dir, const double* ps, const double* geoF, const double* geoC,
                              double* flux, cudaStream_t s) {
  const int NT = (dir == 1) ? c.N2T : c.N3T;
  const long long other = (dir == 1) ? c.nfk : c.nfj;
  const long long warps = (long long)((c.N1T + QI - 1) / QI) * ((NT - 5 + 32 / QI - 2) / (32 / QI - 1)) * other;
  const size_t park = PAIR ? 0 : 3 * (8 + C + V) * 128 * sizeof(double);
  const unsigned nb = nblk(warps * 32, 128);
  // one kernel per reconstruction scheme, as for the X1 faces
#define GRIM_STRIP_RS(RS)                                                                                  \
  do {                                                                                                     \
    if (dir == 1) k_face_flux_strip<C, V, QI, MINB, PAIR, 1, RS><<<nb, 128, park, s>>>(c, ps, geoF, geoC, flux); \
    else k_face_flux_strip<C, V, QI, MINB, PAIR, 2, RS><<<nb, 128, park, s>>>(c, ps, geoF, geoC, flux);        \
  } while (0)
  switch (c.reconstruction) {
    case GRIM_WENO5: GRIM_STRIP_RS(GRIM_WENO5); break;
    case GRIM_PPM: GRIM_STRIP_RS(GRIM_PPM); break;
    case GRIM_MP5: GRIM_STRIP_RS(GRIM_MP5); break;
    default: GRIM_STRIP_RS(GRIM_MINMOD); break;
  }
#undef GRIM_STRIP_RS
}
static int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}
template <int C, int V, int MINB, int RS, bool PAIR>
static void face_x1_tma_launch_rs(const DevCfg& c, const CUtensorMap* tmap, const double* geoF, double* flux,
                                  DevState* st, cudaStream_t s) {
  constexpr int DOF = 8 + C + V;
  const int nw = 4;
  const size_t smem = ((size_t)nw * 2 * DOF * kX1Box + 3 * DOF * 128) * sizeof(double) + 2 * nw * 8;
  // the attribute belongs to the function on each device that launches it
  static unsigned long long attrDevices = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attrDevices & (1ULL << dev))) {
    cudaFuncSetAttribute(k_face_flux_x1_tma<C, V, MINB, RS, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    attrDevices |= 1ULL << dev;
  }
  k_face_flux_x1_tma<C, V, MINB, RS, PAIR><<<sm_count() * MINB, 32 * nw, smem, s>>>(*tmap, c, geoF, flux, st);
}
// the reconstruction scheme becomes a compile-time constant of the TMA
// kernels: one scheme's code per kernel keeps the instruction footprint small
template <int C, int V, int MINB, bool PAIR = false>
static void face_x1_tma_launch(const DevCfg& c, const CUtensorMap* tmap, const double* geoF, double* flux,
                               DevState* st, cudaStream_t s) {
  switch (c.reconstruction) {
    case GRIM_WENO5: face_x1_tma_launch_rs<C, V, MINB, GRIM_WENO5, PAIR>(c, tmap, geoF, flux, st, s); break;
    case GRIM_PPM: face_x1_tma_launch_rs<C, V, MINB, GRIM_PPM, PAIR>(c, tmap, geoF, flux, st, s); break;
    case GRIM_MP5: face_x1_tma_launch_rs<C, V, MINB, GRIM_MP5, PAIR>(c, tmap, geoF, flux, st, s); break;
    default: face_x1_tma_launch_rs<C, V, MINB, GRIM_MINMOD, PAIR>(c, tmap, geoF, flux, st, s); break;
  }
}
template <int C, int V, int MINB, int RS, bool PAIR>
static void face_strip_tma_launch_rs(const DevCfg& c, int dir, const CUtensorMap* tmap, const double* geoF,
                                     const double* geoC, double* flux, DevState* st, cudaStream_t s) {
  constexpr int DOF = 8 + C + V;
  const int nw = 4;
  const size_t smem = ((size_t)nw * 2 * 4 * kStripRows * DOF + 3 * DOF * 128) * sizeof(double) + 2 * nw * 8;
  static unsigned long long attrDevices = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attrDevices & (1ULL << dev))) {
    cudaFuncSetAttribute(k_face_flux_strip_tma<C, V, MINB, 1, RS, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    cudaFuncSetAttribute(k_face_flux_strip_tma<C, V, MINB, 2, RS, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    attrDevices |= 1ULL << dev;
  }
  if (dir == 1)
    k_face_flux_strip_tma<C, V, MINB, 1, RS, PAIR>
        <<<sm_count() * MINB, 32 * nw, smem, s>>>(tmap[1], c, geoF, geoC, flux, st);
  else
    k_face_flux_strip_tma<C, V, MINB, 2, RS, PAIR>
        <<<sm_count() * MINB, 32 * nw, smem, s>>>(tmap[2], c, geoF, geoC, flux, st);
}
template <int C, int V, int MINB, bool PAIR = false>
static void face_strip_tma_launch(const DevCfg& c, int dir, const CUtensorMap* tmap, const double* geoF,
                                  const double* geoC, double* flux, DevState* st, cudaStream_t s) {
  switch (c.reconstruction) {
    case GRIM_WENO5:
      face_strip_tma_launch_rs<C, V, MINB, GRIM_WENO5, PAIR>(c, dir, tmap, geoF, geoC, flux, st, s);
      break;
    case GRIM_PPM: face_strip_tma_launch_rs<C, V, MINB, GRIM_PPM, PAIR>(c, dir, tmap, geoF, geoC, flux, st, s); break;
    case GRIM_MP5: face_strip_tma_launch_rs<C, V, MINB, GRIM_MP5, PAIR>(c, dir, tmap, geoF, geoC, flux, st, s); break;
    default:
      face_strip_tma_launch_rs<C, V, MINB, GRIM_MINMOD, PAIR>(c, dir, tmap, geoF, geoC, flux, st, s);
      break;
  }
}
template <int C, int V>
static void face_flux_t(const DevCfg& c, int dir, const double* ps, const double* geoF, const double* geoC,
                        double* flux, int variant, const CUtensorMap* tmap, DevState* st, cudaStream_t s) {
  if constexpr (C == 0 && V == 0) {
    if (dir == 0) {
      if ((variant == 2 || variant == 3 || variant == 5) && tmap && st) {
        if (variant == 5) face_x1_tma_launch<C, V, 3, true>(c, &tmap[0], geoF, flux, st, s);
        else if (variant == 3) face_x1_tma_launch<C, V, 4>(c, &tmap[0], geoF, flux, st, s);
        else face_x1_tma_launch<C, V, 3>(c, &tmap[0], geoF, flux, st, s);
      } else if (variant == 6) {
        face_x1_launch<C, V, 4, true>(c, ps, geoF, flux, s);
      } else if (variant == 4 || variant == 5) {
        face_x1_launch<C, V, 3, true>(c, ps, geoF, flux, s);
      } else if (variant == 1 || variant == 3) {
        face_x1_launch<C, V, 4>(c, ps, geoF, flux, s);
      } else {
        face_x1_launch<C, V, 3>(c, ps, geoF, flux, s);
      }
      return;
    }
    if (variant >= 8 && tmap && st) {
      if (variant == 11) face_strip_tma_launch<C, V, 4, true>(c, dir, tmap, geoF, geoC, flux, st, s);
      else if (variant == 10) face_strip_tma_launch<C, V, 3, true>(c, dir, tmap, geoF, geoC, flux, st, s);
      else if (variant == 9) face_strip_tma_launch<C, V, 4>(c, dir, tmap, geoF, geoC, flux, st, s);
      else face_strip_tma_launch<C, V, 3>(c, dir, tmap, geoF, geoC, flux, st, s);
      return;
    }
    switch (variant) {
      case 8: face_strip_launch<C, V, 4, 3>(c, dir, ps, geoF, geoC, flux, s); break;
      case 10: face_strip_launch<C, V, 4, 3, true>(c, dir, ps, geoF, geoC, flux, s); break;
      case 11: face_strip_launch<C, V, 4, 4, true>(c, dir, ps, geoF, geoC, flux, s); break;
      case 9: face_strip_launch<C, V, 4, 4>(c, dir, ps, geoF, geoC, flux, s); break;
      case 1: face_strip_launch<C, V, 4, 4>(c, dir, ps, geoF, geoC, flux, s); break;
      case 2: face_strip_launch<C, V, 2, 3>(c, dir, ps, geoF, geoC, flux, s); break;
      case 3: face_strip_launch<C, V, 2, 4>(c, dir, ps, geoF, geoC, flux, s); break;
      case 4: face_strip_launch<C, V, 8, 3>(c, dir, ps, geoF, geoC, flux, s); break;
      case 5: face_strip_launch<C, V, 8, 4>(c, dir, ps, geoF, geoC, flux, s); break;
      case 6: face_strip_launch<C, V, 8, 3, true>(c, dir, ps, geoF, geoC, flux, s); break;
      case 7: face_strip_launch<C, V, 4, 3, true>(c, dir, ps, geoF, geoC, flux, s); break;
      default: face_strip_launch<C, V, 4, 3>(c, dir, ps, geoF, geoC, flux, s); break;
    }
  } else {
    // EMHD elements need more registers: two resident blocks; variant 1
    // stages the stencils with TMA
    if (dir == 0) {
      if (variant == 1 && tmap && st) face_x1_tma_launch<C, V, 2>(c, &tmap[0], geoF, flux, st, s);
      else face_x1_launch<C, V, 2>(c, ps, geoF, flux, s);
    } else {
      if (variant == 1 && tmap && st) face_strip_tma_launch<C, V, 2>(c, dir, tmap, geoF, geoC, flux, st, s);
      else face_strip_launch<C, V, 4, 2>(c, dir, ps, geoF, geoC, flux, s);
    }
  }
}
void face_flux(const DevCfg& c, int dir, const double* ps, const double* geoF, const double* geoC, double* flux,
               int variant, const CUtensorMap* tmap, DevState* st, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, face_flux_t, c, dir, ps, geoF, geoC, flux, variant, tmap, st, s);
}
// X1: 0, 1 = register budget 3 / 4 blocks; 2, 3 = the same with TMA-staged
// rows (when the caller has a tensor map of the primitives); 4 = both face
// states evaluated side by side; 5 = TMA-staged rows with both states side
// by side, 3 blocks per SM; 6 = both states side by side, 4 blocks per SM.
// X2 / X3: 0-5 = lane split x register budget;
// 6, 7 = side by side with 8 / 4 i per warp; 8, 9 = TMA-staged chunks, 3 / 4
// blocks per SM; 10, 11 = TMA-staged chunks side by side, 3 / 4 blocks per
// SM.
// EMHD (10 dof), every direction: 0 = plain, 1 = TMA-staged, 2 blocks per SM.
// tmap points at the caller's three tensor maps (X1, X2, X3 box shapes) of
// the prim array, or is null (the TMA variants then run their plain
// counterparts).
int face_variants(const DevCfg& c, int dir) {
  (void)dir;
  if (c.conduction || c.viscosity) return 2;  // plain / TMA-staged, 2 blocks per SM
  return dir == 0 ? 7 : 12;
}
#endif  // !GRIM_SKIP_FACES

#if !defined(GRIM_ONLY_FACES)
template <int C, int V>
static void stage_epilogue_t(const DevCfg& c, int stage, const StageBufs& b, cudaStream_t s) {
  if (c.metric != GRIM_MINKOWSKI || C || V) {
    // centre half first: the flux half's induction reads its consOld
    k_stage_epilogue<C, V, 1><<<nblk(c.Zint, 128), 128, 0, s>>>(c, stage, b);
    k_stage_epilogue<C, V, 2><<<nblk(c.Zint, 128), 128, 0, s>>>(c, stage, b);
  } else {
    // no explicit sources: one kernel
    k_stage_epilogue<C, V, 0><<<nblk(c.Zint, 128), 128, 0, s>>>(c, stage, b);
  }
}
void stage_epilogue(const DevCfg& c, int stage, const StageBufs& b, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, stage_epilogue_t, c, stage, b, s);
}

template <int C, int V>
static void dt_speeds_t(const DevCfg& c, const double* p, const double* geoC, int mode, DevState* st,
                        cudaStream_t s) {
  k_dt_speeds<C, V><<<nblk(c.Z, 256), 256, 0, s>>>(c, p, geoC, mode, st);
}
void dt_speeds(const DevCfg& c, const double* p, const double* geoC, int mode, DevState* st, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, dt_speeds_t, c, p, geoC, mode, st, s);
}
void dt_update(DevState* st, double courant, double maxInc, cudaStream_t s) {
  k_dt_update<<<1, 32, 0, s>>>(st, courant, maxInc);
}
void advance_time(DevState* st, cudaStream_t s) { k_advance_time<<<1, 32, 0, s>>>(st); }

template <int C, int V>
static void newton_fd_init_t(const DevCfg& c, int stage, const StageBufs& b, cudaStream_t s) {
  k_newton_fd_init<C, V><<<nblk(c.Zint, 128), 128, 0, s>>>(c, stage, b);
}
void newton_fd_init(const DevCfg& c, int stage, const StageBufs& b, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, newton_fd_init_t, c, stage, b, s);
}
template <int C, int V>
static void newton_fd_iter_t(const DevCfg& c, int stage, int it, const StageBufs& b, cudaStream_t s) {
  k_newton_fd_iter<C, V><<<nblk(c.Zint, 128), 128, 0, s>>>(c, stage, it, b);
}
void newton_fd_iter(const DevCfg& c, int stage, int it, const StageBufs& b, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, newton_fd_iter_t, c, stage, it, b, s);
}

template <int C, int V>
static void newton_fast_t(const DevCfg& c, int stage, const StageBufs& b, int mode, const int* list,
                          long long nlist, cudaStream_t s) {
  if (nlist <= 0) return;
  if (mode == GRIM_NEWTON_MIXED32)
    k_newton_fast<C, V, float><<<nblk(nlist, 128), 128, 0, s>>>(c, stage, b, list, nlist);
  else
    k_newton_fast<C, V, double><<<nblk(nlist, 128), 128, 0, s>>>(c, stage, b, list, nlist);
}
void newton_fast(const DevCfg& c, int stage, const StageBufs& b, int mode, const int* list, long long nlist,
                 cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, newton_fast_t, c, stage, b, mode, list, nlist, s);
}

#ifdef GRIM_FAST_MATH
bool newton_defer(const DevCfg& c, int stage, const StageBufs& b, int mode, cudaStream_t s) {
  if (c.conduction || c.viscosity || mode != GRIM_NEWTON_MIXED32 || c.maxIter < 2 || c.Z > 0x7fffffffLL)
    return false;
  static int grid = 0;
  if (!grid) {
    int dev = 0, sms = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_newton_defer<float>, 32 * kDeferWarps, 0);
    grid = sms * (per > 0 ? per : 1);
  }
  if (c.Zint > 0) k_newton_defer<float><<<grid, 32 * kDeferWarps, 0, s>>>(c, stage, b, c.Zint);
  return true;
}
#endif

static int persistent_blocks() {
  static int nb = 0;
  if (!nb) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    nb = sms * 8;
  }
  return nb;
}
template <int C, int V>
static void newton_list_t(const DevCfg& c, int stage, const StageBufs& b, int mode, cudaStream_t s) {
  const int nb = persistent_blocks();
  cudaMemsetAsync(b.st->listCount, 0, sizeof(b.st->listCount), s);
  k_newton_list_init<C, V><<<nb, 128, 0, s>>>(c, stage, b);
  for (int it = 1; it <= c.maxIter; it++) {
    // the list this launch appends to starts empty
    cudaMemsetAsync(&b.st->listCount[it & 1], 0, sizeof(unsigned long long), s);
    if (mode == GRIM_NEWTON_MIXED32)
      k_newton_list_iter<C, V, float><<<nb, 128, 0, s>>>(c, stage, it, b);
    else
      k_newton_list_iter<C, V, double><<<nb, 128, 0, s>>>(c, stage, it, b);
  }
}
void newton_list(const DevCfg& c, int stage, const StageBufs& b, int mode, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, newton_list_t, c, stage, b, mode, s);
}

template <int C, int V>
static void batch_newton_t(const DevCfg& c0, const BatchEntry* tbl, int nprob, long long total, int maxIter, int stage,
                           int mode, BatchState* bs, cudaStream_t s) {
  (void)c0;
  const int nb = persistent_blocks();
  cudaMemsetAsync(bs->listCount, 0, sizeof(bs->listCount), s);
  k_batch_list_init<C, V><<<nb, 128, 0, s>>>(tbl, nprob, total, stage, bs);
  for (int it = 1; it <= maxIter; it++) {
    cudaMemsetAsync(&bs->listCount[it & 1], 0, sizeof(unsigned long long), s);
    if (mode == GRIM_NEWTON_MIXED32)
      k_batch_list_iter<C, V, float><<<nb, 128, 0, s>>>(tbl, nprob, stage, it, maxIter, bs);
    else
      k_batch_list_iter<C, V, double><<<nb, 128, 0, s>>>(tbl, nprob, stage, it, maxIter, bs);
  }
}
void batch_newton(const DevCfg& c0, const BatchEntry* tbl, int nprob, long long total, int maxIter, int stage,
                  int mode, BatchState* bs, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c0, batch_newton_t, c0, tbl, nprob, total, maxIter, stage, mode, bs, s);
}

template <int C, int V>
static void residual_t(const DevCfg& c, int stage, const StageBufs& b, const double* pg, double* out,
                       cudaStream_t s) {
  k_residual<C, V><<<nblk(c.Z, 128), 128, 0, s>>>(c, stage, b, pg, out);
}
void residual(const DevCfg& c, int stage, const StageBufs& b, const double* pg, double* out, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, residual_t, c, stage, b, pg, out, s);
}
template <int C, int V>
static void jacobian_t(const DevCfg& c, int stage, const StageBufs& b, const double* pg, double* jac, int tangent,
                       cudaStream_t s) {
  k_jacobian<C, V><<<nblk(c.Z, 128), 128, 0, s>>>(c, stage, b, pg, jac, tangent);
}
void jacobian(const DevCfg& c, int stage, const StageBufs& b, const double* pg, double* jac, int tangent,
              cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, jacobian_t, c, stage, b, pg, jac, tangent, s);
}
template <int C, int V>
static void conserved_t(const DevCfg& c, const double* p, const double* geoC, double* out, int fdir, int dir,
                        double* mn, double* mx, cudaStream_t s) {
  k_conserved<C, V><<<nblk(c.Z, 128), 128, 0, s>>>(c, p, geoC, out, fdir, dir, mn, mx);
}
void conserved(const DevCfg& c, const double* p, const double* geoC, double* out, int fdir, int dir, double* mn,
               double* mx, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, conserved_t, c, p, geoC, out, fdir, dir, mn, mx, s);
}
void reconstruct(const DevCfg& c, int dir, const double* p, double* pl, double* pr, cudaStream_t s) {
  k_reconstruct<<<nblk(c.Z, 128), 128, 0, s>>>(c, dir, p, pl, pr);
}
int batch_solve(int n, int batch, const double* A, const double* b, double* x, cudaStream_t s) {
  const unsigned g = nblk(batch, 128);
  switch (n) {
    case 1: k_batch_solve<1><<<g, 128, 0, s>>>(batch, A, b, x); return 0;
    case 2: k_batch_solve<2><<<g, 128, 0, s>>>(batch, A, b, x); return 0;
    case 3: k_batch_solve<3><<<g, 128, 0, s>>>(batch, A, b, x); return 0;
    case 4: k_batch_solve<4><<<g, 128, 0, s>>>(batch, A, b, x); return 0;
    case 5: k_batch_solve<5><<<g, 128, 0, s>>>(batch, A, b, x); return 0;
    case 6: k_batch_solve<6><<<g, 128, 0, s>>>(batch, A, b, x); return 0;
    case 7: k_batch_solve<7><<<g, 128, 0, s>>>(batch, A, b, x); return 0;
    case 8: k_batch_solve<8><<<g, 128, 0, s>>>(batch, A, b, x); return 0;
    default: return -1;
  }
}
static TorusCfg torus_cfg(const DevCfg& c) {
  TorusCfg t;
  t.MaxLorentzFactor = c.maxLF; t.RhoFloorAmpl = c.rhoFloorAmpl; t.UFloorAmpl = c.uFloorAmpl;
  t.RhoFloorSlope = c.rhoFloorSlope; t.UFloorSlope = c.uFloorSlope;
  t.BsqrOverRhoMax = c.bsqOverRhoMax; t.BsqrOverUMax = c.bsqOverUMax;
  return t;
}
template <int C, int V>
static void torus_floor_t(const DevCfg& c, double* p, const double* geoC, const unsigned long long* flag,
                          cudaStream_t s) {
  k_torus_floor<C, V><<<nblk(c.Z, 128), 128, 0, s>>>(c, torus_cfg(c), p, geoC, flag);
}
void torus_floor(const DevCfg& c, double* p, const double* geoC, const unsigned long long* flag, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, torus_floor_t, c, p, geoC, flag, s);
}
template <int C, int V>
static void stage_finish_t(const DevCfg& c, const double* src, double* dst, const double* geoC, bool floors,
                           bool post, const unsigned long long* nanFlag, int dtOn, DevState* st, cudaStream_t s) {
  const TorusCfg t = torus_cfg(c);
  const unsigned nb = (unsigned)nblk(c.Z, 128);
  if (floors && post)
    k_stage_finish<C, V, true, true><<<nb, 128, 0, s>>>(c, t, src, dst, geoC, nanFlag, dtOn, st);
  else if (floors)
    k_stage_finish<C, V, true, false><<<nb, 128, 0, s>>>(c, t, src, dst, geoC, nanFlag, dtOn, st);
  else if (post)
    k_stage_finish<C, V, false, true><<<nb, 128, 0, s>>>(c, t, src, dst, geoC, nanFlag, dtOn, st);
  else
    k_stage_finish<C, V, false, false><<<nb, 128, 0, s>>>(c, t, src, dst, geoC, nanFlag, dtOn, st);
}
void stage_finish(const DevCfg& c, const double* src, double* dst, const double* geoC, bool floors, bool post,
                  const unsigned long long* nanFlag, int dtOn, DevState* st, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, stage_finish_t, c, src, dst, geoC, floors, post, nanFlag, dtOn, st, s);
}
template <int C, int V>
static void torus_observe_t(const DevCfg& c, const double* p, const double* geoC, double volElem, double every,
                            DevState* st, double* partials, double* out, double* hist, int cap, cudaStream_t s) {
  k_torus_obs_partial<C, V><<<kObsBlocks, 128, 0, s>>>(c, p, geoC, volElem, every, st, partials);
  k_torus_obs_final<<<1, 32, 0, s>>>(partials, kObsBlocks, every, st, out, hist, cap);
}
void torus_observe(const DevCfg& c, const double* p, const double* geoC, double volElem, double every, DevState* st,
                   double* partials, double* out, double* hist, int cap, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, torus_observe_t, c, p, geoC, volElem, every, st, partials, out, hist, cap, s);
}
void torus_nan_flag(const DevCfg& c, const double* p, unsigned long long* flag, cudaStream_t s) {
  k_nan_flag<<<nblk(c.Zint, 256), 256, 0, s>>>(c, p, flag);
}
template <int C, int V>
static void torus_bcs_t(const DevCfg& c, double* p, const double* geoC, cudaStream_t s) {
  const long long cols = 2LL * c.ng * c.N2T * c.N3T;
  k_torus_inflow<C, V><<<nblk(cols, 128), 128, 0, s>>>(c, torus_cfg(c), p, geoC);
  if (c.dim >= 2) k_torus_poles<<<nblk(2LL * c.N1T * c.N3T, 128), 128, 0, s>>>(c, p, geoC);
}
void torus_bcs(const DevCfg& c, double* p, const double* geoC, cudaStream_t s) {
  GRIM_EMHD_DISPATCH(c, torus_bcs_t, c, p, geoC, s);
}
void emf(const DevCfg& c, const double* const* flux, double* out, cudaStream_t s) {
  k_emf<<<nblk(c.Z, 256), 256, 0, s>>>(c, flux[0], c.dim >= 2 ? flux[1] : flux[0], c.dim >= 3 ? flux[2] : flux[0],
                                         out);
}
void divb(const DevCfg& c, const double* p, const double* geoC, double* out, cudaStream_t s) {
  k_divb<<<nblk(c.Z, 256), 256, 0, s>>>(c, p, geoC, out);
}
void count_nonfinite(const DevCfg& c, const double* p, DevState* st, cudaStream_t s) {
  k_count_nonfinite<<<nblk(c.Zint, 256), 256, 0, s>>>(c, p, st);
}

#endif  // !GRIM_ONLY_FACES

}  // namespace GRIM_KNS
}  // namespace grim
