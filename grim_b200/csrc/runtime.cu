// runtime.cu -- host runtime behind the C ABI (include/grim_b200.h):
// handle lifecycle, device memory, the timeStep schedule on one CUDA stream,
// optional CUDA-graph replay of a whole step, statistics.
//
// The schedule of grim_time_step follows timeStepper::timeStep
// (src/timestepper/timestep.cpp:3-334):
//   dt update
//   half stage: ghost fill(primOld) -> [dt speeds for the next step]
//               -> [EMHD pre-pass] -> face fluxes per direction
//               -> stage epilogue (CT, divergence, induction, sources,
//                  consOld, Newton guess) -> Newton -> prim copied to primHalf
//   full stage: the same on primHalf -> prim copied to primOld -> ghost fill
//               -> time += dt -> [dt speeds of primOld for the next step]
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "launch.h"

namespace grim {
void launch_geometry(const DevCfg& c, const grim_config& cfg, int location, double* out, double* gamma,
                     cudaStream_t s);
}  // namespace grim

using namespace grim;

static thread_local std::string g_err;
static void set_err(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

#define CK(call)                                                                    \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      set_err("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return GRIM_ECUDA;                                                            \
    }                                                                               \
  } while (0)

struct grim_handle {
  grim_config cfg;
  DevCfg dc;
  int device = 0;
  cudaStream_t stream = nullptr;
  // state grids (dof x Z each)
  double *primOld = nullptr, *prim = nullptr, *primHalf = nullptr;
  // stage buffers
  double *consOld = nullptr, *divF = nullptr, *Sexp = nullptr, *R = nullptr, *l2 = nullptr, *uT = nullptr;
  double* flux[3] = {nullptr, nullptr, nullptr};
  int* list[2] = {nullptr, nullptr};  // compacted Newton worklists
  double* scratch = nullptr;  // test entry points: dof x Z inputs
  double* scratch2 = nullptr;
  // geometry: per location 39 x Z (MKS only), centre Christoffels 64 x Z
  double* geo[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double* gamma = nullptr;
  // torus observers: per-block partials (kObsBlocks x OBS_N), one result
  // (OBS_N) and the history ring (obsCap records of time + OBS_N values)
  double* obs = nullptr;
  int obsCap = 4096;
  DevState* st = nullptr;
  DevState* hst = nullptr;  // pinned mirror
  // mapped pinned word a kernel whose bounded copy wait gave up sets to 1
  // (DevState::hostError is its device alias); the next stepping or
  // synchronising call reports it once as GRIM_ETIMEOUT
  unsigned* hostError = nullptr;
  cudaEvent_t ev[8];
  bool graphOn = false;
  cudaGraphExec_t graph = nullptr;
  grim_stats stats;
  long long launchesPerStep = 0;
  size_t bytesZ = 0;
  int lastStage = GRIM_HALF_STEP;
  // the stage constants (consOld, divF, Sexp, the field guess) are those
  // grim_stage_setup formed, not yet replaced by a step or a stencil call
  bool stageReady = false;
  // per-kernel-group device timing (grim_profile_steps): event pairs
  // recorded around each launch on the handle's stream
  // TMA descriptors of the arrays the X1 face kernel reads (primOld,
  // primHalf, scratch) as (i, j, k, var); valid when haveTmap
  bool haveTmap = false;
  CUtensorMap tmap[3][3];  // [primOld, primHalf, scratch][box for X1, X2, X3 faces]
  bool tmapMissing[3] = {false, false, false};
  // face-kernel launch variants per direction, [exact unit, fast unit]
  int faceVariant[2][3] = {{0, 0, 0}, {0, 0, 0}};
  // dt held at its current value instead of computeDt (the adjoint's runs)
  bool fixedDt = false;
  // adjoint: checkpoints of primOld every adjEvery steps of the last
  // grim_adjoint_forward, segment states and the reverse sweep's buffers
  int adjSteps = 0, adjEvery = 0;
  double adjT0 = 0., adjDt = 0.;
  std::vector<double*> adjCkpt;
  std::vector<double*> adjSeg;  // 2 * every + 1 states: S[0..every], H[0..every-1]
  double* adjWork = nullptr;    // AdjointBufs storage
  // grim_time_steps_host: two staging buffers each way (dof x Z), an upload
  // and a download stream so both directions of PCIe and the step overlap
  double* ioIn[2] = {nullptr, nullptr};
  double* ioOut[2] = {nullptr, nullptr};
  cudaStream_t ioUp = nullptr, ioDown = nullptr;
  cudaEvent_t ioEv[8];  // [0,2) upload done, [2,4) input consumed, [4,6) output staged, [6,8) download done
  bool ioReady = false;
  bool profOn = false;
  std::vector<cudaEvent_t> profEv;
  std::vector<int> profGroup;
  size_t profUsed = 0;
};

// brackets one launch (or a run of launches of the same group) with events
struct ProfScope {
  grim_handle* h;
  size_t slot;
  ProfScope(grim_handle* hh, int group) : h(hh), slot(SIZE_MAX) {
    if (!h->profOn) return;
    if (h->profUsed * 2 + 2 > h->profEv.size()) {
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      h->profEv.push_back(a);
      h->profEv.push_back(b);
      h->profGroup.push_back(0);
    }
    slot = h->profUsed++;
    h->profGroup[slot] = group;
    cudaEventRecord(h->profEv[2 * slot], h->stream);
  }
  ~ProfScope() {
    if (slot != SIZE_MAX) cudaEventRecord(h->profEv[2 * slot + 1], h->stream);
  }
};
#define PROF(group) ProfScope prof_scope_(h, group)

static void free_all(grim_handle* h) {
  double** bufs[] = {&h->primOld, &h->prim, &h->primHalf, &h->consOld, &h->divF, &h->Sexp, &h->R,
                     &h->l2, &h->uT, &h->flux[0], &h->flux[1], &h->flux[2], &h->scratch, &h->scratch2,
                     &h->geo[0], &h->geo[1], &h->geo[2], &h->geo[3], &h->geo[4], &h->gamma, &h->obs};
  for (double** b : bufs)
    if (*b) { cudaFree(*b); *b = nullptr; }
  if (h->st) { cudaFree(h->st); h->st = nullptr; }
  if (h->hst) { cudaFreeHost(h->hst); h->hst = nullptr; }
  if (h->hostError) { cudaFreeHost(h->hostError); h->hostError = nullptr; }
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  for (int l = 0; l < 2; l++)
    if (h->list[l]) { cudaFree(h->list[l]); h->list[l] = nullptr; }
  for (double* p : h->adjCkpt) cudaFree(p);
  for (double* p : h->adjSeg) cudaFree(p);
  h->adjCkpt.clear();
  h->adjSeg.clear();
  if (h->adjWork) { cudaFree(h->adjWork); h->adjWork = nullptr; }
  for (cudaEvent_t e : h->profEv) cudaEventDestroy(e);
  h->profEv.clear();
  h->profGroup.clear();
  for (int i = 0; i < 2; i++) {
    if (h->ioIn[i]) { cudaFree(h->ioIn[i]); h->ioIn[i] = nullptr; }
    if (h->ioOut[i]) { cudaFree(h->ioOut[i]); h->ioOut[i] = nullptr; }
  }
  if (h->ioReady) {
    for (int i = 0; i < 8; i++) cudaEventDestroy(h->ioEv[i]);
    cudaStreamDestroy(h->ioUp);
    cudaStreamDestroy(h->ioDown);
    h->ioReady = false;
  }
}

static int make_devcfg(const grim_config& c, DevCfg& d) {
  if (c.dim < 1 || c.dim > 3) { set_err("dim must be 1, 2 or 3"); return GRIM_EINVAL; }
  if (c.numGhost != 3) { set_err("numGhost must be 3"); return GRIM_EINVAL; }
  if (c.N1 < 4 || (c.dim >= 2 && c.N2 < 4) || (c.dim >= 3 && c.N3 < 4)) {
    set_err("each active dimension needs at least 4 zones"); return GRIM_EINVAL;
  }
  if (c.reconstruction < 0 || c.reconstruction > 3) { set_err("bad reconstruction"); return GRIM_EINVAL; }
  if (c.maxNonLinearIter < 1 || c.maxNonLinearIter > 15) { set_err("maxNonLinearIter must be 1..15"); return GRIM_EINVAL; }
  if (c.maxLineSearchIters < 1 || c.maxLineSearchIters > 32) { set_err("maxLineSearchIters must be 1..32"); return GRIM_EINVAL; }
  if (c.metric != GRIM_MINKOWSKI && c.metric != GRIM_MODIFIED_KERR_SCHILD) { set_err("bad metric %d", c.metric); return GRIM_EINVAL; }
  if (c.riemannSolver != GRIM_HLL && c.riemannSolver != GRIM_LOCAL_LAX_FRIEDRICH) {
    set_err("bad riemannSolver %d", c.riemannSolver); return GRIM_EINVAL;
  }
  if (c.closure < GRIM_CLOSURE_CONST_TAU || c.closure > GRIM_CLOSURE_TAU_PROFILE) { set_err("bad closure %d", c.closure); return GRIM_EINVAL; }
  if (c.problem != GRIM_PROBLEM_NONE && c.problem != GRIM_PROBLEM_TORUS) { set_err("bad problem %d", c.problem); return GRIM_EINVAL; }
  if (c.newtonMode < GRIM_NEWTON_PARITY_FD64 || c.newtonMode > GRIM_NEWTON_FD64_FAST) {
    set_err("bad newtonMode %d", c.newtonMode); return GRIM_EINVAL;
  }
  if (c.perZoneConvergence < 0 || c.perZoneConvergence > 3) {
    set_err("perZoneConvergence must be 0..3"); return GRIM_EINVAL;
  }
  // coordinatesGrid (grid.cpp:142-146) divides each active extent by N
  if (!(c.X1End > c.X1Start) || (c.dim >= 2 && !(c.X2End > c.X2Start)) || (c.dim >= 3 && !(c.X3End > c.X3Start))) {
    set_err("each active direction needs XEnd > XStart"); return GRIM_EINVAL;
  }
  memset(&d, 0, sizeof(d));
  d.dim = c.dim; d.ng = c.numGhost;
  d.N1 = c.N1; d.N2 = c.dim >= 2 ? c.N2 : 1; d.N3 = c.dim >= 3 ? c.N3 : 1;
  d.g1 = d.ng; d.g2 = c.dim >= 2 ? d.ng : 0; d.g3 = c.dim >= 3 ? d.ng : 0;
  d.N1T = d.N1 + 2 * d.g1; d.N2T = d.N2 + 2 * d.g2; d.N3T = d.N3 + 2 * d.g3;
  // face rows: the interior and one row beyond it on each side (the corner
  // EMFs of the interior's edges read one row of fluxes outside it)
  d.fj0 = std::max(d.g2 - 1, 0);
  d.nfj = std::min(d.N2 + d.g2, d.N2T - 1) - d.fj0 + 1;
  d.fk0 = std::max(d.g3 - 1, 0);
  d.nfk = std::min(d.N3 + d.g3, d.N3T - 1) - d.fk0 + 1;
  d.Z = (long long)d.N1T * d.N2T * d.N3T;
  d.Zint = (long long)d.N1 * d.N2 * d.N3;
  d.GZ = (long long)d.N1T * d.N2T;
  if (d.Z >= (1LL << 31)) {  // 32-bit zone indices in the kernels
    set_err("grid of %lld zones with ghosts: at most 2^31 - 1", d.Z); return GRIM_EINVAL;
  }
  d.conduction = c.conduction ? 1 : 0; d.viscosity = c.viscosity ? 1 : 0;
  d.nf = 5 + d.conduction + d.viscosity; d.dof = d.nf + 3;
  d.Q = 5; d.DP = 5 + d.conduction; d.B1 = d.nf;
  d.hoCond = c.highOrderTermsConduction; d.hoVisc = c.highOrderTermsViscosity;
  d.metric = c.metric; d.reconstruction = c.reconstruction; d.riemann = c.riemannSolver;
  d.closure = c.closure; d.problem = c.problem;
  d.maxIter = c.maxNonLinearIter; d.maxLS = c.maxLineSearchIters;
  d.bc[0] = c.boundaryLeft; d.bc[1] = c.boundaryRight; d.bc[2] = c.boundaryBottom; d.bc[3] = c.boundaryTop;
  d.bc[4] = c.boundaryBack; d.bc[5] = c.boundaryFront;
  for (int q = 0; q < 6; q++)
    if (d.bc[q] < GRIM_PERIODIC || d.bc[q] > GRIM_EXCHANGE) { set_err("bad boundary condition %d", d.bc[q]); return GRIM_EINVAL; }
  // boundary.cpp fills OUTFLOW and MIRROR sides only; a DIRICHLET side is
  // the problem's own boundary hook, which none of the supported problems has
  for (int q = 0; q < 6; q++)
    if (d.bc[q] == GRIM_DIRICHLET) {
      set_err("GRIM_DIRICHLET sides are a problem hook's; give the side GRIM_EXCHANGE and set its ghosts instead");
      return GRIM_ENOTSUP;
    }
  if (c.N3Global < 0 || (c.N3Global > 0 && (c.dim < 3 || c.N3Global < c.N3))) {
    set_err("N3Global: a slab of a 3D grid with N3 <= N3Global"); return GRIM_EINVAL;
  }
  // coordinatesGrid (grid.cpp:142-146): dX from the constructor's N
  d.dX[0] = (c.X1End - c.X1Start) / c.N1;
  d.dX[1] = (c.X2End - c.X2Start) / c.N2;
  // a slab: the global extent over the global plane count
  d.dX[2] = (c.X3End - c.X3Start) / (c.N3Global > 0 ? c.N3Global : c.N3);
  for (int i = 0; i < 3; i++) d.invdX[i] = 1. / d.dX[i];
  d.X1Start = c.X1Start; d.X2Start = c.X2Start; d.X3Start = c.X3Start; d.X2End = c.X2End;
  d.Gam = c.adiabaticIndex;
  d.rhoFloor = c.rhoFloorInFluidElement; d.uFloor = c.uFloorInFluidElement;
  d.bSqrFloor = c.bSqrFloorInFluidElement; d.TFloor = c.temperatureFloorInFluidElement;
  d.CondAlpha = c.ConductionAlpha; d.ViscAlpha = c.ViscosityAlpha;
  d.CondClosure = c.ConductionClosureFactor; d.ViscClosure = c.ViscosityClosureFactor;
  d.theta = c.slopeLimTheta;
  d.atol = c.nonlinearsolve_atol; d.rtol = c.nonlinearsolve_rtol;
  if (!(c.nonlinearsolve_ulps >= 0.)) { set_err("nonlinearsolve_ulps must be >= 0"); return GRIM_EINVAL; }
  d.tolUlps = c.nonlinearsolve_ulps;
  d.jacEps = c.JacobianAssembleEpsilon; d.lsFloor = c.linesearchfloor;
  d.tau0 = c.closureTau0; d.tau1 = c.closureTau1;
  d.maxLF = c.MaxLorentzFactor; d.rhoFloorAmpl = c.RhoFloorAmpl; d.uFloorAmpl = c.UFloorAmpl;
  d.rhoFloorSlope = c.RhoFloorSlope; d.uFloorSlope = c.UFloorSlope;
  d.bsqOverRhoMax = c.BsqrOverRhoMax; d.bsqOverUMax = c.BsqrOverUMax;
  d.dbgSkipCopies = 0;
  if ((c.problem == GRIM_PROBLEM_TORUS || c.closure == GRIM_CLOSURE_TORUS) && c.metric == GRIM_MINKOWSKI) {
    set_err("the torus problem and closure need the MKS metric"); return GRIM_EINVAL;
  }
  return GRIM_OK;
}

static bool use_exact(const grim_handle* h) { return h->cfg.newtonMode == GRIM_NEWTON_PARITY_FD64; }
// the reference's FD-Jacobian Newton with global break, in either unit
static bool is_fd(const grim_handle* h) {
  return h->cfg.newtonMode == GRIM_NEWTON_PARITY_FD64 || h->cfg.newtonMode == GRIM_NEWTON_FD64_FAST;
}

// the three tensor maps (X1, X2, X3 box shapes) of a prim array of this
// handle, or null when the array has none or direction dir's box does not fit
static const CUtensorMap* tmap_for(const grim_handle* h, const double* p, int dir) {
  if (!h->haveTmap || h->tmapMissing[dir]) return nullptr;
  if (p == h->primOld) return h->tmap[0];
  if (p == h->primHalf) return h->tmap[1];
  if (p == h->scratch) return h->tmap[2];
  return nullptr;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependency on the driver library)
static bool encode_prim_tmap(const DevCfg& c, double* base, int dir, CUtensorMap* out) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return false;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  // rows of N1T doubles must be 16-byte strided; the boxes must fit: X1
  // faces stage 40 zones along i, X2 / X3 faces 4 i x 12 zones along j / k
  if (c.N1T % 2 != 0 || c.N1T < 40 || c.dof > 256) return false;
  if (dir == 1 && c.N2T < 12) return false;
  if (dir == 2 && c.N3T < 12) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)c.N1T, (cuuint64_t)c.N2T, (cuuint64_t)c.N3T, (cuuint64_t)c.dof};
  const cuuint64_t strides[3] = {(cuuint64_t)c.N1T * 8, (cuuint64_t)c.N1T * c.N2T * 8, (cuuint64_t)c.Z * 8};
  const cuuint32_t box[4] = {dir == 0 ? 40u : 4u, dir == 1 ? 12u : 1u, dir == 2 ? 12u : 1u, (cuuint32_t)c.dof};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = encode(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base, dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

static StageBufs stage_bufs(grim_handle* h, int stage, bool guessOld = false) {
  StageBufs b;
  memset(&b, 0, sizeof(b));
  b.guessOld = guessOld ? 1 : 0;
  b.ps = (stage == GRIM_HALF_STEP) ? h->primOld : h->primHalf;
  b.pold = h->primOld;
  b.prim = h->prim;
  const bool mink = h->cfg.metric == GRIM_MINKOWSKI;
  b.geoC = mink ? nullptr : h->geo[GRIM_CENTER];
  b.gamma = mink ? nullptr : h->gamma;
  b.geoF[0] = mink ? nullptr : h->geo[GRIM_LEFT];
  b.geoF[1] = mink ? nullptr : h->geo[GRIM_BOTTOM];
  b.geoF[2] = b.geoC;
  for (int d = 0; d < 3; d++) b.flux[d] = h->flux[d];
  b.uT = h->uT;
  b.consOld = h->consOld;
  b.divF = h->divF;
  b.Sexp = h->Sexp;
  b.R = h->R;
  b.l2 = h->l2;
  b.st = h->st;
  b.list[0] = h->list[0];
  b.list[1] = h->list[1];
  return b;
}

// ---------------------------------------------------------------------------
// the step schedule (all asynchronous on h->stream)
// ---------------------------------------------------------------------------
#define KNS_CALL(h, fn, ...)                                           \
  do {                                                                 \
    if (use_exact(h)) grim::exact::fn(__VA_ARGS__);                    \
    else grim::fast::fn(__VA_ARGS__);                                  \
  } while (0)

#define KNS_CALL_RET(h, out, fn, ...)                                  \
  do {                                                                 \
    if (use_exact(h)) out = grim::exact::fn(__VA_ARGS__);              \
    else out = grim::fast::fn(__VA_ARGS__);                            \
  } while (0)

static long long g_launch_counter = 0;

// a step's per-zone fast Newton takes the half stage's guess straight from
// primOld; the stand-alone stage pieces (grim_stage_setup and
// grim_newton_solve) and the batch keep it in prim
static bool step_guess_old(const grim_handle* h) {
  return !is_fd(h) && h->cfg.perZoneConvergence != 2;
}
static void enqueue_stencil(grim_handle* h, int stage, bool guessOld = false) {
  const DevCfg& c = h->dc;
  cudaStream_t s = h->stream;
  StageBufs b = stage_bufs(h, stage, guessOld);
  if (c.conduction || c.viscosity) {
    PROF(GRIM_PROF_EMHD_PREPASS);
    KNS_CALL(h, emhd_prepass, c, b.ps, b.geoC, h->uT, s);
    g_launch_counter++;
  }
  for (int d = 0; d < c.dim; d++) {
    PROF(GRIM_PROF_FACES_X1 + d);
    KNS_CALL(h, face_flux, c, d, b.ps, b.geoF[d], b.geoC, h->flux[d], h->faceVariant[use_exact(h) ? 0 : 1][d],
             tmap_for(h, b.ps, d), h->st, s);
    g_launch_counter++;
  }
  PROF(GRIM_PROF_EPILOGUE);
  KNS_CALL(h, stage_epilogue, c, stage, b, s);
  g_launch_counter += (c.metric != GRIM_MINKOWSKI || c.conduction || c.viscosity) ? 2 : 1;
}

// the torus step's per-zone fast Newton counts, as it writes the full
// stage's result, the zones fullStepDiagnostics would find a NaN in (so the
// count needs no pass of its own); the other Newton forms leave the count
// to k_nan_flag
static bool newton_counts_nan(const grim_handle* h) {
  return h->cfg.problem == GRIM_PROBLEM_TORUS && !is_fd(h) && h->cfg.perZoneConvergence != 2;
}

// returns whether the launch counts the NaN zones (countNan asked for it
// and the Newton form does it)
static bool enqueue_newton(grim_handle* h, int stage, bool guessOld = false, bool countNan = false) {
  const DevCfg& c = h->dc;
  cudaStream_t s = h->stream;
  StageBufs b = stage_bufs(h, stage, guessOld);
  PROF(GRIM_PROF_NEWTON);
  countNan = countNan && newton_counts_nan(h);
  if (countNan) {
    cudaMemsetAsync(&h->st->nanFlag, 0, sizeof(unsigned long long), s);
    b.nanCount = &h->st->nanFlag;
  }
  if (h->cfg.newtonMode == GRIM_NEWTON_PARITY_FD64) {
    grim::exact::newton_fd_init(c, stage, b, s);
    g_launch_counter++;
    for (int it = 0; it < c.maxIter; it++) {
      grim::exact::newton_fd_iter(c, stage, it, b, s);
      g_launch_counter++;
    }
  } else if (h->cfg.newtonMode == GRIM_NEWTON_FD64_FAST) {
    grim::fast::newton_fd_init(c, stage, b, s);
    g_launch_counter++;
    for (int it = 0; it < c.maxIter; it++) {
      grim::fast::newton_fd_iter(c, stage, it, b, s);
      g_launch_counter++;
    }
  } else if (h->cfg.perZoneConvergence == 2) {
    grim::fast::newton_list(c, stage, b, h->cfg.newtonMode, s);
    g_launch_counter += 1 + c.maxIter;
  } else if (h->cfg.perZoneConvergence == 3 && grim::fast::newton_defer(c, stage, b, h->cfg.newtonMode, s)) {
    g_launch_counter++;
  } else {
    grim::fast::newton_fast(c, stage, b, h->cfg.newtonMode, nullptr, c.Zint, s);
    g_launch_counter++;
  }
  return countNan;
}

static void enqueue_dt_speeds(grim_handle* h, const double* p, int mode) {
  const DevCfg& c = h->dc;
  PROF(GRIM_PROF_DT);
  cudaMemsetAsync(&h->st->maxInvDt, 0, sizeof(double), h->stream);
  const bool mink = h->cfg.metric == GRIM_MINKOWSKI;
  KNS_CALL(h, dt_speeds, c, p, mink ? nullptr : h->geo[GRIM_CENTER], mode, h->st, h->stream);
  g_launch_counter++;
}

// torus: setProblemSpecificBCs (inflow check + pole fix) after the
// stage-start boundary fill (timestep.cpp:17-22, :186-191)
static void enqueue_problem_bcs(grim_handle* h, double* p) {
  if (h->cfg.problem != GRIM_PROBLEM_TORUS) return;
  PROF(GRIM_PROF_BOUNDARY);
  KNS_CALL(h, torus_bcs, h->dc, p, h->geo[GRIM_CENTER], h->stream);
  g_launch_counter += 2;
}
// fullStepDiagnostics: NaN reset + floors on primOld (torus/problem.cpp:719-746)
static void enqueue_full_diagnostics(grim_handle* h) {
  if (h->cfg.problem != GRIM_PROBLEM_TORUS) return;
  PROF(GRIM_PROF_DIAGNOSTICS);
  cudaMemsetAsync(&h->st->nanFlag, 0, sizeof(unsigned long long), h->stream);
  KNS_CALL(h, torus_nan_flag, h->dc, h->primOld, &h->st->nanFlag, h->stream);
  KNS_CALL(h, torus_floor, h->dc, h->primOld, h->geo[GRIM_CENTER], &h->st->nanFlag, h->stream);
  g_launch_counter += 2;
}

// The step in segments around the two stencil + Newton pairs, so that a
// batch of problems can interleave its problems around one shared Newton
// launch: pre_half -> stencil(half) -> Newton(half) -> mid -> stencil(full)
// -> Newton(full) -> post.
static void enqueue_pre_half(grim_handle* h, bool timed) {
  const DevCfg& c = h->dc;
  cudaStream_t s = h->stream;
  if (timed) cudaEventRecord(h->ev[0], s);
  // computeDt (timestep.cpp:8): dt from the last elemOld state
  if (!h->fixedDt) {
    PROF(GRIM_PROF_DT);
    KNS_CALL(h, dt_update, h->st, h->cfg.CourantFactor, h->cfg.maxDtIncrement, s);
    g_launch_counter++;
  }
  cudaMemsetAsync(h->st->count, 0, sizeof(h->st->count), s);
  cudaMemsetAsync(h->st->itersDone, 0, sizeof(h->st->itersDone), s);
  cudaMemsetAsync(h->st->finalUnconv, 0, sizeof(h->st->finalUnconv), s);
  cudaMemsetAsync(h->st->itHist, 0, sizeof(h->st->itHist), s);
  cudaMemsetAsync(&h->st->nonFinite, 0, sizeof(unsigned long long), s);
  // ---- half stage
  {
    PROF(GRIM_PROF_BOUNDARY);
    KNS_CALL(h, ghost_fill, c, h->primOld, c.dof, s);
    g_launch_counter++;
  }
  enqueue_problem_bcs(h, h->primOld);
  if (!h->cfg.elemOldFromFullStep) enqueue_dt_speeds(h, h->primOld, 0);
  if (timed) cudaEventRecord(h->ev[1], s);
}

// primHalfStep = prim, communicate, halfStepDiagnostics as one pass
static void enqueue_mid_finish(grim_handle* h) {
  const DevCfg& c = h->dc;
  PROF(GRIM_PROF_COPY);
  const bool torus = h->cfg.problem == GRIM_PROBLEM_TORUS;
  const double* geoC = h->cfg.metric == GRIM_MINKOWSKI ? nullptr : h->geo[GRIM_CENTER];
  KNS_CALL(h, stage_finish, c, h->prim, h->primHalf, geoC, torus, false, nullptr, 0, h->st, h->stream);
  g_launch_counter++;
}
// the full stage's boundaries on primHalfStep
static void enqueue_mid_fill(grim_handle* h) {
  {
    PROF(GRIM_PROF_BOUNDARY);
    KNS_CALL(h, ghost_fill, h->dc, h->primHalf, h->dc.dof, h->stream);
    g_launch_counter++;
  }
  enqueue_problem_bcs(h, h->primHalf);
}
static void enqueue_mid(grim_handle* h) {
  enqueue_mid_finish(h);
  enqueue_mid_fill(h);
}

// the torus observers of primOld (ObserversTorus.hpp): into out (device,
// OBS_N values) and / or, with toHistory, the handle's record ring
static void enqueue_observers(grim_handle* h, double every, double* out, bool toHistory) {
  const DevCfg& c = h->dc;
  double volElem = c.dX[0];
  if (c.dim > 1) volElem *= c.dX[1];
  if (c.dim > 2) volElem *= c.dX[2];
  const double* geoC = h->cfg.metric == GRIM_MINKOWSKI ? nullptr : h->geo[GRIM_CENTER];
  double* hist = h->obs + (size_t)kObsBlocks * OBS_N + OBS_N;
  grim::exact::torus_observe(c, h->primOld, geoC, volElem, every, h->st, h->obs, out,
                             toHistory ? hist : nullptr, h->obsCap, h->stream);
}

// primOld = prim, communicate, fullStepDiagnostics (torus: NaN reset and
// floors), the next computeDt's speeds when the element is re-set from the
// full step (linear_modes/problem.cpp:287) and the non-finite count, as one
// pass after the NaN count
// time advance and the NaN count of fullStepDiagnostics (on the Newton
// result, whose interior the finish copies unchanged), unless the full
// stage's Newton counted it
static void enqueue_post_count(grim_handle* h, bool nanCounted) {
  const DevCfg& c = h->dc;
  cudaStream_t s = h->stream;
  {
    PROF(GRIM_PROF_DT);
    grim::exact::advance_time(h->st, s);
    g_launch_counter++;
  }
  if (h->cfg.problem == GRIM_PROBLEM_TORUS && !nanCounted) {
    PROF(GRIM_PROF_DIAGNOSTICS);
    cudaMemsetAsync(&h->st->nanFlag, 0, sizeof(unsigned long long), s);
    KNS_CALL(h, torus_nan_flag, c, h->prim, &h->st->nanFlag, s);
    g_launch_counter++;
  }
}
static void enqueue_post_finish(grim_handle* h, bool timed) {
  const DevCfg& c = h->dc;
  cudaStream_t s = h->stream;
  const bool torus = h->cfg.problem == GRIM_PROBLEM_TORUS;
  {
    PROF(GRIM_PROF_COPY);
    const int dtOn = h->cfg.elemOldFromFullStep ? 1 : 0;
    if (dtOn) cudaMemsetAsync(&h->st->maxInvDt, 0, sizeof(double), s);
    const double* geoC = h->cfg.metric == GRIM_MINKOWSKI ? nullptr : h->geo[GRIM_CENTER];
    KNS_CALL(h, stage_finish, c, h->prim, h->primOld, geoC, torus, true, &h->st->nanFlag, dtOn, h->st, s);
    g_launch_counter++;
  }
  if (h->cfg.ObserveEveryDt > 0.) {
    // on-the-fly observers of fullStepDiagnostics (problem.cpp:754-778): the
    // kernels read time and dt on the device and do nothing between records
    PROF(GRIM_PROF_DIAGNOSTICS);
    enqueue_observers(h, h->cfg.ObserveEveryDt, nullptr, true);
    g_launch_counter += 2;
  }
  if (timed) cudaEventRecord(h->ev[7], s);
}
static void enqueue_post(grim_handle* h, bool timed, bool nanCounted = false) {
  enqueue_post_count(h, nanCounted);
  enqueue_post_finish(h, timed);
}

// the step in the four segments of a slab-decomposed run (grim_step_segment)
static void enqueue_segment(grim_handle* h, int seg) {
  switch (seg) {
    case GRIM_SEG_PRE: enqueue_pre_half(h, false); break;
    case GRIM_SEG_HALF:
      enqueue_stencil(h, GRIM_HALF_STEP, step_guess_old(h));
      enqueue_newton(h, GRIM_HALF_STEP, step_guess_old(h));
      enqueue_mid_finish(h);
      break;
    case GRIM_SEG_FULL:
      enqueue_mid_fill(h);
      enqueue_stencil(h, GRIM_FULL_STEP);
      enqueue_post_count(h, enqueue_newton(h, GRIM_FULL_STEP, false, true));
      break;
    default: enqueue_post_finish(h, false); break;
  }
}

static void enqueue_step(grim_handle* h, bool timed) {
  cudaStream_t s = h->stream;
  enqueue_pre_half(h, timed);
  enqueue_stencil(h, GRIM_HALF_STEP, step_guess_old(h));
  if (timed) cudaEventRecord(h->ev[2], s);
  enqueue_newton(h, GRIM_HALF_STEP, step_guess_old(h));
  if (timed) cudaEventRecord(h->ev[3], s);
  enqueue_mid(h);
  if (timed) cudaEventRecord(h->ev[4], s);
  enqueue_stencil(h, GRIM_FULL_STEP);
  if (timed) cudaEventRecord(h->ev[5], s);
  const bool nanCounted = enqueue_newton(h, GRIM_FULL_STEP, false, true);
  if (timed) cudaEventRecord(h->ev[6], s);
  enqueue_post(h, timed, nanCounted);
}

// the memory kind of a caller's pointer: GRIM_HOST or GRIM_DEVICE, nothing else
static bool mem_kind_ok(int memKind) {
  if (memKind == GRIM_HOST || memKind == GRIM_DEVICE) return true;
  set_err("memKind %d: GRIM_HOST or GRIM_DEVICE", memKind);
  return false;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* grim_version(void) { return "grim_b200 0.1 (sm_100a)"; }
const char* grim_last_error(void) { return g_err.c_str(); }

int grim_create(const grim_config* cfg, int device, grim_handle** out) {
  if (!cfg || !out) { set_err("null argument"); return GRIM_EINVAL; }
  *out = nullptr;
  grim_handle* h = new grim_handle();
  h->cfg = *cfg;
  int rc = make_devcfg(*cfg, h->dc);
  if (rc) { delete h; return rc; }
  h->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { set_err("cudaSetDevice(%d): %s", device, cudaGetErrorString(e)); delete h; return GRIM_ECUDA; }
  const DevCfg& c = h->dc;
  const size_t Zb = (size_t)c.Z * sizeof(double);
  h->bytesZ = Zb;
  auto alloc = [&](double** p, size_t words) -> bool {
    if (cudaMalloc(p, words * Zb) != cudaSuccess) return false;
    return cudaMemset(*p, 0, words * Zb) == cudaSuccess;
  };
  bool ok = alloc(&h->primOld, c.dof) && alloc(&h->prim, c.dof) && alloc(&h->primHalf, c.dof) &&
            alloc(&h->consOld, c.dof) && alloc(&h->divF, c.dof) && alloc(&h->Sexp, c.nf) && alloc(&h->R, c.nf) &&
            alloc(&h->l2, 2) && alloc(&h->scratch, c.dof) && alloc(&h->scratch2, (size_t)c.dof * 3);
  for (int d = 0; ok && d < c.dim; d++) ok = alloc(&h->flux[d], c.dof);
  if (ok && (c.conduction || c.viscosity)) ok = alloc(&h->uT, 5);
  if (ok && cfg->metric != GRIM_MINKOWSKI) {
    // one (i, j) plane per word (the metric does not depend on X3)
    auto allocPlane = [&](double** p, size_t words) -> bool {
      const size_t b = words * (size_t)c.GZ * sizeof(double);
      if (cudaMalloc(p, b) != cudaSuccess) return false;
      return cudaMemset(*p, 0, b) == cudaSuccess;
    };
    for (int l = 0; ok && l < 5; l++) ok = allocPlane(&h->geo[l], 39);
    if (ok) ok = allocPlane(&h->gamma, 64);
  }
  for (int l = 0; ok && l < 2; l++) ok = cudaMalloc(&h->list[l], (size_t)c.Zint * sizeof(int)) == cudaSuccess;
  if (ok) {
    const size_t words = (size_t)kObsBlocks * OBS_N + OBS_N + (size_t)h->obsCap * (OBS_N + 1);
    ok = cudaMalloc(&h->obs, words * sizeof(double)) == cudaSuccess &&
         cudaMemset(h->obs, 0, words * sizeof(double)) == cudaSuccess;
  }
  if (ok) ok = cudaMalloc(&h->st, sizeof(DevState)) == cudaSuccess;
  if (ok) ok = cudaMallocHost(&h->hst, sizeof(DevState)) == cudaSuccess;
  if (ok) ok = cudaHostAlloc(&h->hostError, sizeof(unsigned), cudaHostAllocMapped) == cudaSuccess;
  if (!ok) {
    set_err("device allocation failed (%zu MB per grid variable)", Zb >> 20);
    free_all(h); delete h; return GRIM_ENOMEM;
  }
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_err("stream creation failed"); free_all(h); delete h; return GRIM_ECUDA;
  }
  for (int i = 0; i < 8; i++) cudaEventCreate(&h->ev[i]);
  {
    // X1 maps are required; X2 / X3 maps are built when the grid has room
    // for their boxes (a missing one leaves its direction on the plain kernel)
    double* arrays[3] = {h->primOld, h->primHalf, h->scratch};
    bool ok = true;
    for (int a = 0; a < 3 && ok; a++) {
      ok = encode_prim_tmap(c, arrays[a], 0, &h->tmap[a][0]);
      for (int d = 1; ok && d < 3; d++)
        if (d < c.dim && !encode_prim_tmap(c, arrays[a], d, &h->tmap[a][d])) h->tmapMissing[d] = true;
    }
    h->haveTmap = ok;
  }
  // geometry (geometry.cpp ctor at LEFT/RIGHT/BOTTOM/TOP/CENTER, timestepper.cpp:236-283)
  if (cfg->metric != GRIM_MINKOWSKI) {
    for (int l = 0; l < 5; l++)
      launch_geometry(c, *cfg, l, h->geo[l], l == GRIM_CENTER ? h->gamma : nullptr, h->stream);
  }
  // device scalars; the elements are first set on all-zero grids
  // (timestepper.cpp:287-295), which is the state the first computeDt sees
  memset(h->hst, 0, sizeof(DevState));
  *(volatile unsigned*)h->hostError = 0u;
  {
    unsigned* alias = nullptr;
    e = cudaHostGetDevicePointer((void**)&alias, h->hostError, 0);
    if (e != cudaSuccess) {
      set_err("mapping the host error word: %s", cudaGetErrorString(e));
      free_all(h); delete h; return GRIM_ECUDA;
    }
    h->hst->hostError = alias;
  }
  h->hst->dt = cfg->dt;
  h->hst->time = cfg->time;
  h->hst->first = 1;
  cudaMemcpyAsync(h->st, h->hst, sizeof(DevState), cudaMemcpyHostToDevice, h->stream);
  enqueue_dt_speeds(h, h->primOld, 2);
  e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    set_err("initialisation failed: %s", cudaGetErrorString(e));
    free_all(h); delete h; return GRIM_ECUDA;
  }
  memset(&h->stats, 0, sizeof(h->stats));
  *out = h;
  return GRIM_OK;
}

int grim_destroy(grim_handle* h) {
  if (!h) return GRIM_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_all(h);
  for (int i = 0; i < 8; i++) cudaEventDestroy(h->ev[i]);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return GRIM_OK;
}

int grim_dims(const grim_handle* h, int* a, int* b, int* c, int* dof, int* nf) {
  if (!h) return GRIM_EINVAL;
  if (a) *a = h->dc.N1T;
  if (b) *b = h->dc.N2T;
  if (c) *c = h->dc.N3T;
  if (dof) *dof = h->dc.dof;
  if (nf) *nf = h->dc.nf;
  return GRIM_OK;
}

static double* pick(grim_handle* h, int which) {
  if (which == GRIM_PRIM_OLD) return h->primOld;
  if (which == GRIM_PRIM) return h->prim;
  if (which == GRIM_PRIM_HALF) return h->primHalf;
  return nullptr;
}

int grim_set_prims(grim_handle* h, int which, const double* src, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !src) { set_err("null argument"); return GRIM_EINVAL; }
  double* dst = pick(h, which);
  if (!dst) { set_err("bad state selector %d", which); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  const size_t bytes = (size_t)h->dc.dof * h->bytesZ;
  CK(cudaMemcpyAsync(dst, src, bytes, memKind == GRIM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     h->stream));
  if (memKind != GRIM_DEVICE) CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

int grim_get_prims(grim_handle* h, int which, double* dst, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !dst) { set_err("null argument"); return GRIM_EINVAL; }
  double* src = pick(h, which);
  if (!src) { set_err("bad state selector %d", which); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  const size_t bytes = (size_t)h->dc.dof * h->bytesZ;
  CK(cudaMemcpyAsync(dst, src, bytes, memKind == GRIM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     h->stream));
  if (memKind != GRIM_DEVICE) CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

// ---------------------------------------------------------------------------
// checkpoint files: grid::dump / grid::load (grid.cpp:367-381, 482-499) in
// PETSc's binary Vec format (io.cu), the restart flow of the constructor
// (timestepper.cpp:386-445) and CheckWallClockTermination's write
// (torus/problem.cpp:880-907)
// ---------------------------------------------------------------------------
static long long natural_words(const grim_handle* h) { return h->dc.Zint * (long long)h->dc.dof; }

int grim_dump(grim_handle* h, int which, const char* fileName) {
  if (!h || !fileName) { set_err("null argument"); return GRIM_EINVAL; }
  double* src = pick(h, which);
  if (!src) { set_err("bad state selector %d", which); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  std::vector<double> all((size_t)h->dc.dof * h->dc.Z), nat((size_t)natural_words(h));
  CK(cudaMemcpyAsync(all.data(), src, all.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  int rc = grim_natural_from_prims(&h->cfg, all.data(), nat.data());
  if (rc) return rc;
  return grim_petsc_vec_write(fileName, nat.data(), (long long)nat.size());
}

int grim_load(grim_handle* h, int which, const char* fileName) {
  if (!h || !fileName) { set_err("null argument"); return GRIM_EINVAL; }
  double* dst = pick(h, which);
  if (!dst) { set_err("bad state selector %d", which); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  std::vector<double> nat((size_t)natural_words(h)), all((size_t)h->dc.dof * h->dc.Z, 0.);
  int rc = grim_petsc_vec_read(fileName, nat.data(), (long long)nat.size());
  if (rc) return rc;
  rc = grim_prims_from_natural(&h->cfg, nat.data(), all.data());
  if (rc) return rc;
  // VecLoad into the global vector, then DMGlobalToLocal: the interior from
  // the file, the ghosts as communicate leaves them
  CK(cudaMemcpyAsync(dst, all.data(), all.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  KNS_CALL(h, communicate, h->dc, dst, h->dc.dof, h->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

int grim_write_restart(grim_handle* h, const char* restartFileName, const char* restartFileTime, char* written,
                       int writtenCap) {
  if (!h || !restartFileName || !restartFileTime) { set_err("null argument"); return GRIM_EINVAL; }
  double time = 0., dt = 0.;
  int rc = grim_get_time(h, &time, &dt);
  if (rc) return rc;
  // restartVarsT + the index floor(100 time) zero-padded to 8 digits
  char name[64];
  std::snprintf(name, sizeof(name), "restartVarsT%08lld.bin", (long long)std::floor(time * 100));
  rc = grim_dump(h, GRIM_PRIM_OLD, name);
  if (rc) return rc;
  FILE* fn = std::fopen(restartFileName, "w");
  FILE* ft = std::fopen(restartFileTime, "w");
  bool ok = fn && ft;
  // std::ofstream << double: 6 significant digits, as the reference writes
  if (ok) ok = std::fprintf(fn, "%s\n", name) > 0 && std::fprintf(ft, "%g\n", time) > 0;
  if (fn) ok = (std::fclose(fn) == 0) && ok;
  if (ft) ok = (std::fclose(ft) == 0) && ok;
  if (!ok) { set_err("grim_write_restart: cannot write %s / %s", restartFileName, restartFileTime); return GRIM_EINVAL; }
  if (written && writtenCap > 0) std::snprintf(written, (size_t)writtenCap, "%s", name);
  return GRIM_OK;
}

int grim_restart(grim_handle* h, const char* restartFileName, const char* restartFileTime, const char* restartFile) {
  if (!h) { set_err("null argument"); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  FILE* fn = restartFileName ? std::fopen(restartFileName, "r") : nullptr;
  FILE* ft = restartFileTime ? std::fopen(restartFileTime, "r") : nullptr;
  int rc = GRIM_OK;
  if (fn && ft) {
    double t = 0.;
    char name[4096];
    const bool ok = std::fscanf(ft, "%lf", &t) == 1 && std::fscanf(fn, "%4095s", name) == 1;
    std::fclose(fn);
    std::fclose(ft);
    if (!ok) { set_err("grim_restart: unreadable %s / %s", restartFileName, restartFileTime); return GRIM_EINVAL; }
    double t0 = 0., dt = 0.;
    rc = grim_get_time(h, &t0, &dt);
    if (!rc) rc = grim_set_time(h, t, dt);
    if (!rc) rc = grim_load(h, GRIM_PRIM_OLD, name);
  } else {
    if (fn) std::fclose(fn);
    if (ft) std::fclose(ft);
    if (!restartFile) { set_err("grim_restart: no restart name / time files and no restart file"); return GRIM_EINVAL; }
    rc = grim_load(h, GRIM_PRIM_OLD, restartFile);
  }
  if (rc) return rc;
  // fullStepDiagnostics "to reset the time step" (timestepper.cpp:443-444):
  // NaN reset and floors for the torus, then the element the next computeDt
  // reads
  enqueue_full_diagnostics(h);
  if (h->cfg.ObserveEveryDt > 0.) enqueue_observers(h, h->cfg.ObserveEveryDt, nullptr, true);
  enqueue_dt_speeds(h, h->primOld, 0);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

// GRIM_ETIMEOUT once per raised host error word (a bounded copy wait of an
// earlier launch on this handle gave up); clears the word
static int take_async_error(grim_handle* h) {
  if (!h->hostError || *(volatile unsigned*)h->hostError == 0u) return GRIM_OK;
  *(volatile unsigned*)h->hostError = 0u;
  set_err("a bounded wait on an asynchronous copy gave up in an earlier launch on this handle: the face fluxes of "
          "that stage were not computed, so the state is wrong; set the primitives again before stepping");
  return GRIM_ETIMEOUT;
}

static int run_steps(grim_handle* h, int nsteps) {
  {
    const int rc = take_async_error(h);
    if (rc) return rc;
  }
  h->stageReady = false;
  CK(cudaSetDevice(h->device));
  for (int n = 0; n < nsteps; n++) {
    const bool last = (n == nsteps - 1);
    if (h->graphOn) {
      if (!h->graph) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        long long before = g_launch_counter;
        enqueue_step(h, false);
        h->launchesPerStep = g_launch_counter - before;
        CK(cudaStreamEndCapture(h->stream, &g));
        cudaError_t e = cudaGraphInstantiate(&h->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { set_err("graph instantiate: %s", cudaGetErrorString(e)); return GRIM_ECUDA; }
      }
      if (last) cudaEventRecord(h->ev[0], h->stream);
      CK(cudaGraphLaunch(h->graph, h->stream));
      if (last) cudaEventRecord(h->ev[7], h->stream);
    } else {
      long long before = g_launch_counter;
      enqueue_step(h, last);
      h->launchesPerStep = g_launch_counter - before;
    }
  }
  CK(cudaGetLastError());
  return GRIM_OK;
}

int grim_time_step(grim_handle* h, int* numReads, int* numWrites) {
  if (!h) return GRIM_EINVAL;
  int rc = run_steps(h, 1);
  // algorithmic words per zone of one step: both stages read prims (dof)
  // and write the new prims (dof) plus the stage constants
  if (numReads) *numReads = 2 * h->dc.dof;
  if (numWrites) *numWrites = 2 * h->dc.dof;
  return rc;
}

int grim_time_steps(grim_handle* h, int nsteps) {
  if (!h || nsteps < 0) { set_err("grim_time_steps: null handle or nsteps < 0"); return GRIM_EINVAL; }
  return run_steps(h, nsteps);
}

}  // extern "C"

// interior zones, [var][k][j][i] contiguous (dof x Zint) <-> the same zones
// of a grid array with ghosts; one row of blocks per variable
__global__ void k_interior_copy(DevCfg c, const double* __restrict__ src, double* __restrict__ dst, int toGrid) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.Zint) return;
  const long long v = blockIdx.y;
  const long long z = v * c.Z + interior_to_z(c, n);
  const long long t = v * c.Zint + n;
  if (toGrid) dst[z] = src[t];
  else dst[t] = src[z];
}
static void interior_copy(const DevCfg& c, const double* src, double* dst, bool toGrid, cudaStream_t s) {
  const dim3 grid((unsigned)((c.Zint + 255) / 256), (unsigned)c.dof);
  k_interior_copy<<<grid, 256, 0, s>>>(c, src, dst, toGrid ? 1 : 0);
}

// fluxCT (constrainedtransport.cpp:3-51) on the face fluxes f[0..dim): the
// field rows replaced by averages of the edge EMFs emf = [E1 | E2 | E3] x Z,
// each with its neighbour one zone up along the other direction taken by
// circular shift over the whole array, as af::shift takes it; a
// direction's own field row is zero.  One thread per zone, dim >= 2.
__global__ void k_flux_ct(DevCfg c, double* __restrict__ f1, double* __restrict__ f2, double* __restrict__ f3,
                          const double* __restrict__ emf) {
  const long long z = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= c.Z) return;
  const long long Z = c.Z;
  int i, j, k;
  zijk(c, z, i, j, k);
  const long long zi = zidx(c, (i + 1) % c.N1T, j, k), zj = zidx(c, i, (j + 1) % c.N2T, k);
  const long long b1 = (long long)c.B1 * Z + z, b2 = b1 + Z, b3 = b2 + Z;
  const double* e1 = emf;
  const double* e2 = emf + Z;
  const double* e3 = emf + 2 * Z;
  f1[b1] = 0.;
  f1[b2] = 0.5 * (e3[z] + e3[zj]);
  f2[b1] = -0.5 * (e3[z] + e3[zi]);
  f2[b2] = 0.;
  if (c.dim == 3) {
    const long long zk = zidx(c, i, j, (k + 1) % c.N3T);
    f1[b3] = -0.5 * (e2[z] + e2[zk]);
    f2[b3] = 0.5 * (e1[z] + e1[zk]);
    f3[b1] = 0.5 * (e2[z] + e2[zi]);
    f3[b2] = -0.5 * (e1[z] + e1[zj]);
    f3[b3] = 0.;
  }
}

extern "C" {

// nsteps of (primOld <- hostIn[k]; timeStep; hostOut[k] <- primOld) with the
// copies of one step overlapping the other steps' work: uploads on one
// stream, downloads on another, each through two device staging buffers,
// the step on the handle's stream between a device copy (or an interior
// scatter / gather) in and one out.
int grim_time_steps_host(grim_handle* h, int nsteps, const double* const* hostIn, double* const* hostOut,
                         int layout) {
  if (!h || nsteps < 0 || (layout != GRIM_LAYOUT_GHOSTED && layout != GRIM_LAYOUT_INTERIOR)) {
    set_err("grim_time_steps_host: bad argument");
    return GRIM_EINVAL;
  }
  {
    const int rc = take_async_error(h);
    if (rc) return rc;
  }
  h->stageReady = false;
  CK(cudaSetDevice(h->device));
  const bool interior = layout == GRIM_LAYOUT_INTERIOR;
  const size_t bytes = (size_t)h->dc.dof * h->bytesZ;
  const size_t hostBytes = interior ? (size_t)h->dc.dof * h->dc.Zint * sizeof(double) : bytes;
  if (!h->ioReady) {
    bool ok = true;
    for (int i = 0; i < 2; i++) {
      if (!h->ioIn[i]) ok = ok && cudaMalloc(&h->ioIn[i], bytes) == cudaSuccess;
      if (!h->ioOut[i]) ok = ok && cudaMalloc(&h->ioOut[i], bytes) == cudaSuccess;
    }
    if (!ok) {
      cudaGetLastError();
      for (int i = 0; i < 2; i++) {
        cudaFree(h->ioIn[i]);
        cudaFree(h->ioOut[i]);
        h->ioIn[i] = h->ioOut[i] = nullptr;
      }
      set_err("grim_time_steps_host: staging allocation failed (4 x %zu MB)", bytes >> 20);
      return GRIM_ENOMEM;
    }
    CK(cudaStreamCreateWithFlags(&h->ioUp, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&h->ioDown, cudaStreamNonBlocking));
    for (int i = 0; i < 8; i++) CK(cudaEventCreateWithFlags(&h->ioEv[i], cudaEventDisableTiming));
    h->ioReady = true;
  }
  cudaEvent_t* upDone = h->ioEv;
  cudaEvent_t* inFree = h->ioEv + 2;
  cudaEvent_t* outStaged = h->ioEv + 4;
  cudaEvent_t* outFree = h->ioEv + 6;
  // one step of the pipeline; an error ends the loop below, which still
  // waits for every copy already issued (they read or write the caller's
  // buffers)
  auto pipeline_step = [&](int k) -> int {
    const int s = k & 1;
    if (hostIn && hostIn[k]) {
      // staging buffer s is free once the step of k - 2 has copied it in
      CK(cudaStreamWaitEvent(h->ioUp, inFree[s], 0));
      CK(cudaMemcpyAsync(h->ioIn[s], hostIn[k], hostBytes, cudaMemcpyHostToDevice, h->ioUp));
      CK(cudaEventRecord(upDone[s], h->ioUp));
      CK(cudaStreamWaitEvent(h->stream, upDone[s], 0));
      if (interior) {
        // the periodic ghosts as grid::communicate forms them; the step's
        // boundary pass fills the others
        interior_copy(h->dc, h->ioIn[s], h->primOld, true, h->stream);
        KNS_CALL(h, communicate, h->dc, h->primOld, h->dc.dof, h->stream);
      } else {
        CK(cudaMemcpyAsync(h->primOld, h->ioIn[s], bytes, cudaMemcpyDeviceToDevice, h->stream));
      }
      CK(cudaEventRecord(inFree[s], h->stream));
    }
    const int rc = run_steps(h, 1);
    if (rc) return rc;
    if (hostOut && hostOut[k]) {
      // staging buffer s is free once the download of k - 2 has finished
      CK(cudaStreamWaitEvent(h->stream, outFree[s], 0));
      if (interior) interior_copy(h->dc, h->primOld, h->ioOut[s], false, h->stream);
      else CK(cudaMemcpyAsync(h->ioOut[s], h->primOld, bytes, cudaMemcpyDeviceToDevice, h->stream));
      CK(cudaEventRecord(outStaged[s], h->stream));
      CK(cudaStreamWaitEvent(h->ioDown, outStaged[s], 0));
      CK(cudaMemcpyAsync(hostOut[k], h->ioOut[s], hostBytes, cudaMemcpyDeviceToHost, h->ioDown));
      CK(cudaEventRecord(outFree[s], h->ioDown));
    }
    return GRIM_OK;
  };
  int rc = GRIM_OK;
  for (int k = 0; k < nsteps && rc == GRIM_OK; k++) rc = pipeline_step(k);
  const cudaError_t e1 = cudaStreamSynchronize(h->ioUp);
  const cudaError_t e2 = cudaStreamSynchronize(h->stream);
  const cudaError_t e3 = cudaStreamSynchronize(h->ioDown);
  if (rc) return rc;
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
    set_err("grim_time_steps_host: %s",
            cudaGetErrorString(e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3)));
    return GRIM_ECUDA;
  }
  return take_async_error(h);
}

int grim_get_time(grim_handle* h, double* t, double* dt) {
  if (!h) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(h->hst, h->st, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (t) *t = h->hst->time;
  if (dt) *dt = h->hst->dt;
  return GRIM_OK;
}

int grim_set_time(grim_handle* h, double t, double dt) {
  if (!h) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(h->hst, h->st, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->hst->time = t;
  h->hst->dt = dt;
  CK(cudaMemcpyAsync(h->st, h->hst, sizeof(DevState), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

int grim_compute_dt(grim_handle* h) {
  if (!h) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  KNS_CALL(h, dt_update, h->st, h->cfg.CourantFactor, h->cfg.maxDtIncrement, h->stream);
  CK(cudaGetLastError());
  return GRIM_OK;
}

int grim_apply_boundaries(grim_handle* h, int which) {
  if (!h) { set_err("null argument"); return GRIM_EINVAL; }
  double* p = pick(h, which);
  if (!p) { set_err("bad state selector %d", which); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  KNS_CALL(h, communicate, h->dc, p, h->dc.dof, h->stream);
  KNS_CALL(h, ghost_fill, h->dc, p, h->dc.dof, h->stream);
  CK(cudaGetLastError());
  return GRIM_OK;
}

int grim_communicate(grim_handle* h, int which) {
  if (!h) { set_err("null argument"); return GRIM_EINVAL; }
  double* p = pick(h, which);
  if (!p) { set_err("bad state selector %d", which); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  KNS_CALL(h, communicate, h->dc, p, h->dc.dof, h->stream);
  CK(cudaGetLastError());
  return GRIM_OK;
}

// copy a caller array (host or device) of nv x Z words into a device buffer
static int stage_in(grim_handle* h, double* dst, const double* src, int nv, int memKind) {
  CK(cudaMemcpyAsync(dst, src, (size_t)nv * h->bytesZ,
                     memKind == GRIM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream));
  return GRIM_OK;
}
static int stage_out(grim_handle* h, double* dst, const double* src, size_t bytes, int memKind) {
  CK(cudaMemcpyAsync(dst, src, bytes, memKind == GRIM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

int grim_compute_div_fluxes(grim_handle* h, const double* prim, double* divF, double* fluxes, double* emf,
                            int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !prim) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  h->stageReady = false;  // the pass below replaces divF and the field guess
  int rc = stage_in(h, h->scratch, prim, c.dof, memKind);
  if (rc) return rc;
  // a stencil pass on the scratch prims as a half stage with dt = 0 keeps
  // the stored state untouched except the stage buffers
  StageBufs b = stage_bufs(h, GRIM_HALF_STEP);
  b.ps = h->scratch;
  b.pold = h->scratch;
  double* tmpPrim = h->scratch2;  // receives the guess
  b.prim = tmpPrim;
  if (c.conduction || c.viscosity) KNS_CALL(h, emhd_prepass, c, b.ps, b.geoC, h->uT, h->stream);
  for (int d = 0; d < c.dim; d++)
    KNS_CALL(h, face_flux, c, d, b.ps, b.geoF[d], b.geoC, h->flux[d], h->faceVariant[use_exact(h) ? 0 : 1][d],
             tmap_for(h, b.ps, d), h->st, h->stream);
  // divergence of all dof rows (the time step needs the fluid rows only)
  b.divFB = 1;
  KNS_CALL(h, stage_epilogue, c, GRIM_HALF_STEP, b, h->stream);
  CK(cudaGetLastError());
  if (divF) {
    rc = stage_out(h, divF, h->divF, (size_t)c.dof * h->bytesZ, memKind);
    if (rc) return rc;
  }
  if (fluxes) {
    for (int d = 0; d < 3; d++) {
      double* dst = fluxes + (size_t)d * c.dof * c.Z;
      if (d < c.dim) {
        rc = stage_out(h, dst, h->flux[d], (size_t)c.dof * h->bytesZ, memKind);
        if (rc) return rc;
      }
    }
  }
  if (emf) {
    // three rows of Z; the scratch prims are no longer needed
    const double* fl[3] = {h->flux[0], h->flux[1], h->flux[2]};
    grim::exact::emf(c, fl, h->scratch, h->stream);
    CK(cudaGetLastError());
    rc = stage_out(h, emf, h->scratch, 3 * h->bytesZ, memKind);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

int grim_compute_emf(grim_handle* h, const double* prim, double* emf, int memKind) {
  if (!emf) { set_err("null argument"); return GRIM_EINVAL; }
  return grim_compute_div_fluxes(h, prim, nullptr, nullptr, emf, memKind);
}

int grim_flux_ct(grim_handle* h, const double* prim, double* fluxes, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !prim || !fluxes) { set_err("null argument"); return GRIM_EINVAL; }
  // the Riemann fluxes of prim into the handle's face-flux buffers
  int rc = grim_compute_div_fluxes(h, prim, nullptr, nullptr, nullptr, memKind);
  if (rc) return rc;
  const DevCfg& c = h->dc;
  if (c.dim >= 2) {
    const double* fl[3] = {h->flux[0], h->flux[1], h->flux[2]};
    grim::exact::emf(c, fl, h->scratch, h->stream);
    k_flux_ct<<<(unsigned)((c.Z + 255) / 256), 256, 0, h->stream>>>(c, h->flux[0], h->flux[1],
                                                                     c.dim == 3 ? h->flux[2] : nullptr, h->scratch);
    CK(cudaGetLastError());
  }
  for (int d = 0; d < c.dim; d++) {
    rc = stage_out(h, fluxes + (size_t)d * c.dof * c.Z, h->flux[d], (size_t)c.dof * h->bytesZ, memKind);
    if (rc) return rc;
  }
  return GRIM_OK;
}

int grim_capture_graph(grim_handle* h, int enable) { return grim_enable_graph(h, enable); }

int grim_reconstruct(grim_handle* h, const double* prim, int dir, double* pl, double* pr, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !prim || !pl || !pr || dir < 0 || dir >= h->dc.dim) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  int rc = stage_in(h, h->scratch, prim, c.dof, memKind);
  if (rc) return rc;
  double* dl = h->scratch2;
  double* dr = h->scratch2 + (size_t)c.dof * c.Z;
  KNS_CALL(h, reconstruct, c, dir, h->scratch, dl, dr, h->stream);
  CK(cudaGetLastError());
  rc = stage_out(h, pl, dl, (size_t)c.dof * h->bytesZ, memKind);
  if (rc) return rc;
  return stage_out(h, pr, dr, (size_t)c.dof * h->bytesZ, memKind);
}

int grim_step_segment(grim_handle* h, int segment) {
  if (!h || segment < GRIM_SEG_PRE || segment > GRIM_SEG_POST) { set_err("bad segment"); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  h->stageReady = false;
  enqueue_segment(h, segment);
  CK(cudaGetLastError());
  return GRIM_OK;
}

int grim_halo_x3(grim_handle* h, int which, int side, int unpack, void* buf) {
  if (!h || !buf || (side != 0 && side != 1)) { set_err("bad argument"); return GRIM_EINVAL; }
  double* p = pick(h, which);
  if (!p) { set_err("bad state selector %d", which); return GRIM_EINVAL; }
  const DevCfg& c = h->dc;
  if (c.dim != 3 || c.N3 < c.g3) { set_err("grim_halo_x3: a 3D grid with at least 3 planes"); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  const size_t plane = (size_t)c.N1T * c.N2T;
  // the 3 planes next to the end (pack) or its 3 ghost planes (unpack)
  const int k0 = unpack ? (side == 0 ? 0 : c.N3 + c.g3) : (side == 0 ? c.g3 : c.N3);
  double* grid = p + (size_t)k0 * plane;
  const size_t width = (size_t)c.g3 * plane * sizeof(double), pitch = (size_t)c.Z * sizeof(double);
  if (unpack)
    CK(cudaMemcpy2DAsync(grid, pitch, buf, width, width, (size_t)c.dof, cudaMemcpyDeviceToDevice, h->stream));
  else
    CK(cudaMemcpy2DAsync(buf, width, grid, pitch, width, (size_t)c.dof, cudaMemcpyDeviceToDevice, h->stream));
  return GRIM_OK;
}

static void* scalar_ptr(grim_handle* h, int which, size_t* bytes) {
  if (which == GRIM_SCALAR_MAXINVDT) { *bytes = sizeof(double); return &h->st->maxInvDt; }
  if (which == GRIM_SCALAR_NANFLAG) { *bytes = sizeof(unsigned long long); return &h->st->nanFlag; }
  return nullptr;
}
int grim_scalar_get(grim_handle* h, int which, void* devBuf) {
  if (!h || !devBuf) { set_err("null argument"); return GRIM_EINVAL; }
  size_t n = 0;
  void* src = scalar_ptr(h, which, &n);
  if (!src) { set_err("bad scalar %d", which); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(devBuf, src, n, cudaMemcpyDeviceToDevice, h->stream));
  return GRIM_OK;
}
int grim_scalar_set(grim_handle* h, int which, const void* devBuf) {
  if (!h || !devBuf) { set_err("null argument"); return GRIM_EINVAL; }
  size_t n = 0;
  void* dst = scalar_ptr(h, which, &n);
  if (!dst) { set_err("bad scalar %d", which); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(dst, devBuf, n, cudaMemcpyDeviceToDevice, h->stream));
  return GRIM_OK;
}

int grim_torus_observers(grim_handle* h, double* out) {
  if (!h || !out) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  double* res = h->obs + (size_t)kObsBlocks * OBS_N;
  enqueue_observers(h, 0., res, false);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, res, OBS_N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

int grim_get_observations(grim_handle* h, double* out, int maxRecords, int* nRecords) {
  if (!h || !nRecords || maxRecords < 0 || (maxRecords > 0 && !out)) {
    set_err("grim_get_observations: bad argument"); return GRIM_EINVAL;
  }
  CK(cudaSetDevice(h->device));
  unsigned long long count = 0;
  CK(cudaMemcpyAsync(&count, &h->st->obsCount, sizeof(count), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const unsigned long long cap = (unsigned long long)h->obsCap;
  const unsigned long long kept = count < cap ? count : cap;
  const unsigned long long n = kept < (unsigned long long)maxRecords ? kept : (unsigned long long)maxRecords;
  const double* hist = h->obs + (size_t)kObsBlocks * OBS_N + OBS_N;
  // the n most recent records, oldest first: at most two contiguous runs
  // of the ring
  const size_t rec = (OBS_N + 1) * sizeof(double);
  const unsigned long long first = (count - n) % cap;
  const unsigned long long run1 = (first + n <= cap) ? n : cap - first;
  if (run1) CK(cudaMemcpyAsync(out, hist + first * (OBS_N + 1), run1 * rec, cudaMemcpyDeviceToHost, h->stream));
  if (n > run1)
    CK(cudaMemcpyAsync(out + run1 * (OBS_N + 1), hist, (n - run1) * rec, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  *nRecords = (int)n;
  return GRIM_OK;
}

int grim_compute_divb(grim_handle* h, const double* prim, double* divB, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !prim || !divB) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  int rc = stage_in(h, h->scratch, prim, c.dof, memKind);
  if (rc) return rc;
  const bool mink = h->cfg.metric == GRIM_MINKOWSKI;
  grim::exact::divb(c, h->scratch, mink ? nullptr : h->geo[GRIM_CENTER], h->scratch2, h->stream);
  CK(cudaGetLastError());
  return stage_out(h, divB, h->scratch2, h->bytesZ, memKind);
}

int grim_element_fluxes(grim_handle* h, const double* prim, int dir, double* out, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !prim || !out) { set_err("null argument"); return GRIM_EINVAL; }
  if (dir < 0 || dir > 3) { set_err("grim_element_fluxes: direction %d outside 0..3", dir); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  int rc = stage_in(h, h->scratch, prim, c.dof, memKind);
  if (rc) return rc;
  const bool mink = h->cfg.metric == GRIM_MINKOWSKI;
  KNS_CALL(h, conserved, c, h->scratch, mink ? nullptr : h->geo[GRIM_CENTER], h->scratch2, dir, 0, nullptr,
           nullptr, h->stream);
  CK(cudaGetLastError());
  return stage_out(h, out, h->scratch2, (size_t)c.dof * h->bytesZ, memKind);
}

int grim_conserved(grim_handle* h, const double* prim, double* cons, int memKind) {
  return grim_element_fluxes(h, prim, 0, cons, memKind);
}

int grim_char_speeds(grim_handle* h, const double* prim, int dir, double* mn, double* mx, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !prim || !mn || !mx || dir < 0 || dir > 2) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  int rc = stage_in(h, h->scratch, prim, c.dof, memKind);
  if (rc) return rc;
  const bool mink = h->cfg.metric == GRIM_MINKOWSKI;
  double* a = h->scratch2;
  double* b = h->scratch2 + c.Z;
  KNS_CALL(h, conserved, c, h->scratch, mink ? nullptr : h->geo[GRIM_CENTER], nullptr, 0, dir, a, b, h->stream);
  CK(cudaGetLastError());
  rc = stage_out(h, mn, a, h->bytesZ, memKind);
  if (rc) return rc;
  return stage_out(h, mx, b, h->bytesZ, memKind);
}

int grim_stage_setup(grim_handle* h, int stage) {
  if (!h || (stage != GRIM_HALF_STEP && stage != GRIM_FULL_STEP)) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  double* ps = (stage == GRIM_HALF_STEP) ? h->primOld : h->primHalf;
  KNS_CALL(h, ghost_fill, c, ps, c.dof, h->stream);
  enqueue_problem_bcs(h, ps);
  enqueue_stencil(h, stage);
  h->lastStage = stage;
  h->stageReady = true;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

int grim_get_stage_grid(grim_handle* h, int which, double* out, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !out) { set_err("null argument"); return GRIM_EINVAL; }
  const DevCfg& c = h->dc;
  const double* src = which == GRIM_STAGE_CONS_OLD ? h->consOld
                      : which == GRIM_STAGE_DIV_FLUXES ? h->divF
                      : which == GRIM_STAGE_SOURCES_EXPLICIT ? h->Sexp : nullptr;
  if (!src) { set_err("bad stage grid %d", which); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  const int rows = which == GRIM_STAGE_CONS_OLD ? c.dof : c.nf;
  return stage_out(h, out, src, (size_t)rows * h->bytesZ, memKind);
}

// the Newton pieces read the constants of the stage grim_stage_setup formed
static int stage_ready(grim_handle* h, const char* what) {
  if (h->stageReady) return GRIM_OK;
  set_err("%s: no stage set up (grim_stage_setup), or a step or stencil call has replaced it since", what);
  return GRIM_ESTATE;
}

int grim_residual(grim_handle* h, const double* pg, double* res, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !pg || !res) return GRIM_EINVAL;
  if (const int rc = stage_ready(h, "grim_residual")) return rc;
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  int rc = stage_in(h, h->scratch, pg, c.dof, memKind);
  if (rc) return rc;
  StageBufs b = stage_bufs(h, h->lastStage);
  KNS_CALL(h, residual, c, h->lastStage, b, h->scratch, h->scratch2, h->stream);
  CK(cudaGetLastError());
  return stage_out(h, res, h->scratch2, (size_t)c.nf * h->bytesZ, memKind);
}

static int jac_common(grim_handle* h, const double* pg, double* jac, int memKind, int tangent) {
  if (!h || !pg || !jac) return GRIM_EINVAL;
  if (const int rc = stage_ready(h, "Jacobian")) return rc;
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  int rc = stage_in(h, h->scratch, pg, c.dof, memKind);
  if (rc) return rc;
  double* dj = nullptr;
  const size_t bytes = (size_t)c.Z * c.nf * c.nf * sizeof(double);
  CK(cudaMallocAsync((void**)&dj, bytes, h->stream));
  StageBufs b = stage_bufs(h, h->lastStage);
  if (tangent)
    grim::fast::jacobian(c, h->lastStage, b, h->scratch, dj, tangent, h->stream);
  else
    grim::exact::jacobian(c, h->lastStage, b, h->scratch, dj, 0, h->stream);
  CK(cudaGetLastError());
  rc = stage_out(h, jac, dj, bytes, memKind);
  cudaFreeAsync(dj, h->stream);
  cudaStreamSynchronize(h->stream);
  return rc;
}
int grim_jacobian_fd(grim_handle* h, const double* pg, double* jac, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  return jac_common(h, pg, jac, memKind, 0);
}
int grim_jacobian_tangent(grim_handle* h, const double* pg, double* jac, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  return jac_common(h, pg, jac, memKind, 1);
}
int grim_jacobian_form(grim_handle* h, const double* pg, double* jac, int form, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (form < GRIM_JAC_FD64 || form > GRIM_JAC_FAST32) {
    set_err("grim_jacobian_form: unknown form %d", form);
    return GRIM_EINVAL;
  }
  return jac_common(h, pg, jac, memKind, form);
}

int grim_newton_solve(grim_handle* h, int* iters) {
  if (!h) return GRIM_EINVAL;
  if (const int rc = stage_ready(h, "grim_newton_solve")) return rc;
  CK(cudaSetDevice(h->device));
  cudaMemsetAsync(h->st->count, 0, sizeof(h->st->count), h->stream);
  cudaMemsetAsync(h->st->itersDone, 0, sizeof(h->st->itersDone), h->stream);
  cudaMemsetAsync(h->st->finalUnconv, 0, sizeof(h->st->finalUnconv), h->stream);
  enqueue_newton(h, h->lastStage);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->hst, h->st, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (iters) *iters = (int)h->hst->itersDone[h->lastStage];
  return GRIM_OK;
}

int grim_batch_solve(int n, int batch, const double* A, const double* b, double* x, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (n < 1 || n > 8 || batch < 0 || !A || !b || !x) return GRIM_EINVAL;
  if (batch == 0) return GRIM_OK;
  cudaStream_t s = 0;
  const size_t bA = (size_t)batch * n * n * sizeof(double), bb = (size_t)batch * n * sizeof(double);
  const double *dA = A, *db = b;
  double* dx = x;
  double *tA = nullptr, *tb = nullptr, *tx = nullptr;
  if (memKind != GRIM_DEVICE) {
    CK(cudaMalloc(&tA, bA));
    CK(cudaMalloc(&tb, bb));
    CK(cudaMalloc(&tx, bb));
    CK(cudaMemcpy(tA, A, bA, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(tb, b, bb, cudaMemcpyHostToDevice));
    dA = tA; db = tb; dx = tx;
  }
  grim::exact::batch_solve(n, batch, dA, db, dx, s);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && memKind != GRIM_DEVICE) e = cudaMemcpy(x, tx, bb, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (tA) cudaFree(tA);
  if (tb) cudaFree(tb);
  if (tx) cudaFree(tx);
  if (e != cudaSuccess) { set_err("batch solve: %s", cudaGetErrorString(e)); return GRIM_ECUDA; }
  return GRIM_OK;
}

// The library keeps one (i, j) plane per geometry word (the metric does not
// depend on X3); the ABI exchanges full [word][k][j][i] arrays.
static int plane_to_full(grim_handle* h, double* dst, const double* src, int rows, int memKind) {
  const DevCfg& c = h->dc;
  const cudaMemcpyKind kind = memKind == GRIM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t pb = (size_t)c.GZ * sizeof(double);
  for (int w = 0; w < rows; w++)
    for (int k = 0; k < c.N3T; k++)
      CK(cudaMemcpyAsync(dst + (size_t)w * c.Z + (size_t)k * c.GZ, src + (size_t)w * c.GZ, pb, kind, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}
static int full_to_plane(grim_handle* h, double* dst, const double* src, int rows, int memKind) {
  const DevCfg& c = h->dc;
  const cudaMemcpyKind kind = memKind == GRIM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const size_t pb = (size_t)c.GZ * sizeof(double);
  for (int w = 0; w < rows; w++)  // the k = 0 plane of each word
    CK(cudaMemcpyAsync(dst + (size_t)w * c.GZ, src + (size_t)w * c.Z, pb, kind, h->stream));
  return GRIM_OK;
}

int grim_get_geometry(grim_handle* h, int location, double* out, double* gamma, double* xc, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || location < 0 || location > 4) { set_err("grim_get_geometry: null handle or bad location"); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  if (h->cfg.metric == GRIM_MINKOWSKI) {
    // the stepping kernels take Minkowski as a compile-time constant and
    // store nothing; the geometry kernel's Minkowski branch evaluates the
    // same metric (and zero connection) for the caller, in a scratch plane
    double* tmp = nullptr;
    const size_t words = (size_t)(39 + 64) * (size_t)c.GZ;  // 39 words per location, 64 Christoffels
    CK(cudaMallocAsync((void**)&tmp, words * sizeof(double), h->stream));
    grim::launch_geometry(c, h->cfg, location, tmp, location == GRIM_CENTER ? tmp + (size_t)39 * c.GZ : nullptr,
                          h->stream);
    int rc = GRIM_OK;
    if (out) rc = plane_to_full(h, out, tmp, 34, memKind);
    if (!rc && xc) rc = plane_to_full(h, xc, tmp + 34 * c.GZ, 5, memKind);
    if (!rc && gamma && location == GRIM_CENTER) rc = plane_to_full(h, gamma, tmp + (size_t)39 * c.GZ, 64, memKind);
    cudaFreeAsync(tmp, h->stream);
    CK(cudaStreamSynchronize(h->stream));
    return rc;
  }
  if (out) {
    int rc = plane_to_full(h, out, h->geo[location], 34, memKind);
    if (rc) return rc;
  }
  if (xc) {
    int rc = plane_to_full(h, xc, h->geo[location] + 34 * c.GZ, 5, memKind);
    if (rc) return rc;
  }
  if (gamma && location == GRIM_CENTER) return plane_to_full(h, gamma, h->gamma, 64, memKind);
  return GRIM_OK;
}

int grim_set_geometry(grim_handle* h, int location, const double* in, const double* gamma, const double* xc,
                      int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || location < 0 || location > 4) return GRIM_EINVAL;
  if (h->cfg.metric == GRIM_MINKOWSKI) { set_err("Minkowski geometry is compile-time"); return GRIM_ENOTSUP; }
  CK(cudaSetDevice(h->device));
  int rc = GRIM_OK;
  if (in) rc = full_to_plane(h, h->geo[location], in, 34, memKind);
  if (!rc && xc) rc = full_to_plane(h, h->geo[location] + 34 * h->dc.GZ, xc, 5, memKind);
  if (!rc && gamma && location == GRIM_CENTER) rc = full_to_plane(h, h->gamma, gamma, 64, memKind);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  // the first computeDt depends on the geometry: redo it
  enqueue_dt_speeds(h, h->primOld, 2);
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

int grim_problem_init(grim_handle* h) {
  if (!h) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  if (h->cfg.problem == GRIM_PROBLEM_TORUS) {
    // the tail of the torus initialConditions (problem.cpp:525-540):
    // applyFloor, then fullStepDiagnostics (NaN reset + applyFloor); the
    // element left set by them is what the first computeDt sees
    KNS_CALL(h, torus_floor, h->dc, h->primOld, h->geo[GRIM_CENTER], nullptr, h->stream);
    enqueue_full_diagnostics(h);
    enqueue_dt_speeds(h, h->primOld, 0);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

int grim_set_newton_mode(grim_handle* h, int mode, int perZone, double rtol) {
  if (!h || mode < 0 || mode > 3 || perZone < 0 || perZone > 3) {
    set_err("grim_set_newton_mode: null handle, or mode outside 0..3 or perZone outside 0..3");
    return GRIM_EINVAL;
  }
  h->cfg.newtonMode = mode;
  h->cfg.perZoneConvergence = perZone;
  h->cfg.nonlinearsolve_rtol = rtol;
  h->dc.rtol = rtol;
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  return GRIM_OK;
}

int grim_get_stats(grim_handle* h, grim_stats* out) {
  if (!h || !out) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(h->hst, h->st, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  grim_stats s;
  memset(&s, 0, sizeof(s));
  for (int st = 0; st < 2; st++) {
    s.newtonIters[st] = (int)h->hst->itersDone[st];
    if (is_fd(h)) {
      // zones unconverged after the last iteration performed (count[n] is
      // the tally after n updates; the global break stops at a zero)
      const int n = (int)std::min<unsigned long long>(h->hst->itersDone[st], 15ULL);
      s.unconverged[st] = (long long)h->hst->count[st][n];
    } else {
      s.unconverged[st] = (long long)h->hst->finalUnconv[st];
    }
  }
  s.nonFinite = (long long)h->hst->nonFinite;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, h->ev[0], h->ev[7]) == cudaSuccess) s.msStep = ms;
  if (!h->graphOn) {
    float a = 0, b = 0, c2 = 0, d = 0;
    if (cudaEventElapsedTime(&a, h->ev[1], h->ev[2]) == cudaSuccess &&
        cudaEventElapsedTime(&b, h->ev[4], h->ev[5]) == cudaSuccess)
      s.msStencil = a + b;
    if (cudaEventElapsedTime(&c2, h->ev[2], h->ev[3]) == cudaSuccess &&
        cudaEventElapsedTime(&d, h->ev[5], h->ev[6]) == cudaSuccess)
      s.msNewton = c2 + d;
    s.msOther = s.msStep - s.msStencil - s.msNewton;
  }
  // events a caller never recorded (a batch problem's, untimed steps) make
  // the elapsed-time queries fail; that is handled above, so the pending
  // error is cleared rather than left for the next checked call
  (void)cudaGetLastError();
  s.kernelLaunches = h->launchesPerStep;
  s.waitTimeouts = (long long)h->hst->waitTimeouts;
  s.drainTimeouts = (long long)h->hst->drainTimeouts;
  *out = s;
  return GRIM_OK;
}

int grim_get_newton_histogram(grim_handle* h, long long* out) {
  if (!h || !out) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(h->hst, h->st, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int st = 0; st < 2; st++)
    for (int i = 0; i < 16; i++) out[st * 16 + i] = (long long)h->hst->itHist[st][i];
  return GRIM_OK;
}

int grim_profile_steps(grim_handle* h, int nsteps, double* msPerGroup, long long* launchesPerGroup,
                       int ngroups) {
  if (!h || nsteps < 0 || !msPerGroup || ngroups <= 0) { set_err("grim_profile_steps: bad argument"); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  for (int g = 0; g < ngroups; g++) {
    msPerGroup[g] = 0.;
    if (launchesPerGroup) launchesPerGroup[g] = 0;
  }
  for (int n = 0; n < nsteps; n++) {
    h->profOn = true;
    h->profUsed = 0;
    long long before = g_launch_counter;
    enqueue_step(h, false);
    h->launchesPerStep = g_launch_counter - before;
    h->profOn = false;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    for (size_t k = 0; k < h->profUsed; k++) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, h->profEv[2 * k], h->profEv[2 * k + 1]));
      const int g = h->profGroup[k];
      if (g < ngroups) {
        msPerGroup[g] += ms;
        if (launchesPerGroup) launchesPerGroup[g]++;
      }
    }
  }
  return GRIM_OK;
}

int grim_autotune(grim_handle* h, int* variants, double* msBest) {
  if (!h) { set_err("grim_autotune: null handle"); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  const int unit = use_exact(h) ? 0 : 1;
  StageBufs b = stage_bufs(h, GRIM_HALF_STEP);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  for (int d = 0; d < c.dim; d++) {
    int nv = 1;
    KNS_CALL_RET(h, nv, face_variants, c, d);
    double best = 1e30;
    int bestV = 0;
    for (int v = 0; v < nv; v++) {
      KNS_CALL(h, face_flux, c, d, b.ps, b.geoF[d], b.geoC, h->flux[d], v, tmap_for(h, b.ps, d), h->st,
               h->stream);  // warm-up
      CK(cudaEventRecord(e0, h->stream));
      const int reps = 3;
      for (int r = 0; r < reps; r++)
        KNS_CALL(h, face_flux, c, d, b.ps, b.geoF[d], b.geoC, h->flux[d], v, tmap_for(h, b.ps, d), h->st, h->stream);
      CK(cudaEventRecord(e1, h->stream));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      if (ms / reps < best) { best = ms / reps; bestV = v; }
    }
    h->faceVariant[unit][d] = bestV;
    if (variants) variants[d] = bestV;
    if (msBest) msBest[d] = best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  CK(cudaGetLastError());
  return GRIM_OK;
}

int grim_set_face_variant(grim_handle* h, int dir, int variant) {
  if (!h || dir < 0 || dir >= h->dc.dim) { set_err("grim_set_face_variant: bad direction"); return GRIM_EINVAL; }
  int nv = 1;
  KNS_CALL_RET(h, nv, face_variants, h->dc, dir);
  if (variant < 0 || variant >= nv) {
    set_err("grim_set_face_variant: variant %d out of range [0, %d) for direction %d", variant, nv, dir);
    return GRIM_EINVAL;
  }
  h->faceVariant[use_exact(h) ? 0 : 1][dir] = variant;
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  return GRIM_OK;
}

int grim_set_dt_mode(grim_handle* h, int fixed) {
  if (!h) return GRIM_EINVAL;
  h->fixedDt = fixed != 0;
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  return GRIM_OK;
}

static int adjoint_scope(grim_handle* h) {
  const grim_config& c = h->cfg;
  auto ok_bc = [](int b) { return b == GRIM_PERIODIC || b == GRIM_OUTFLOW || b == GRIM_MIRROR; };
  const bool bcs = ok_bc(c.boundaryLeft) && ok_bc(c.boundaryRight) && ok_bc(c.boundaryBottom) &&
                   ok_bc(c.boundaryTop) && (c.dim < 3 || (ok_bc(c.boundaryFront) && ok_bc(c.boundaryBack)));
  const bool emhd = c.conduction || c.viscosity;
  (void)emhd;
  const bool torusOk = c.problem == GRIM_PROBLEM_TORUS && c.metric != GRIM_MINKOWSKI && c.numGhost == 3 &&
                       (c.dim < 2 || c.N2 >= 6);
  if ((c.dim != 2 && c.dim != 3) || !bcs || (c.problem != GRIM_PROBLEM_NONE && !torusOk) || c.N3Global > 0) {
    set_err("adjoint: supported for 2D and 3D ideal or extended MHD (Minkowski or MKS) with periodic, outflow or "
            "mirror boundaries, without problem hooks or with the torus problem's (MKS, N2 >= 6)");
    return GRIM_ENOTSUP;
  }
  return GRIM_OK;
}

static grim::AdjointGeo adjoint_geo(const grim_handle* h) {
  grim::AdjointGeo g;
  const bool mink = h->cfg.metric == GRIM_MINKOWSKI;
  g.geoC = mink ? nullptr : h->geo[GRIM_CENTER];
  g.geoF[0] = mink ? nullptr : h->geo[GRIM_LEFT];
  g.geoF[1] = mink ? nullptr : h->geo[GRIM_BOTTOM];
  g.geoF[2] = g.geoC;
  g.gamma = mink ? nullptr : h->gamma;
  return g;
}

// work buffers of the reverse sweep: g, Ft (dim x dof), ebar (3), q,
// gface (2 dof), lamh, ubar (nf), bacc (3), lam
static int adjoint_work(grim_handle* h, AdjointBufs& w, double*& lam) {
  const DevCfg& c = h->dc;
  if (!h->adjWork) {
    const bool emhd = c.conduction || c.viscosity;
    const size_t words = (size_t)c.Z * (c.dof * (6 + c.dim) + 3 + c.nf + 3 + (emhd ? 2 * c.dof + 25 : 0));
    if (cudaMalloc(&h->adjWork, words * sizeof(double)) != cudaSuccess) {
      set_err("adjoint: work allocation failed");
      return GRIM_ENOMEM;
    }
  }
  double* wp = h->adjWork;
  w.g = wp; wp += (size_t)c.dof * c.Z;
  w.Ft = wp; wp += (size_t)c.dim * c.dof * c.Z;
  w.ebar = wp; wp += (size_t)3 * c.Z;
  w.q = wp; wp += (size_t)c.dof * c.Z;
  w.gface = wp; wp += (size_t)2 * c.dof * c.Z;
  w.lamh = wp; wp += (size_t)c.dof * c.Z;
  w.ubar = wp; wp += (size_t)c.nf * c.Z;
  w.bacc = wp; wp += (size_t)3 * c.Z;
  lam = wp; wp += (size_t)c.dof * c.Z;
  w.p0bar = w.psl = w.sbar = w.uTbar = w.uTs = nullptr;
  if (c.conduction || c.viscosity) {
    w.p0bar = wp; wp += (size_t)c.dof * c.Z;
    w.psl = wp; wp += (size_t)c.dof * c.Z;
    w.sbar = wp; wp += (size_t)15 * c.Z;
    w.uTbar = wp; wp += (size_t)5 * c.Z;
    w.uTs = wp;
  }
  return GRIM_OK;
}

int grim_adjoint_stencil(grim_handle* h, const double* prim, const double* gbar, double* out, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !prim || !gbar || !out) { set_err("grim_adjoint_stencil: null argument"); return GRIM_EINVAL; }
  int rc = adjoint_scope(h);
  if (rc) return rc;
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  const size_t bytes = (size_t)c.dof * h->bytesZ;
  AdjointBufs w;
  double* lam = nullptr;
  rc = adjoint_work(h, w, lam);
  if (rc) return rc;
  const cudaMemcpyKind in = memKind == GRIM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CK(cudaMemcpyAsync(h->scratch, prim, bytes, in, h->stream));
  CK(cudaMemcpyAsync(w.g, gbar, bytes, in, h->stream));
  CK(cudaMemsetAsync(lam, 0, bytes, h->stream));
  grim::adjoint_stencil_t(c, adjoint_geo(h), h->scratch, w.g, w.Ft, w.ebar, w.q, w.gface, lam, h->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, lam, bytes, memKind == GRIM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

int grim_adjoint_forward(grim_handle* h, int nsteps, int every) {
  if (!h || nsteps <= 0 || every <= 0) { set_err("grim_adjoint_forward: bad argument"); return GRIM_EINVAL; }
  int rc = adjoint_scope(h);
  if (rc) return rc;
  h->stageReady = false;
  CK(cudaSetDevice(h->device));
  const size_t bytes = (size_t)h->dc.dof * h->bytesZ;
  const int nck = (nsteps + every - 1) / every;
  while ((int)h->adjCkpt.size() < nck) {
    double* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) { set_err("adjoint: checkpoint allocation failed"); return GRIM_ENOMEM; }
    h->adjCkpt.push_back(p);
  }
  grim_set_dt_mode(h, 1);
  double t0 = 0., dt = 0.;
  rc = grim_get_time(h, &t0, &dt);
  if (rc) return rc;
  for (int n = 0; n < nsteps; n++) {
    if (n % every == 0)
      CK(cudaMemcpyAsync(h->adjCkpt[n / every], h->primOld, bytes, cudaMemcpyDeviceToDevice, h->stream));
    rc = run_steps(h, 1);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(h->stream));
  h->adjSteps = nsteps;
  h->adjEvery = every;
  h->adjT0 = t0;
  h->adjDt = dt;
  return GRIM_OK;
}

int grim_adjoint_backward(grim_handle* h, const double* lambda, double* grad, int memKind) {
  if (!mem_kind_ok(memKind)) return GRIM_EINVAL;
  if (!h || !lambda || !grad) { set_err("grim_adjoint_backward: null argument"); return GRIM_EINVAL; }
  if (h->adjSteps <= 0) { set_err("grim_adjoint_backward: no grim_adjoint_forward run to reverse"); return GRIM_ESTATE; }
  h->stageReady = false;
  CK(cudaSetDevice(h->device));
  const DevCfg& c = h->dc;
  const size_t bytes = (size_t)c.dof * h->bytesZ;
  const int every = h->adjEvery;
  // segment states (six per step: grim::AdjointStates, four more with EMHD)
  // and work buffers
  const int kinds = (c.conduction || c.viscosity) ? 10 : 6;
  while ((int)h->adjSeg.size() < kinds * every + 1) {
    double* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) { set_err("adjoint: segment allocation failed"); return GRIM_ENOMEM; }
    h->adjSeg.push_back(p);
  }
  AdjointBufs w;
  double* lam = nullptr;
  int rcw = adjoint_work(h, w, lam);
  if (rcw) return rcw;
  double* finalState = h->adjSeg[(size_t)kinds * every];
  auto state = [&](int kind, int t) { return h->adjSeg[(size_t)kind * every + t]; };
  CK(cudaMemcpyAsync(lam, lambda, bytes, memKind == GRIM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     h->stream));
  grim::adjoint_zero_ghosts(c, lam, h->stream);
  CK(cudaMemcpyAsync(finalState, h->primOld, bytes, cudaMemcpyDeviceToDevice, h->stream));
  double tFinal = 0., dtNow = 0.;
  int rc = grim_get_time(h, &tFinal, &dtNow);
  if (rc) return rc;
  const double dt = h->adjDt;
  const int nseg = (h->adjSteps + every - 1) / every;
  for (int seg = nseg - 1; seg >= 0; seg--) {
    const int m = std::min(every, h->adjSteps - seg * every);
    CK(cudaMemcpyAsync(h->primOld, h->adjCkpt[seg], bytes, cudaMemcpyDeviceToDevice, h->stream));
    rc = grim_set_time(h, h->adjT0 + (double)seg * every * dt, dt);
    if (rc) return rc;
    // recompute the segment step by step, keeping the states each step's
    // adjoint reads: the start state with its ghosts filled as the step's
    // boundary pass fills them (the stored state holds grid::communicate's
    // zeros on the outflow / mirror sides) and after the problem's hooks,
    // each stage's Newton solution, primHalfStep after its finish (filled,
    // then after the hooks)
    for (int t = 0; t < m; t++) {
      CK(cudaMemcpyAsync(state(0, t), h->primOld, bytes, cudaMemcpyDeviceToDevice, h->stream));
      KNS_CALL(h, ghost_fill, c, state(0, t), c.dof, h->stream);
      enqueue_segment(h, GRIM_SEG_PRE);
      CK(cudaMemcpyAsync(state(1, t), h->primOld, bytes, cudaMemcpyDeviceToDevice, h->stream));
      enqueue_segment(h, GRIM_SEG_HALF);
      if (kinds > 6) {
        const size_t nfBytes = (size_t)c.nf * h->bytesZ;
        CK(cudaMemcpyAsync(state(6, t), h->divF, nfBytes, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(state(7, t), h->Sexp, nfBytes, cudaMemcpyDeviceToDevice, h->stream));
      }
      CK(cudaMemcpyAsync(state(2, t), h->prim, bytes, cudaMemcpyDeviceToDevice, h->stream));
      CK(cudaMemcpyAsync(state(3, t), h->primHalf, bytes, cudaMemcpyDeviceToDevice, h->stream));
      KNS_CALL(h, ghost_fill, c, state(3, t), c.dof, h->stream);
      enqueue_segment(h, GRIM_SEG_FULL);
      if (kinds > 6) {
        const size_t nfBytes = (size_t)c.nf * h->bytesZ;
        CK(cudaMemcpyAsync(state(8, t), h->divF, nfBytes, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(state(9, t), h->Sexp, nfBytes, cudaMemcpyDeviceToDevice, h->stream));
      }
      CK(cudaMemcpyAsync(state(4, t), h->primHalf, bytes, cudaMemcpyDeviceToDevice, h->stream));
      CK(cudaMemcpyAsync(state(5, t), h->prim, bytes, cudaMemcpyDeviceToDevice, h->stream));
      enqueue_segment(h, GRIM_SEG_POST);
      CK(cudaGetLastError());
    }
    for (int t = m - 1; t >= 0; t--) {
      grim::AdjointStates st;
      st.P0fill = state(0, t);
      st.P0eff = state(1, t);
      st.PhSol = state(2, t);
      st.PhFill = state(3, t);
      st.PhEff = state(4, t);
      st.P1Sol = state(5, t);
      st.divFh = st.Sexph = st.divF1 = st.Sexp1 = nullptr;
      if (kinds > 6) {
        st.divFh = state(6, t);
        st.Sexph = state(7, t);
        st.divF1 = state(8, t);
        st.Sexp1 = state(9, t);
      }
      grim::adjoint_step(c, adjoint_geo(h), dt, st, lam, w, h->stream);
    }
    CK(cudaGetLastError());
  }
  grim::adjoint_zero_ghosts(c, lam, h->stream);
  // leave the stepper where the forward run left it
  CK(cudaMemcpyAsync(h->primOld, finalState, bytes, cudaMemcpyDeviceToDevice, h->stream));
  rc = grim_set_time(h, tFinal, dtNow);
  if (rc) return rc;
  CK(cudaMemcpyAsync(grad, lam, bytes, memKind == GRIM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return GRIM_OK;
}

// ---------------------------------------------------------------------------
// ragged batch: independent problems (grid sizes may differ) stepped
// together on one stream; the compacted Newton of each stage is one launch
// per iteration over all problems' unconverged zones
// ---------------------------------------------------------------------------
struct grim_batch {
  int device = 0;
  std::vector<grim_handle*> h;
  cudaStream_t stream = nullptr;
  BatchEntry* tbl = nullptr;   // device
  BatchState* state = nullptr; // device
  int* lists = nullptr;        // device, 2 x total
  long long total = 0;
  int maxIter = 0;
  int mode = GRIM_NEWTON_MIXED32;
  bool graphOn = false;
  cudaGraphExec_t graph = nullptr;
};

static void batch_free(grim_batch* B) {
  if (B->graph) cudaGraphExecDestroy(B->graph);
  if (B->tbl) cudaFree(B->tbl);
  if (B->state) cudaFree(B->state);
  if (B->lists) cudaFree(B->lists);
  for (grim_handle* h : B->h) {
    if (!h) continue;
    h->stream = nullptr;  // the batch's stream, destroyed below
    grim_destroy(h);
  }
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
}

static int batch_upload(grim_batch* B) {
  std::vector<BatchEntry> t(B->h.size());
  long long off = 0;
  B->maxIter = 0;
  for (size_t p = 0; p < B->h.size(); p++) {
    grim_handle* h = B->h[p];
    t[p].c = h->dc;
    t[p].b[GRIM_HALF_STEP] = stage_bufs(h, GRIM_HALF_STEP);
    t[p].b[GRIM_FULL_STEP] = stage_bufs(h, GRIM_FULL_STEP);
    t[p].offset = off;
    off += h->dc.Zint;
    B->maxIter = std::max(B->maxIter, h->dc.maxIter);
  }
  B->total = off;
  CK(cudaMemcpyAsync(B->tbl, t.data(), sizeof(BatchEntry) * t.size(), cudaMemcpyHostToDevice, B->stream));
  CK(cudaStreamSynchronize(B->stream));
  if (B->graph) { cudaGraphExecDestroy(B->graph); B->graph = nullptr; }
  return GRIM_OK;
}

int grim_batch_create(const grim_config* cfgs, int n, int device, grim_batch** out) {
  if (!cfgs || n <= 0 || !out) { set_err("grim_batch_create: bad argument"); return GRIM_EINVAL; }
  *out = nullptr;
  for (int p = 1; p < n; p++)
    if (cfgs[p].conduction != cfgs[0].conduction || cfgs[p].viscosity != cfgs[0].viscosity) {
      set_err("grim_batch_create: the problems of a batch share conduction / viscosity flags");
      return GRIM_EINVAL;
    }
  grim_batch* B = new grim_batch();
  B->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_err("grim_batch_create: stream creation failed");
    delete B;
    return GRIM_ECUDA;
  }
  for (int p = 0; p < n; p++) {
    grim_handle* h = nullptr;
    int rc = grim_create(&cfgs[p], device, &h);
    if (rc) { B->h.push_back(nullptr); batch_free(B); return rc; }
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(h->stream);
    h->stream = B->stream;
    h->cfg.newtonMode = GRIM_NEWTON_MIXED32;
    h->cfg.perZoneConvergence = 2;
    B->h.push_back(h);
  }
  long long total = 0;
  for (grim_handle* h : B->h) total += h->dc.Zint;
  if (total >= (1LL << 31)) { set_err("grim_batch_create: more than 2^31 zones"); batch_free(B); return GRIM_EINVAL; }
  if (cudaMalloc(&B->tbl, sizeof(BatchEntry) * n) != cudaSuccess ||
      cudaMalloc(&B->state, sizeof(BatchState)) != cudaSuccess ||
      cudaMalloc(&B->lists, sizeof(int) * 2 * (size_t)total) != cudaSuccess) {
    set_err("grim_batch_create: device allocation failed");
    batch_free(B);
    return GRIM_ENOMEM;
  }
  BatchState hs;
  memset(&hs, 0, sizeof(hs));
  hs.list[0] = B->lists;
  hs.list[1] = B->lists + total;
  if (cudaMemcpy(B->state, &hs, sizeof(hs), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_err("grim_batch_create: state upload failed");
    batch_free(B);
    return GRIM_ECUDA;
  }
  int rc = batch_upload(B);
  if (rc) { batch_free(B); return rc; }
  *out = B;
  return GRIM_OK;
}

int grim_batch_destroy(grim_batch* B) {
  if (!B) return GRIM_OK;
  cudaSetDevice(B->device);
  cudaStreamSynchronize(B->stream);
  batch_free(B);
  return GRIM_OK;
}

int grim_batch_size(const grim_batch* B) { return B ? (int)B->h.size() : 0; }

int grim_batch_problem(grim_batch* B, int p, grim_handle** h) {
  if (!B || !h || p < 0 || p >= (int)B->h.size()) { set_err("grim_batch_problem: bad index"); return GRIM_EINVAL; }
  *h = B->h[p];
  return GRIM_OK;
}

int grim_batch_set_newton_mode(grim_batch* B, int mode, double rtol) {
  if (!B || (mode != GRIM_NEWTON_MIXED32 && mode != GRIM_NEWTON_TANGENT64)) {
    set_err("grim_batch_set_newton_mode: the batch runs the tangent or mixed compacted Newton");
    return GRIM_EINVAL;
  }
  for (grim_handle* h : B->h) {
    int rc = grim_set_newton_mode(h, mode, 2, rtol);
    if (rc) return rc;
  }
  B->mode = mode;
  return batch_upload(B);
}

static void enqueue_batch_step(grim_batch* B) {
  const DevCfg& c0 = B->h[0]->dc;
  for (grim_handle* h : B->h) enqueue_pre_half(h, false);
  for (grim_handle* h : B->h) enqueue_stencil(h, GRIM_HALF_STEP);
  grim::fast::batch_newton(c0, B->tbl, (int)B->h.size(), B->total, B->maxIter, GRIM_HALF_STEP, B->mode, B->state,
                           B->stream);
  for (grim_handle* h : B->h) enqueue_mid(h);
  for (grim_handle* h : B->h) enqueue_stencil(h, GRIM_FULL_STEP);
  grim::fast::batch_newton(c0, B->tbl, (int)B->h.size(), B->total, B->maxIter, GRIM_FULL_STEP, B->mode, B->state,
                           B->stream);
  for (grim_handle* h : B->h) enqueue_post(h, false);
}

int grim_batch_enable_graph(grim_batch* B, int enable) {
  if (!B) return GRIM_EINVAL;
  B->graphOn = enable != 0;
  if (!B->graphOn && B->graph) { cudaGraphExecDestroy(B->graph); B->graph = nullptr; }
  return GRIM_OK;
}

int grim_batch_time_steps(grim_batch* B, int nsteps) {
  if (!B || nsteps < 0) return GRIM_EINVAL;
  CK(cudaSetDevice(B->device));
  for (grim_handle* h : B->h)
    if (h->fixedDt != B->h[0]->fixedDt) { set_err("grim_batch_time_steps: mixed dt modes"); return GRIM_EINVAL; }
  for (int n = 0; n < nsteps; n++) {
    if (B->graphOn) {
      if (!B->graph) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_batch_step(B);
        CK(cudaStreamEndCapture(B->stream, &g));
        cudaError_t e = cudaGraphInstantiate(&B->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { set_err("batch graph instantiate: %s", cudaGetErrorString(e)); return GRIM_ECUDA; }
      }
      CK(cudaGraphLaunch(B->graph, B->stream));
    } else {
      enqueue_batch_step(B);
    }
  }
  CK(cudaGetLastError());
  return GRIM_OK;
}

int grim_batch_synchronize(grim_batch* B) {
  if (!B) return GRIM_EINVAL;
  CK(cudaSetDevice(B->device));
  CK(cudaStreamSynchronize(B->stream));
  return GRIM_OK;
}

int grim_count_flops(grim_handle* h, double* out) {
  if (!h || !out) { set_err("grim_count_flops: null argument"); return GRIM_EINVAL; }
  CK(cudaSetDevice(h->device));
  double* d = nullptr;
  CK(cudaMalloc(&d, 11 * sizeof(double)));
  CK(cudaMemsetAsync(d, 0, 11 * sizeof(double), h->stream));
  const long long z = interior_to_z(h->dc, h->dc.Zint / 2);
  grim::fast::count_ops(h->dc, h->lastStage, stage_bufs(h, h->lastStage), z, d, h->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, 11 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d);
  if (e != cudaSuccess) { set_err("grim_count_flops: %s", cudaGetErrorString(e)); return GRIM_ECUDA; }
  return GRIM_OK;
}

int grim_enable_graph(grim_handle* h, int enable) {
  if (!h) return GRIM_EINVAL;
  h->graphOn = enable != 0;
  if (!h->graphOn && h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  return GRIM_OK;
}

int grim_synchronize(grim_handle* h) {
  if (!h) return GRIM_EINVAL;
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  return take_async_error(h);
}

int grim_set_debug(grim_handle* h, int setting, int value) {
  if (!h) return GRIM_EINVAL;
  if (setting != GRIM_DEBUG_SKIP_BULK_COPIES) { set_err("grim_set_debug: unknown setting %d", setting); return GRIM_EINVAL; }
  h->dc.dbgSkipCopies = value != 0;
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  return GRIM_OK;
}

void* grim_stream(grim_handle* h) { return h ? (void*)h->stream : nullptr; }

}  // extern "C"

// Configuration translation for entry points that live outside this file
// (the allocation-free divergence in noalloc.cu); same checks as grim_create.
namespace grim {
int devcfg_from_config(const grim_config& c, DevCfg& d) { return make_devcfg(c, d); }
void set_error_message(const char* msg) { set_err("%s", msg); }
}  // namespace grim
