// noalloc.cu -- grim_div_fluxes_noalloc: the flux divergence of a caller's
// primitive array (reconstruction, Riemann fluxes, flux-CT, divergence) with
// every piece of scratch memory taken from one file-scope device array, so
// the call itself allocates nothing.
//
// Some callers cannot call cudaMalloc: a host code whose device memory is
// entirely owned by its own pool allocator, or one that calls in the middle
// of asynchronous work where an allocation (which may synchronise the
// device) is not allowed.  They pass device pointers for the input and the
// output; the face fluxes and the other intermediates live in
// g_noalloc_scratch below.
//
//  * The array holds GRIM_NOALLOC_SCRATCH_WORDS doubles (64 MiB).  Every GPU
//    that loads the library keeps it until the process exits.
//  * Sizes that need more scratch than that are rejected (GRIM_EINVAL with
//    the limit in grim_last_error()).
//  * Host code cannot use the array's name as a device address; the first
//    call on each device looks the address up with cudaGetSymbolAddress
//    (with that device current) and caches it with the device's current
//    context.  Make that first call before any stream capture.  A device
//    reset (cudaDeviceReset) replaces the context and may move the array: a
//    call that finds another context current looks the address up again
//    (again, not inside a stream capture).
//  * All calls share the array and it keeps the last call's contents.  The
//    device scalars the kernels read are cleared at every call.  Calls that
//    overlap on the GPU (different streams, or different host threads on
//    one device) race on the array: serialise them.
//  * Compiled like the parity kernels (no FMA contraction): the result is
//    bit for bit the one of grim_compute_div_fluxes.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "launch.h"

#define GRIM_NOALLOC_SCRATCH_WORDS (8LL * 1024 * 1024)

static __device__ __align__(256) double g_noalloc_scratch[GRIM_NOALLOC_SCRATCH_WORDS];

namespace grim {
int devcfg_from_config(const grim_config& c, DevCfg& d);
void set_error_message(const char* msg);
}  // namespace grim

namespace {
const int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
CUcontext g_scratch_ctx[kMaxDevices] = {nullptr};  // the context each cached address belongs to
std::mutex g_scratch_mu;

// the calling thread's current context (cuCtxGetCurrent through the
// runtime's driver entry point: the library does not link libcuda)
int current_context(CUcontext* ctx) {
  typedef CUresult (*CtxGetCurrent)(CUcontext*);
  static CtxGetCurrent fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      return GRIM_ECUDA;
    fn = reinterpret_cast<CtxGetCurrent>(p);
  }
  return fn(ctx) == CUDA_SUCCESS ? GRIM_OK : GRIM_ECUDA;
}

// device address of g_noalloc_scratch on the current device: looked up with
// cudaGetSymbolAddress (checked) on the first call on a device, and again
// when the device's context has changed since (a device reset); cached
int scratch_address(int device, double** out) {
  if (device < 0 || device >= kMaxDevices) return GRIM_EINVAL;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  // cudaGetDevice does not create the primary context; the lookup below
  // does, so the context is read after it on a first call
  CUcontext ctx = nullptr;
  if (current_context(&ctx) != GRIM_OK) {
    grim::set_error_message("grim_div_fluxes_noalloc: cuCtxGetCurrent failed");
    return GRIM_ECUDA;
  }
  if (!g_scratch_ptr[device] || ctx == nullptr || ctx != g_scratch_ctx[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      grim::set_error_message("grim_div_fluxes_noalloc: cudaGetSymbolAddress of the scratch array failed");
      return GRIM_ECUDA;
    }
    if (current_context(&ctx) != GRIM_OK) {
      grim::set_error_message("grim_div_fluxes_noalloc: cuCtxGetCurrent failed");
      return GRIM_ECUDA;
    }
    g_scratch_ptr[device] = static_cast<double*>(p);
    g_scratch_ctx[device] = ctx;
  }
  *out = g_scratch_ptr[device];
  return GRIM_OK;
}
}  // namespace

extern "C" int grim_div_fluxes_noalloc(const grim_config* cfg, const double* prim, double* divF,
                                       void* stream) {
  using namespace grim;
  if (!cfg || !prim || !divF) {
    set_error_message("grim_div_fluxes_noalloc: null argument");
    return GRIM_EINVAL;
  }
  if (cfg->metric != GRIM_MINKOWSKI) {
    set_error_message("grim_div_fluxes_noalloc: only the Minkowski metric (no geometry arrays)");
    return GRIM_ENOTSUP;
  }
  DevCfg c;
  int rc = devcfg_from_config(*cfg, c);
  if (rc) return rc;
  const long long Z = c.Z;
  const bool emhd = c.conduction || c.viscosity;
  // scratch layout (words): face fluxes dim*dof*Z | consOld dof*Z | guess
  // dof*Z | Sexp nf*Z | uT 5*Z (EMHD) | device scalars
  const long long stateWords = (long long)((sizeof(DevState) + 255) / 256 * 256 / sizeof(double));
  const long long need = (long long)c.dim * c.dof * Z + 2LL * c.dof * Z + (long long)c.nf * Z +
                         (emhd ? 5LL * Z : 0LL) + stateWords;
  if (need > GRIM_NOALLOC_SCRATCH_WORDS) {
    char msg[256];
    snprintf(msg, sizeof(msg),
             "grim_div_fluxes_noalloc: grid needs %lld scratch doubles, the maximum is %lld "
             "(64 MiB); use grim_compute_div_fluxes",
             need, (long long)GRIM_NOALLOC_SCRATCH_WORDS);
    set_error_message(msg);
    return GRIM_EINVAL;
  }
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return GRIM_ECUDA;
  double* base = nullptr;
  rc = scratch_address(device, &base);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* w = base;
  StageBufs b;
  memset(&b, 0, sizeof(b));
  for (int d = 0; d < c.dim; d++) { b.flux[d] = w; w += (long long)c.dof * Z; }
  b.consOld = w; w += (long long)c.dof * Z;
  b.prim = w; w += (long long)c.dof * Z;
  b.Sexp = w; w += (long long)c.nf * Z;
  if (emhd) { b.uT = w; w += 5LL * Z; }
  b.st = reinterpret_cast<DevState*>(w);
  b.ps = prim;
  b.pold = prim;
  b.divF = divF;
  b.divFB = 1;
  b.geoC = nullptr;
  b.gamma = nullptr;
  // dt = 0 for the induction part of the epilogue (its output is not used)
  if (cudaMemsetAsync(b.st, 0, sizeof(DevState), s) != cudaSuccess) return GRIM_ECUDA;
  if (emhd) exact::emhd_prepass(c, prim, nullptr, b.uT, s);
  for (int d = 0; d < c.dim; d++) exact::face_flux(c, d, prim, nullptr, nullptr, b.flux[d], 0, nullptr, nullptr, s);
  exact::stage_epilogue(c, GRIM_HALF_STEP, b, s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error_message(cudaGetErrorString(e));
    return GRIM_ECUDA;
  }
  return GRIM_OK;
}
