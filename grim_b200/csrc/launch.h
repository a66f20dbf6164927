// launch.h -- host-side launchers of the kernels of one translation unit.
// kernels_exact.cu defines them in grim::exact (FP64 without FMA
// contraction: the parity path), kernels_fast.cu in grim::fast.
#pragma once
#include "stage.cuh"

#define GRIM_DECLARE_LAUNCHERS(NS)                                                                      \
  namespace grim {                                                                                      \
  namespace NS {                                                                                        \
  void ghost_fill(const DevCfg& c, double* prim, int nv, cudaStream_t s);                               \
  void communicate(const DevCfg& c, double* prim, int nv, cudaStream_t s);                              \
  void emhd_prepass(const DevCfg& c, const double* ps, const double* geoC, double* uT, cudaStream_t s); \
  void face_flux(const DevCfg& c, int dir, const double* ps, const double* geoF, const double* geoC,    \
                 double* flux, int variant, const CUtensorMap* tmap, DevState* st, cudaStream_t s);    \
  int face_variants(const DevCfg& c, int dir);                                                          \
  void stage_epilogue(const DevCfg& c, int stage, const StageBufs& b, cudaStream_t s);                  \
  void dt_speeds(const DevCfg& c, const double* p, const double* geoC, int mode, DevState* st,          \
                 cudaStream_t s);                                                                       \
  void dt_update(DevState* st, double courant, double maxInc, cudaStream_t s);                          \
  void advance_time(DevState* st, cudaStream_t s);                                                      \
  void newton_fd_init(const DevCfg& c, int stage, const StageBufs& b, cudaStream_t s);                  \
  void newton_fd_iter(const DevCfg& c, int stage, int it, const StageBufs& b, cudaStream_t s);          \
  void newton_fast(const DevCfg& c, int stage, const StageBufs& b, int mode, const int* list,           \
                   long long nlist, cudaStream_t s);                                                    \
  void newton_list(const DevCfg& c, int stage, const StageBufs& b, int mode, cudaStream_t s);          \
  void residual(const DevCfg& c, int stage, const StageBufs& b, const double* pg, double* out,         \
                cudaStream_t s);                                                                        \
  void jacobian(const DevCfg& c, int stage, const StageBufs& b, const double* pg, double* jac,         \
                int tangent, cudaStream_t s);                                                           \
  void conserved(const DevCfg& c, const double* p, const double* geoC, double* out, int fdir, int dir, \
                 double* mn, double* mx, cudaStream_t s);                                               \
  void reconstruct(const DevCfg& c, int dir, const double* p, double* pl, double* pr, cudaStream_t s); \
  int batch_solve(int n, int batch, const double* A, const double* b, double* x, cudaStream_t s);      \
  void count_nonfinite(const DevCfg& c, const double* p, DevState* st, cudaStream_t s);                \
  void divb(const DevCfg& c, const double* p, const double* geoC, double* out, cudaStream_t s);        \
  void emf(const DevCfg& c, const double* const* flux, double* out, cudaStream_t s);                   \
  void torus_floor(const DevCfg& c, double* p, const double* geoC, const unsigned long long* flag,     \
                   cudaStream_t s);                                                                     \
  void torus_nan_flag(const DevCfg& c, const double* p, unsigned long long* flag, cudaStream_t s);      \
  void torus_observe(const DevCfg& c, const double* p, const double* geoC, double volElem, double every, \
                     DevState* st, double* partials, double* out, double* hist, int cap, cudaStream_t s); \
  void stage_finish(const DevCfg& c, const double* src, double* dst, const double* geoC, bool floors,   \
                    bool post, const unsigned long long* nanFlag, int dtOn, DevState* st,               \
                    cudaStream_t s);                                                                    \
  void torus_bcs(const DevCfg& c, double* p, const double* geoC, cudaStream_t s);                      \
  }                                                                                                     \
  }

GRIM_DECLARE_LAUNCHERS(exact)
GRIM_DECLARE_LAUNCHERS(fast)

namespace grim {
// adjoint.cu: work buffers of the reverse sweep (dof x Z unless noted)
struct AdjointBufs {
  double* g;     // dL/d divF of the stage
  double* Ft;    // dim x dof x Z: face-flux adjoints per direction
  double* ebar;  // 3 x Z: edge EMF adjoints (e3, e1, e2)
  double* q;     // stencil adjoint before the periodic fold
  double* gface; // 2 x dof x Z: adjoints of the two reconstructed states of the faces along one direction
  double* lamh;  // dL/dPh
  double* ubar;  // nf x Z: dL/dU(P0)
  double* bacc;  // 3 x Z: dL/dB0 through the induction
  // EMHD: dL/dP0 through both stages' constants (dof x Z), dL/dPs through
  // the full stage's reference element (dof x Z), the source's slope
  // adjoints (15 x Z), the u_mu, T adjoints (5 x Z), u_mu, T of Ps (5 x Z)
  double* p0bar;
  double* psl;
  double* sbar;
  double* uTbar;
  double* uTs;
};
// the geometry the adjoint reads (all null in Minkowski)
struct AdjointGeo {
  const double* geoC;     // centre planes
  const double* geoF[3];  // face planes per direction (X3: the centre's)
  const double* gamma;    // centre Christoffel planes
};
// the states one step's adjoint reads (dof x Z each)
struct AdjointStates {
  const double* P0fill;  // the step's start state, ghosts filled by the boundary pass
  const double* P0eff;   // the same after the problem's boundary hooks (the half stage's input)
  const double* PhSol;   // the half stage's Newton solution (before its finish)
  const double* PhFill;  // primHalfStep after the half stage's finish, ghosts filled
  const double* PhEff;   // the same after the problem's boundary hooks (the full stage's input)
  const double* P1Sol;   // the full stage's Newton solution (before its finish)
  // EMHD: each stage's divF and Sexp (nf x Z; the row normalisation of q
  // and deltaP multiplies them)
  const double* divFh;
  const double* Sexph;
  const double* divF1;
  const double* Sexp1;
};
// lam (dL/dP1, interior) -> dL/dP0 for one step of fixed dt
void adjoint_step(const DevCfg& c, const AdjointGeo& geo, double dt, const AdjointStates& st, double* lam,
                  const AdjointBufs& w, cudaStream_t s);
void adjoint_zero_ghosts(const DevCfg& c, double* a, cudaStream_t s);
// out = D(P)^T g: the transpose of the flux divergence with its ghost fill
void adjoint_stencil_t(const DevCfg& c, const AdjointGeo& geo, const double* P, const double* g, double* Ft,
                       double* ebar, double* q, double* gface, double* out, cudaStream_t s);
}  // namespace grim

namespace grim {
namespace fast {
// the compacted Newton of a ragged batch: one launch per iteration over
// all problems' unconverged zones (tbl, bs in device memory)
void batch_newton(const DevCfg& c0, const BatchEntry* tbl, int nprob, long long total, int maxIter, int stage,
                  int mode, BatchState* bs, cudaStream_t s);
// the deferred-tail Newton (ideal MHD, mixed form, maxIter >= 2): one
// persistent launch per stage; false when the configuration is not one it
// runs (the caller then runs newton_fast)
bool newton_defer(const DevCfg& c, int stage, const StageBufs& b, int mode, cudaStream_t s);
// algorithmic flop counts of one zone's residual / tangent / solve
void count_ops(const DevCfg& c, int stage, const StageBufs& b, long long z, double* out, cudaStream_t s);
}  // namespace fast
}  // namespace grim
