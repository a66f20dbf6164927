// grim_b200_timestepper.hpp -- header-only C++ facade over the C ABI with
// the reference's class and member names, for C++ drivers that used
// AFD-Illinois/grim's timeStepper (src/timestepper/timestepper.hpp:19-132).
//
//   grim_config cfg = ...;            // params:: values
//   grimb200::timeStepper ts(cfg);    // timeStepper::timeStepper
//   ts.primOld.setVars(host);         // gridPy.setVars layout [var][k][j][i]
//   int r, w; ts.timeStep(r, w);      // timeStepper::timeStep
//   ts.primOld.getVars(host);
//
// Errors from the C ABI are thrown as grimb200::error (the reference's
// timeStepper has no error channel; it aborts).
#ifndef GRIM_B200_TIMESTEPPER_HPP_
#define GRIM_B200_TIMESTEPPER_HPP_

#include <stdexcept>
#include <string>
#include <vector>

#include "grim_b200.h"

namespace grimb200 {

struct error : std::runtime_error {
  int status;
  error(const std::string& what, int s) : std::runtime_error(what), status(s) {}
};

inline void check(int rc, const char* what) {
  if (rc != GRIM_OK) throw error(std::string(what) + ": " + grim_last_error(), rc);
}

class timeStepper;

// One state grid (the reference's grid: vars[] of N1Total x N2Total x N3Total)
class grid {
 public:
  int numVars = 0, N1Total = 0, N2Total = 0, N3Total = 0;
  size_t size() const { return (size_t)numVars * N1Total * N2Total * N3Total; }
  void getVars(double* host) const { check(grim_get_prims(h_, which_, host, GRIM_HOST), "getVars"); }
  void setVars(const double* host) { check(grim_set_prims(h_, which_, host, GRIM_HOST), "setVars"); }
  std::vector<double> getVars() const {
    std::vector<double> v(size());
    getVars(v.data());
    return v;
  }
  void getVarsDevice(double* dev) const { check(grim_get_prims(h_, which_, dev, GRIM_DEVICE), "getVarsDevice"); }
  void setVarsDevice(const double* dev) { check(grim_set_prims(h_, which_, dev, GRIM_DEVICE), "setVarsDevice"); }
  // grid::communicate + boundaries::applyBoundaryConditions
  void communicate() { check(grim_apply_boundaries(h_, which_), "communicate"); }

 private:
  friend class timeStepper;
  grim_handle* h_ = nullptr;
  int which_ = GRIM_PRIM_OLD;
};

class timeStepper {
 public:
  double dt = 0., time = 0.;
  int N1 = 0, N2 = 0, N3 = 0, numGhost = 3, dim = 2, numVars = 0;
  grid prim, primOld, primHalfStep;

  explicit timeStepper(const grim_config& cfg, int device = 0) {
    check(grim_create(&cfg, device, &h_), "timeStepper");
    int a, b, c, dof, nf;
    check(grim_dims(h_, &a, &b, &c, &dof, &nf), "dims");
    N1 = cfg.N1; N2 = cfg.N2; N3 = cfg.N3; numGhost = cfg.numGhost; dim = cfg.dim; numVars = dof;
    for (grid* g : {&prim, &primOld, &primHalfStep}) {
      g->h_ = h_; g->numVars = dof; g->N1Total = a; g->N2Total = b; g->N3Total = c;
    }
    prim.which_ = GRIM_PRIM;
    primOld.which_ = GRIM_PRIM_OLD;
    primHalfStep.which_ = GRIM_PRIM_HALF;
    sync_time();
  }
  ~timeStepper() { grim_destroy(h_); }
  timeStepper(const timeStepper&) = delete;
  timeStepper& operator=(const timeStepper&) = delete;

  // timeStepper::timeStep (timestep.cpp:3-334)
  void timeStep(int& numReads, int& numWrites) {
    check(grim_time_step(h_, &numReads, &numWrites), "timeStep");
    sync_time();
  }
  // timeStepper::computeDt (timestep.cpp:336-400)
  void computeDt(int& numReads, int& numWrites) {
    check(grim_compute_dt(h_), "computeDt");
    numReads = numWrites = 0;
    sync_time();
  }
  // the problem's tail of initialConditions (torus floors + diagnostics)
  void initialConditionsDone() { check(grim_problem_init(h_), "problem_init"); }
  // timeStepper::computeDivOfFluxes (fvmfluxes.cpp:3-183) on a host array
  void computeDivOfFluxes(const double* primHost, double* divFluxesHost) {
    check(grim_compute_div_fluxes(h_, primHost, divFluxesHost, nullptr, nullptr, GRIM_HOST),
          "computeDivOfFluxes");
  }
  // timeStepper::computeEMF / fluxCT (constrainedtransport.cpp:3-83) on
  // the Riemann fluxes of a host array: 3 x Z EMFs; dim x dof x Z fluxes
  void computeEMF(const double* primHost, double* emfHost) {
    check(grim_compute_emf(h_, primHost, emfHost, GRIM_HOST), "computeEMF");
  }
  void fluxCT(const double* primHost, double* fluxesHost) {
    check(grim_flux_ct(h_, primHost, fluxesHost, GRIM_HOST), "fluxCT");
  }
  // timeStepper::computeDivB (constrainedtransport.cpp:85-110), 1 x Z
  void computeDivB(const double* primHost, double* divBHost) {
    check(grim_compute_divb(h_, primHost, divBHost, GRIM_HOST), "computeDivB");
  }
  // fluidElement::set + computeFluxes(dir) (physics.cpp:53-217) at the zone
  // centres, dof x Z; dir 0 gives the conserved variables
  void computeFluxes(const double* primHost, int dir, double* fluxHost) {
    check(grim_element_fluxes(h_, primHost, dir, fluxHost, GRIM_HOST), "computeFluxes");
  }
  // consOld / divFluxes / sourcesExplicit of the last stage
  // (GRIM_STAGE_*; grim_get_stage_grid)
  void stageGrid(int which, double* outHost) {
    check(grim_get_stage_grid(h_, which, outHost, GRIM_HOST), "stageGrid");
  }
  void setNewtonMode(int mode, int perZone, double rtol) {
    check(grim_set_newton_mode(h_, mode, perZone, rtol), "setNewtonMode");
  }
  void enableGraph(bool on) { check(grim_enable_graph(h_, on ? 1 : 0), "enableGraph"); }
  grim_stats stats() {
    grim_stats s;
    check(grim_get_stats(h_, &s), "stats");
    return s;
  }
  grim_handle* handle() { return h_; }

 private:
  grim_handle* h_ = nullptr;
  void sync_time() { check(grim_get_time(h_, &time, &dt), "get_time"); }
};

}  // namespace grimb200

#endif  // GRIM_B200_TIMESTEPPER_HPP_
