// A C++ driver written against the reference-shaped facade
// (include/grim_b200_timestepper.hpp): 2D ideal fast mode 32^2, a few
// timesteps, prints time and checksums of the primitives, of the element
// fluxes along X1 and X0 and of |div B| of the final state.  The GPU test
// compares its output with the Python binding of the same library.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "grim_b200_timestepper.hpp"

int main(int argc, char** argv) {
  const int N = 32, steps = (argc > 1) ? atoi(argv[1]) : 3;
  grim_config c;
  memset(&c, 0, sizeof(c));
  c.N1 = N; c.N2 = N; c.N3 = 1; c.dim = 2; c.numGhost = 3;
  c.boundaryLeft = c.boundaryRight = c.boundaryTop = c.boundaryBottom = GRIM_PERIODIC;
  c.boundaryFront = c.boundaryBack = GRIM_PERIODIC;
  c.metric = GRIM_MINKOWSKI;
  c.reconstruction = GRIM_MINMOD; c.riemannSolver = GRIM_LOCAL_LAX_FRIEDRICH;
  c.maxNonLinearIter = 3; c.maxLineSearchIters = 3;
  c.elemOldFromFullStep = 1;
  c.newtonMode = GRIM_NEWTON_PARITY_FD64;
  c.X1Start = 0.; c.X1End = 1.; c.X2Start = 0.; c.X2End = 1.; c.X3Start = 0.; c.X3End = 1.;
  c.dt = 0.5 / N;
  c.rhoFloorInFluidElement = c.uFloorInFluidElement = 1e-20;
  c.bSqrFloorInFluidElement = c.temperatureFloorInFluidElement = 1e-20;
  c.adiabaticIndex = 4. / 3.;
  c.slopeLimTheta = 2.;
  c.nonlinearsolve_atol = 1e-20; c.JacobianAssembleEpsilon = 4e-8; c.linesearchfloor = 1e-24;
  c.CourantFactor = 0.5; c.maxDtIncrement = 1.3; c.closureTau0 = 1.;
  grimb200::timeStepper ts(c);
  std::vector<double> P(ts.primOld.size());
  const int n1 = ts.primOld.N1Total, n2 = ts.primOld.N2Total;
  const double base[8] = {1., 2., 0., 0., 0., 0.1, 0.3, 0.};
  for (int v = 0; v < 8; v++)
    for (int j = 0; j < n2; j++)
      for (int i = 0; i < n1; i++) {
        const double x = (i - 3 + 0.5) / N, y = (j - 3 + 0.5) / N;
        P[(size_t)v * n1 * n2 + (size_t)j * n1 + i] = base[v] + 1e-4 * (v + 1) * cos(2 * M_PI * (x + y) + v);
      }
  ts.primOld.setVars(P.data());
  int r, w;
  for (int s = 0; s < steps; s++) ts.timeStep(r, w);
  std::vector<double> Q = ts.primOld.getVars();
  double sum = 0.;
  for (int v = 0; v < 8; v++)
    for (int j = 3; j < 3 + N; j++)
      for (int i = 3; i < 3 + N; i++) sum += Q[(size_t)v * n1 * n2 + (size_t)j * n1 + i];
  // the element's X1 fluxes and the conserved variables of the final state,
  // and the corner divergence of its field
  std::vector<double> F(Q.size()), U(Q.size()), D((size_t)n1 * n2);
  ts.computeFluxes(Q.data(), 1, F.data());
  ts.computeFluxes(Q.data(), 0, U.data());
  ts.computeDivB(Q.data(), D.data());
  double sumF = 0., sumU = 0., sumD = 0.;
  for (int v = 0; v < 8; v++)
    for (int j = 3; j < 3 + N; j++)
      for (int i = 3; i < 3 + N; i++) {
        sumF += F[(size_t)v * n1 * n2 + (size_t)j * n1 + i];
        sumU += U[(size_t)v * n1 * n2 + (size_t)j * n1 + i];
      }
  for (int j = 3; j < 3 + N; j++)
    for (int i = 3; i < 3 + N; i++) sumD += fabs(D[(size_t)j * n1 + i]);
  printf("%.17g %.17g %.17g %.17g %.17g\n", ts.time, sum, sumF, sumU, sumD);
  return 0;
}
