/*
 * grim_oracle.h -- C ABI of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain C++ restatement, in FP64
 * with -ffp-contract=off, of the implicit GRMHD/EMHD timestep of
 * AFD-Illinois/grim (src/timestepper, src/physics, src/reconstruction,
 * src/geometry, src/boundary).  It is used by tests/, by the cpu_baseline leg
 * of bench.py and by __graft_entry__.smoke() as the checker; no product code
 * links or calls it.
 *
 * The configuration struct has the same field list and order as the
 * product's grim_config so one Python dict marshals into both.
 */
#ifndef GRIM_ORACLE_H_
#define GRIM_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_config {
  /* ---- integers ---- */
  int N1, N2, N3, dim, numGhost;
  int boundaryLeft, boundaryRight, boundaryTop, boundaryBottom;
  int boundaryFront, boundaryBack;
  int metric;
  int DerefineThetaHorizon, DoCylindrify;
  int conduction, viscosity;
  int highOrderTermsConduction, highOrderTermsViscosity;
  int reconstruction, riemannSolver;
  int maxNonLinearIter, maxLineSearchIters;
  int closure;
  int problem;
  int elemOldFromFullStep;
  int newtonMode;
  int perZoneConvergence;
  int N3Global;
  int reserved_i[4];
  /* ---- doubles ---- */
  double blackHoleSpin, hSlope;
  double X1Start, X1End, X2Start, X2End, X3Start, X3End;
  double time, dt;
  double X1cyl, X2cyl;
  double rhoFloorInFluidElement, uFloorInFluidElement;
  double bSqrFloorInFluidElement, temperatureFloorInFluidElement;
  double adiabaticIndex, ConductionAlpha, ViscosityAlpha;
  double ConductionClosureFactor, ViscosityClosureFactor;
  double slopeLimTheta;
  double nonlinearsolve_atol, nonlinearsolve_rtol;
  double JacobianAssembleEpsilon, linesearchfloor;
  double CourantFactor, maxDtIncrement;
  double closureTau0, closureTau1;
  double MaxLorentzFactor, RhoFloorAmpl, UFloorAmpl, RhoFloorSlope, UFloorSlope;
  double BsqrOverRhoMax, BsqrOverUMax;
  double ObserveEveryDt;
  double nonlinearsolve_ulps;  // product-only (rounding floor of the fast Newton test); the oracle ignores it
  double reserved_d[4];
} orc_config;

typedef struct orc_handle orc_handle;

/* which state buffer a get/set refers to */
enum { ORC_PRIM_OLD = 0, ORC_PRIM = 1, ORC_PRIM_HALF = 2 };

int  orc_create(const orc_config* cfg, orc_handle** out);
void orc_destroy(orc_handle* h);
int  orc_num_vars(const orc_handle* h, int* dof, int* numFluidVars);
int  orc_dims(const orc_handle* h, int* N1T, int* N2T, int* N3T);

/* prims in [var][k][j][i] order, ghosts included */
int  orc_set_prims(orc_handle* h, int which, const double* src);
int  orc_get_prims(const orc_handle* h, int which, double* dst);

int  orc_time_step(orc_handle* h, int nsteps);
int  orc_get_time(const orc_handle* h, double* time, double* dt);
int  orc_set_time(orc_handle* h, double time, double dt);
int  orc_compute_dt(orc_handle* h);

/* boundary fill of a [var][k][j][i] array in place (nv vars) */
int  orc_apply_boundaries(const orc_handle* h, double* prim, int nv);

/* geometry at a location (0 CENTER, 1 LEFT, 2 RIGHT, 3 TOP, 4 BOTTOM):
 * out = [16 gCov | 16 gCon | g | alpha] x Z,  gamma = 64 x Z (center only),
 * xcoords = [x1 | x2 | x1^1.5 | radial rho floor | radial u floor] x Z */
int  orc_geometry(const orc_handle* h, int location, double* out, double* gamma,
                  double* xcoords);

/* stage pieces on a given prim array (ghosts already filled):
 * divF (dof x Z), fluxes (3 x dof x Z, may be NULL), emf (3 x Z, may be NULL) */
int  orc_div_fluxes(orc_handle* h, const double* prim, double* divF,
                    double* fluxes, double* emf);
/* reconstruction of one direction: left/right faces (dof x Z each) */
int  orc_reconstruct(orc_handle* h, const double* prim, int dir,
                     double* primLeft, double* primRight);
/* conserved variables U = computeFluxes(0) of prim, dof x Z */
int  orc_conserved(orc_handle* h, const double* prim, double* cons);
int  orc_element_fluxes(orc_handle* h, const double* prim, int dir, double* out);
int  orc_get_stage_grid(const orc_handle* h, int which, double* out);
int  orc_compute_divb(orc_handle* h, const double* prim, double* divB);
/* torus observers on primOld: mass, EMag, ETh, rhoMax, betaMin, MdotIn,
 * MdotOut, unbound and relativistic unbound MdotOut (9 values) */
int  orc_torus_observers(orc_handle* h, double* out);
/* characteristic speeds of prim at the centre in one direction */
int  orc_char_speeds(orc_handle* h, const double* prim, int dir,
                     double* minSpeed, double* maxSpeed);

/* Half-stage set-up on primOld (BCs, elemOld, consOld, sources, divF,
 * induction), leaving the Newton guess in prim; then residual / FD Jacobian
 * of an arbitrary guess and the Newton solve itself. */
int  orc_stage_setup(orc_handle* h, int stage);
int  orc_residual(orc_handle* h, const double* primGuess, double* residual);
int  orc_jacobian_fd(orc_handle* h, const double* primGuess, double* jac);
int  orc_newton(orc_handle* h, int* iters_done);

/* dense solve of a batch of n x n systems with the oracle's pivoted
 * elimination; A is [batch][n][n] row-major, b [batch][n] -> x */
int  orc_batch_solve(int n, int batch, const double* A, const double* b, double* x);

/* per-call statistics of the last Newton solves */
int  orc_last_newton_stats(const orc_handle* h, int* iters_half, int* iters_full);

/* the problem's tail of initialConditions (torus: floors + diagnostics) */
int  orc_problem_init(orc_handle* h);

int  orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
