/*
 * grim_b200.h -- C ABI of the B200 (sm_100a) implicit GRMHD/EMHD timestep.
 *
 * Drop-in for the reference's timeStepper (AFD-Illinois/grim,
 * src/timestepper/timestepper.hpp:19-132): one handle owns the grids,
 * geometry, stage buffers and one CUDA stream, exactly as one timeStepper
 * object owns its grids, geometry objects and fluid elements.
 *
 * Conventions
 *  - Every call returns an int status: 0 = OK, < 0 = error (GRIM_E*).
 *    No exceptions cross the ABI.  A refused argument (NULL handle or
 *    buffer, a selector, kind or count outside its range) returns
 *    GRIM_EINVAL before any work is enqueued, and grim_last_error() says
 *    which; grim_destroy(NULL) and grim_batch_destroy(NULL) do nothing.
 *  - Primitive arrays are FP64 in [var][k][j][i] order including ghost
 *    zones (i fastest), the layout of the reference's grid::vars and of
 *    gridPy.getVars (src/grid/gridPy.pyx:185-221).  N1T = N1 + 2*numGhost,
 *    N2T/N3T likewise for active dimensions (1 otherwise).
 *  - Pointers passed with GRIM_HOST are host memory (pageable or pinned),
 *    GRIM_DEVICE pointers are device memory on the handle's GPU (any other
 *    memKind is GRIM_EINVAL).  The library copies; the caller keeps ownership.
 *  - All work is asynchronous on the handle's stream except the getters of
 *    scalars and statistics, which synchronise.  Calls on one handle are not
 *    thread-safe; different handles are independent.
 */
#ifndef GRIM_B200_H_
#define GRIM_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define GRIM_OK            0
#define GRIM_EINVAL       -1   /* bad argument or configuration */
#define GRIM_ECUDA        -2   /* a CUDA runtime call failed */
#define GRIM_ENOMEM       -3   /* device allocation failed */
#define GRIM_ESTATE       -4   /* call not valid in the current state */
#define GRIM_ENOTSUP      -5   /* configuration not supported */
#define GRIM_ETIMEOUT     -6   /* a bounded device wait gave up */
/* Non-finite primitives are not an error status: a step counts them
 * (grim_stats.nonFinite) and the torus problem resets them, as the
 * reference's fullStepDiagnostics does (torus/problem.cpp:719-878). */

/* ---- enums (src/params.hpp:32-94; MP5, closures, Newton modes are new) -- */
enum { GRIM_PERIODIC = 0, GRIM_OUTFLOW = 1, GRIM_MIRROR = 2, GRIM_DIRICHLET = 3,
       GRIM_EXCHANGE = 4 /* ghosts filled by the caller's halo exchange (slab of a decomposed grid) */ };
enum { GRIM_MINKOWSKI = 0, GRIM_MODIFIED_KERR_SCHILD = 1 };
enum { GRIM_MINMOD = 0, GRIM_WENO5 = 1, GRIM_PPM = 2, GRIM_MP5 = 3 };
enum { GRIM_HLL = 0, GRIM_LOCAL_LAX_FRIEDRICH = 1 };
enum { GRIM_CENTER = 0, GRIM_LEFT = 1, GRIM_RIGHT = 2, GRIM_TOP = 3, GRIM_BOTTOM = 4 };
enum { GRIM_HALF_STEP = 0, GRIM_FULL_STEP = 1 };
enum { GRIM_CLOSURE_CONST_TAU = 0, GRIM_CLOSURE_TORUS = 1, GRIM_CLOSURE_TAU_PROFILE = 2 };
enum { GRIM_PROBLEM_NONE = 0, GRIM_PROBLEM_TORUS = 1 };
enum {
  GRIM_NEWTON_PARITY_FD64 = 0, /* reference method: FD Jacobian, FP64, global break */
  GRIM_NEWTON_TANGENT64   = 1, /* exact forward-tangent Jacobian, FP64 solve */
  GRIM_NEWTON_MIXED32     = 2, /* FP32 tangent Jacobian + FP32 solve, FP64 residual */
  GRIM_NEWTON_FD64_FAST   = 3  /* the reference method (FD Jacobian, FP64 solve, line search,
                                  global break) in the fast path's arithmetic and kernels: the
                                  FD baseline the fast forms are timed against */
};
enum { GRIM_HOST = 0, GRIM_DEVICE = 1 };
enum { GRIM_PRIM_OLD = 0, GRIM_PRIM = 1, GRIM_PRIM_HALF = 2 };

/*
 * Configuration.  Field names are the reference's params:: globals
 * (src/params.hpp:96-210) and timeStepper constructor arguments
 * (timestepper.hpp:94-111).  Integers first, then doubles.
 */
typedef struct grim_config {
  int N1, N2, N3, dim, numGhost;
  int boundaryLeft, boundaryRight, boundaryTop, boundaryBottom;
  int boundaryFront, boundaryBack;
  int metric;
  int DerefineThetaHorizon, DoCylindrify;
  int conduction, viscosity;
  int highOrderTermsConduction, highOrderTermsViscosity;
  int reconstruction, riemannSolver;
  int maxNonLinearIter, maxLineSearchIters;
  int closure;              /* setFluidElementParameters variant */
  int problem;              /* problem hooks: BCs, flux filter, floors */
  int elemOldFromFullStep;  /* 1: fullStepDiagnostics re-sets elemOld */
  int newtonMode;           /* GRIM_NEWTON_* */
  int perZoneConvergence;   /* 0: global break (reference), 1: per zone, 2: compacted,
                               3: per zone with the last update deferred */
  int N3Global;             /* > 0: the handle holds N3 of N3Global X3 planes of a slab
                               decomposition; X3Start / X3End are the global extent */
  int reserved_i[4];
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
  double ObserveEveryDt;    /* > 0: record the torus observers whenever a step's
                               time crosses a multiple of it (problem.cpp:754) */
  double nonlinearsolve_ulps; /* > 0: a zone also counts as converged once its
                               residual is within this many ulps of the residual's
                               largest term, |U|/dt' at the solution, i.e. max over
                               the conserved rows of |divF + S - U_old/dt'| (the
                               rounding floor of an FP64 residual); 0: the
                               reference's test */
  double reserved_d[4];
} grim_config;

typedef struct grim_handle grim_handle;

/* Per-call statistics (grim_get_stats).  Times are CUDA-event milliseconds
 * of the last grim_time_step call, measured on the handle's stream. */
typedef struct grim_stats {
  int    newtonIters[2];       /* Newton iterations of the half / full stage */
  long long unconverged[2];    /* zones above tolerance when each stage ended */
  long long nonFinite;         /* NaN/Inf primitives after the last step */
  double msStep;               /* whole grim_time_step */
  double msStencil;            /* stencil kernels, both stages */
  double msNewton;             /* Newton kernels, both stages */
  double msOther;              /* ghost fill, dt, copies */
  long long kernelLaunches;    /* launches of this library's kernels in the step */
  long long waitTimeouts;      /* bounded waits on asynchronous copies that gave up, since creation */
  long long drainTimeouts;     /* of those, give-ups whose copies in flight did not land either */
  double reserved[6];
} grim_stats;

/* ---- lifecycle: timeStepper::timeStepper / ~timeStepper
 *      (timestepper.cpp:4-470) ------------------------------------------
 * The configuration is checked before any CUDA call; GRIM_EINVAL, with
 * grim_last_error() naming the field, for: dim outside 1..3, numGhost != 3,
 * fewer than 4 zones in an active direction, more than 2^31 - 1 zones with
 * ghosts, an enum field outside its GRIM_* values (metric, reconstruction,
 * riemannSolver, closure, problem, newtonMode, the six boundaries),
 * perZoneConvergence outside 0..3, maxNonLinearIter outside 1..15,
 * maxLineSearchIters outside 1..32, XEnd <= XStart in an active direction,
 * a negative or NaN nonlinearsolve_ulps, an N3Global that is not a 3D slab
 * count >= N3, and the torus problem or closure without the MKS metric. */
int grim_create(const grim_config* cfg, int device, grim_handle** out);
int grim_destroy(grim_handle* h);
int grim_dims(const grim_handle* h, int* N1T, int* N2T, int* N3T, int* dof, int* numFluidVars);
const char* grim_version(void);
const char* grim_last_error(void);

/* ---- state: grid::vars through gridPy.getVars / setVars
 *      (gridPy.pyx:185-221); which = GRIM_PRIM_OLD | GRIM_PRIM | GRIM_PRIM_HALF */
int grim_set_prims(grim_handle* h, int which, const double* src, int memKind);
int grim_get_prims(grim_handle* h, int which, double* dst, int memKind);

/* the problem's tail of timeStepper::initialConditions after the caller has
 * set primOld: for the torus the floors and the first fullStepDiagnostics
 * (torus/problem.cpp:525-540); nothing for the other problems */
int grim_problem_init(grim_handle* h);

/* ---- stepping: timeStepper::timeStep (timestep.cpp:3-334); numReads and
 *      numWrites report the algorithmic words per zone, may be NULL ------ */
int grim_time_step(grim_handle* h, int* numReads, int* numWrites);
int grim_time_steps(grim_handle* h, int nsteps);
/* nsteps of: primOld <- hostIn[k] (when hostIn and hostIn[k] are not NULL),
 * one timeStep, hostOut[k] <- primOld (when hostOut and hostOut[k] are not
 * NULL).  The host arrays are, by layout:
 *   GRIM_LAYOUT_GHOSTED   the whole [var][k][j][i] array with ghosts, as
 *                         grim_set_prims / grim_get_prims: the same results
 *                         as those calls made one after another;
 *   GRIM_LAYOUT_INTERIOR  [var][k][j][i] of the interior zones only
 *                         (dof x N1 x N2 x N3): the input's ghost zones are
 *                         formed from its interior, the periodic ones as
 *                         grid::communicate forms them (grim_communicate),
 *                         the others by the step's boundary pass; the
 *                         results equal the ghosted calls given arrays whose
 *                         ghosts were communicated (a slab's GRIM_EXCHANGE
 *                         halo keeps its values: the caller's to fill).
 * The upload of step k + 1, the step k and the download of step k - 1 run
 * at once (two device staging buffers each way, an upload and a download
 * stream).  Host buffers must be pinned (cudaHostAlloc / cudaHostRegister)
 * for the copies to overlap.  Returns when every step and copy is done;
 * the first call allocates the staging buffers (4 x dof x Z doubles). */
enum { GRIM_LAYOUT_GHOSTED = 0, GRIM_LAYOUT_INTERIOR = 1 };
int grim_time_steps_host(grim_handle* h, int nsteps, const double* const* hostIn, double* const* hostOut,
                         int layout);
int grim_get_time(grim_handle* h, double* time, double* dt);
int grim_set_time(grim_handle* h, double time, double dt);

/* ---- checkpoint files (grid::dump / grid::load, grid.cpp:367-381 and
 *      482-499).  The reference writes the DMDA global vector (interior
 *      zones, natural order, variables interleaved: [k][j][i][var]) with
 *      PETSc's HDF5 viewer; these files hold the same vector in PETSc's
 *      binary Vec format (big-endian int32 class id 1211214, int32 length,
 *      big-endian doubles), which PETSc's VecLoad reads.  HDF5 is not
 *      linked.  A load fills the interior and leaves the ghosts as
 *      communicate does (DMGlobalToLocal). --------------------------------- */
int grim_dump(grim_handle* h, int which, const char* fileName);
int grim_load(grim_handle* h, int which, const char* fileName);
/* CheckWallClockTermination's write (torus/problem.cpp:880-907): primOld to
 * restartVarsT<floor(100 time), 8 digits>.bin, its name into
 * restartFileName and the time (6 significant digits, as std::ostream
 * prints it) into restartFileTime; written (may be NULL) gets the name. */
int grim_write_restart(grim_handle* h, const char* restartFileName, const char* restartFileTime, char* written,
                       int writtenCap);
/* the constructor's restart branch (timestepper.cpp:386-445): with both
 * restartFileName and restartFileTime present, time from the one and
 * primOld from the file the other names; else primOld from restartFile
 * (GRIM_EINVAL when it is NULL or missing).  Then fullStepDiagnostics and
 * the element the next computeDt reads; dt keeps its current value. */
int grim_restart(grim_handle* h, const char* restartFileName, const char* restartFileTime, const char* restartFile);
/* the format pieces, host only (no GPU): the PETSc binary Vec file and the
 * reorder between [var][k][j][i] with ghosts and the natural interior.
 * grim_petsc_vec_read returns GRIM_ENOTSUP for an HDF5 file (the reference's
 * own .h5 restart files), GRIM_EINVAL for anything else it cannot read. */
int grim_petsc_vec_write(const char* fileName, const double* v, long long n);
int grim_petsc_vec_read(const char* fileName, double* v, long long n);
int grim_natural_from_prims(const grim_config* cfg, const double* prims, double* natural);
int grim_prims_from_natural(const grim_config* cfg, const double* natural, double* prims);

/* ---- slab decomposition along X3 (one handle per GPU; the caller moves
 *      the halos and reduces the two scalars, e.g. over NCCL).  A step is
 *      the four segments in order, with, between them:
 *        before 0: maxInvDt <- max over ranks (the next computeDt)
 *        after 1:  X3 halo of GRIM_PRIM_HALF (the stage-end communicate)
 *        after 2:  nanFlag <- sum over ranks (fullStepDiagnostics)
 *        after 3:  X3 halo of GRIM_PRIM_OLD
 *      Ghost sides with boundary GRIM_EXCHANGE are left to the caller; the
 *      dt reduction skips them (they repeat a neighbour's interior). ----- */
enum { GRIM_SEG_PRE = 0, GRIM_SEG_HALF = 1, GRIM_SEG_FULL = 2, GRIM_SEG_POST = 3 };
int grim_step_segment(grim_handle* h, int segment);
/* halo planes of a state: side 0 = low X3 end, 1 = high; pack copies the 3
 * interior planes next to that end into buf, unpack writes buf into the 3
 * ghost planes of that end.  buf: device, dof x 3 x N1T x N2T doubles
 * ([var][plane][j][i]); asynchronous on the handle's stream. */
int grim_halo_x3(grim_handle* h, int which, int side, int unpack, void* buf);
/* device scalars a decomposed run reduces across ranks: 0 = maxInvDt
 * (double), 1 = nanFlag (unsigned 64-bit); devBuf is device memory;
 * asynchronous on the handle's stream */
enum { GRIM_SCALAR_MAXINVDT = 0, GRIM_SCALAR_NANFLAG = 1 };
int grim_scalar_get(grim_handle* h, int which, void* devBuf);
int grim_scalar_set(grim_handle* h, int which, const void* devBuf);

/* ---- torus observers (ObserversTorus.hpp:6-253; fullStepDiagnostics,
 *      torus/problem.cpp:754-778).  Nine values, in this order: baryon mass,
 *      magnetic energy, thermal energy (integrals of rho, b^2, u times
 *      dV sqrt(-g) gamma / alpha over the interior), rho max, plasma beta
 *      min, mass flux through the first (MdotIn) and last (MdotOut) interior
 *      X1 columns, and the unbound (Bernoulli < -1) and relativistic
 *      unbound (also gamma > 2) parts of MdotOut.  The sums are combined in a
 *      fixed order (reproducible run to run). ----------------------------- */
/* now, on primOld; out[9] */
int grim_torus_observers(grim_handle* h, double* out);
/* the records written by grim_time_step when cfg.ObserveEveryDt > 0 (one per
 * step whose time crosses a multiple of it), 10 doubles each: time, then
 * the nine values.  The handle keeps the last 4096; out receives the most
 * recent min(kept, maxRecords), oldest first; *nRecords their number. */
int grim_get_observations(grim_handle* h, double* out, int maxRecords, int* nRecords);

/* ---- stage pieces (timestepper.hpp:88-123) ---------------------------- */
/* computeDt (timestep.cpp:336-400): updates dt from the current elemOld state */
int grim_compute_dt(grim_handle* h);
/* ghost fill of one state buffer: periodic wrap + outflow/mirror
 * (boundary.cpp:5-241, grid.cpp:306-315) */
int grim_apply_boundaries(grim_handle* h, int which);
/* grid::communicate alone (grid.cpp:306-360): the periodic directions'
 * ghosts become images of the interior, the physical ghosts zero (the
 * never-written part of PETSc's local vector) */
int grim_communicate(grim_handle* h, int which);
/* computeDivOfFluxes (fvmfluxes.cpp:3-183) incl. fluxCT/computeEMF
 * (constrainedtransport.cpp:3-83) on a caller's prim array; outputs may be
 * NULL.  divF: dof x Z (the field rows from the constrained-transport
 * fluxes), fluxes: 3 x dof x Z (the Riemann fluxes, before flux-CT), emf:
 * 3 x Z (X1, X2, X3). */
int grim_compute_div_fluxes(grim_handle* h, const double* prim, double* divF,
                            double* fluxes, double* emf, int memKind);
/* computeEMF (constrainedtransport.cpp:53-83) from the Riemann fluxes of a
 * caller's prim array: emf = [emfX1 | emfX2 | emfX3] x Z (emfX3 from 2D on,
 * emfX1 and emfX2 in 3D, zero otherwise) */
int grim_compute_emf(grim_handle* h, const double* prim, double* emf, int memKind);
/* fluxCT (constrainedtransport.cpp:3-51): the Riemann fluxes of a caller's
 * prim array with the field rows replaced by the averages of the edge EMFs
 * (neighbours by circular shift over the whole array, as af::shift takes
 * them), on the GPU: fluxes = dim x dof x Z; in 1D the Riemann fluxes */
int grim_flux_ct(grim_handle* h, const double* prim, double* fluxes, int memKind);
/* reconstruction of one direction (reconstruction.cpp:3-36) */
int grim_reconstruct(grim_handle* h, const double* prim, int dir,
                     double* primLeft, double* primRight, int memKind);
/* computeDivB diagnostic (constrainedtransport.cpp:85-110): divB (1 x Z)
 * at the zone corners from sqrt(-g) B with circular shifts over the whole
 * array; 2D only, zeros otherwise (the reference leaves it unwritten). */
int grim_compute_divb(grim_handle* h, const double* prim, double* divB, int memKind);
/* conserved variables and characteristic speeds of a prim array at the
 * zone centres (physics.cpp:185-217, riemannsolver.cpp:54-200) */
int grim_conserved(grim_handle* h, const double* prim, double* cons, int memKind);
/* fluidElement::set then computeFluxes(dir) (physics.cpp:53-217) at the zone
 * centres with the centre geometry: out (dof x Z) = the fluxes along X^dir,
 * dir 0..3 (0: the conserved variables, as grim_conserved); the reference's
 * fluidElementPy.computeFluxes (physicsPy.pyx:31-42) */
int grim_element_fluxes(grim_handle* h, const double* prim, int dir, double* out, int memKind);
int grim_char_speeds(grim_handle* h, const double* prim, int dir,
                     double* minSpeed, double* maxSpeed, int memKind);

/* ---- Newton pieces (solve.cpp, residual.cpp) -------------------------- */
/* Stage set-up of timeStep (BCs, elemOld, consOld, sources, divF,
 * induction) on the current state, leaving the Newton guess in GRIM_PRIM. */
int grim_stage_setup(grim_handle* h, int stage);
/* The stage grids the last stage left (grim_stage_setup, or the full stage
 * of a step), timeStepperPy's consOld, divFluxes and sourcesExplicit
 * (timestep.cpp:26-79, 180-237): GRIM_STAGE_CONS_OLD is dof x Z (the
 * conserved variables of primOld, formed on the half stage);
 * GRIM_STAGE_DIV_FLUXES and GRIM_STAGE_SOURCES_EXPLICIT are nf x Z, the
 * fluid rows (the field rows of the divergence go straight into the
 * induction update and are not kept; the explicit sources have none).
 * Interior zones only: the ghost entries of out are unspecified.  With the
 * Minkowski metric and ideal MHD the explicit sources are zero and never
 * written. */
enum { GRIM_STAGE_CONS_OLD = 0, GRIM_STAGE_DIV_FLUXES = 1, GRIM_STAGE_SOURCES_EXPLICIT = 2 };
int grim_get_stage_grid(grim_handle* h, int which, double* out, int memKind);
/* computeResidual (residual.cpp:3-180) of a guess: nf x Z */
int grim_residual(grim_handle* h, const double* primGuess, double* residual, int memKind);
/* FD Jacobian (solve.cpp:82-109): [Z][nf][nf], J[z][i][j] = dR_i/dP_j */
int grim_jacobian_fd(grim_handle* h, const double* primGuess, double* jac, int memKind);
/* exact forward-tangent Jacobian of the same residual, same layout (the
 * form the fast Newton uses, in FP64: closed-form dU/dP for ideal MHD, a
 * forward-tangent pass of the residual with EMHD) */
int grim_jacobian_tangent(grim_handle* h, const double* primGuess, double* jac, int memKind);
/* the Jacobian in a chosen form, same layout; extends solve.cpp:82-109 for
 * tests of the fast Newton's Jacobians against each other */
enum {
  GRIM_JAC_FD64 = 0,     /* = grim_jacobian_fd */
  GRIM_JAC_FAST64 = 1,   /* = grim_jacobian_tangent */
  GRIM_JAC_DUAL64 = 2,   /* forward-tangent pass of the residual, also for ideal MHD */
  GRIM_JAC_FAST32 = 3    /* the mixed Newton's Jacobian: FAST64's form on FP32 geometry, in FP32 */
};
int grim_jacobian_form(grim_handle* h, const double* primGuess, double* jac, int form, int memKind);
/* solve() on GRIM_PRIM with the configured newtonMode.
 * grim_residual, the grim_jacobian_* calls and grim_newton_solve read the
 * stage grim_stage_setup formed: they return GRIM_ESTATE before the first
 * grim_stage_setup and after any call that replaces its constants (a step,
 * a step segment, grim_compute_div_fluxes, the adjoint calls). */
int grim_newton_solve(grim_handle* h, int* itersDone);
/* batched pivoted solve of nf x nf systems (the af::solve of solve.cpp:220)
 * A: [batch][n][n] row-major, b: [batch][n] */
int grim_batch_solve(int n, int batch, const double* A, const double* b, double* x, int memKind);

/* ---- geometry (geometry.cpp:4-680) ------------------------------------ */
/* out = [16 gCov | 16 gCon | g | alpha] x Z; gamma (center only) 64 x Z;
 * aux 5 x Z = [x1 | x2 | x1^1.5 | RhoFloorAmpl x1^RhoFloorSlope |
 * UFloorAmpl x1^UFloorSlope] (physical coordinates and the geometry-only
 * fields of the torus closure and floors).  get copies out, set replaces the
 * device copy.  The metrics do not depend on X3: the library stores one
 * (i, j) plane per word, get repeats it over k and set takes the k = 0
 * plane of its input. */
int grim_get_geometry(grim_handle* h, int location, double* out, double* gamma,
                      double* xcoords, int memKind);
int grim_set_geometry(grim_handle* h, int location, const double* in,
                      const double* gamma, const double* xcoords, int memKind);

/* ---- options, statistics, graphs ------------------------------------- */
/* mode: GRIM_NEWTON_*; perZoneConvergence for the tangent / mixed modes:
 * 1 = one kernel, each thread iterates its zone to convergence; 2 = one
 * launch per iteration over a compacted worklist of unconverged zones;
 * 3 = one persistent kernel whose warps run the first maxIter - 1 updates
 * of 32 zones together and gather the zones still unconverged, 32 at a
 * time, for the last update (ideal MHD in the mixed mode with
 * maxNonLinearIter >= 2; anything else runs as 1).  1 and 3 give the same
 * bits. */
int grim_set_newton_mode(grim_handle* h, int mode, int perZoneConvergence, double rtol);
/* zones by Newton iterations used in the last step: out[stage*16 + iters]
 * (tangent / mixed modes) */
int grim_get_newton_histogram(grim_handle* h, long long* out);
int grim_get_stats(grim_handle* h, grim_stats* out);
/* capture timeStep into a CUDA graph and replay it from grim_time_step
 * (grim_capture_graph is the same call) */
int grim_enable_graph(grim_handle* h, int enable);
int grim_capture_graph(grim_handle* h, int enable);
int grim_synchronize(grim_handle* h);

/* Bounded waits.  The TMA-staged face kernels wait on their copies for at
 * most 1 s.  A wait that gives up leaves that kernel's flux rows unwritten,
 * so the stage it belongs to is wrong: it is counted in
 * grim_stats.waitTimeouts and raises an error word in mapped host memory.
 * The next grim_time_step, grim_time_steps or grim_synchronize on the
 * handle that finds the word raised (grim_synchronize always does: it waits
 * first; the stepping calls see it once the kernel has ended) clears it and
 * returns GRIM_ETIMEOUT without stepping; the primitives must then be set
 * again.  The give-up path waits (again bounded) for the copies its warp
 * still has in flight; if one of those does not land either
 * (grim_stats.drainTimeouts), destroy the handle. */
enum {
  GRIM_DEBUG_SKIP_BULK_COPIES = 1  /* value != 0: the TMA-staged face kernels
                                      issue no copies, so their waits run out */
};
/* test hook: set a debug setting; no counterpart in the reference */
int grim_set_debug(grim_handle* h, int setting, int value);
/* the handle's cudaStream_t, as void* */
void* grim_stream(grim_handle* h);

/* ---- self-tests (extends timeStepper::bandwidthTest, timestepper.cpp:473-526):
 *      FP64 and FP32 FMA throughput (TFLOP/s, 2 flops per FMA) and HBM copy
 *      bandwidth (GB/s, read + write) of a device; any pointer may be NULL */
int grim_measure_peaks(int device, double* fp64_tflops, double* fp32_tflops, double* hbm_gbs);

/* ---- measurement.  The reference's own measure is the hand-counted
 *      numReads/numWrites traffic model plus wall time of timeStep
 *      (src/timestepper/timestepper.cpp:473-526, timestep.cpp:330-333).
 *
 * grim_profile_steps runs nsteps steps without the graph and returns the
 * device time of each kernel group, measured with CUDA events recorded
 * around its launches on the handle's stream, summed over the steps, and
 * the number of bracketed launch runs per group. */
enum {
  GRIM_PROF_BOUNDARY = 0,    /* ghost fill, communicate, inflow / pole hooks */
  GRIM_PROF_FACES_X1 = 1,    /* reconstruction + Riemann fluxes at X1 faces */
  GRIM_PROF_FACES_X2 = 2,
  GRIM_PROF_FACES_X3 = 3,
  GRIM_PROF_EPILOGUE = 4,    /* CT EMFs, divergence, sources, induction, guess */
  GRIM_PROF_NEWTON = 5,      /* every Newton kernel of a stage */
  GRIM_PROF_DT = 6,          /* characteristic speeds, dt, time advance */
  GRIM_PROF_DIAGNOSTICS = 7, /* floors, NaN reset / count (outside the stage finish) */
  GRIM_PROF_COPY = 8,        /* stage finish: the state copy with communicate's ghosts,
                                fused with the torus floors, the next dt's speeds and
                                the non-finite count of the step */
  GRIM_PROF_EMHD_PREPASS = 9,
  GRIM_PROF_GROUPS = 10
};
int grim_profile_steps(grim_handle* h, int nsteps, double* msPerGroup, long long* launchesPerGroup,
                       int ngroups);
/* Algorithmic flop counts of one zone (the middle interior zone of the
 * last set-up stage), counted by running the kernels' templated physics on
 * a counting scalar: out[0] residual (FP64), out[1] Jacobian in FP32 (the
 * closed form for ideal MHD, the forward tangent otherwise), out[2] the
 * same in FP64, out[3] pivoted solve FP32, out[4] the same in FP64, out[5]
 * divisions and out[6] sqrt+exp of the residual, out[7] the generic
 * forward-tangent pass in FP32; stencil work in FP64: out[8] the
 * reconstruction of one zone along one direction (all dof), out[9] the
 * Riemann solve of one face, out[10] the epilogue's centre work of one zone
 * (element, conserved vector, geometric source contraction).  Adds and
 * multiplies count 1 each, as do divide, sqrt and exp; out holds 11. */
int grim_count_flops(grim_handle* h, double* out);
/* Autotuner of the face-flux kernels' launch shapes (register budget per
 * thread, lane split between i and the face direction): times every
 * variant of each direction on the state in primOld for the handle's
 * current Newton mode (its compilation unit) and keeps the fastest.
 * variants[d] and msBest[d] (may be null) receive the choice and its time
 * per launch.  In the FP64 parity path (no FMA contraction) every variant
 * gives the same bits; in the fast path they agree to roundoff. */
int grim_autotune(grim_handle* h, int* variants, double* msBest);
/* Forces one variant (for tests); GRIM_EINVAL when out of range. */
int grim_set_face_variant(grim_handle* h, int dir, int variant);

/* ---- adjoint (reverse) sweep of whole timesteps.  No counterpart in the
 *      reference, which has no derivatives; it reverses the reference's
 *      timeStep (timestep.cpp:3-334) with the Newton solves differentiated
 *      implicitly (converged solves; their iterations are not taped).
 *
 * grim_set_dt_mode(h, 1) holds dt at its current value (grim_set_time)
 * instead of timeStepper::computeDt; 0 restores computeDt.
 *
 * grim_adjoint_forward advances nsteps from primOld with dt held fixed,
 * keeping primOld every `every` steps on the device (checkpoints).  primOld
 * must carry periodic ghost images of its interior (grim_apply_boundaries).
 * grim_adjoint_backward takes lambda = dL/d(final primOld) (dof x Z; only
 * interior zones are read) and returns grad = dL/d(initial primOld) for the
 * interior zones (ghost entries zero; the ghosts are images of interior
 * zones and their share is folded in).  Each segment between checkpoints
 * is recomputed forward once; the stepper is left at the final state.
 * Without a grim_adjoint_forward run to reverse it returns GRIM_ESTATE.
 * Supported: 2D and 3D, ideal or extended MHD (conduction and / or
 * viscosity), Minkowski or modified Kerr-Schild (geometric source, face
 * metric), periodic / outflow / mirror boundaries, no problem hooks or the
 * torus problem's (floors after each stage, inflow check and pole fix at
 * the start of each stage, flux filter; MKS, N2 >= 6), ideal or extended
 * MHD.  GRIM_ENOTSUP otherwise (1D, a slab of a decomposed grid).  A zone that
 * fullStepDiagnostics' NaN reset replaces carries no derivative.  Every accumulation is a gather in a fixed
 * order (no atomics): a gradient is the same bits run to run and for any
 * checkpoint interval. */
int grim_set_dt_mode(grim_handle* h, int fixed);

/* ---- ragged batch.  No counterpart in the reference (one problem per
 *      run).  Independent problems, grid sizes free, step together on one
 *      stream: per problem the stencil launches of timeStep, and for each
 *      stage ONE compacted Newton launch per iteration over the unconverged
 *      zones of all problems (tangent or mixed mode).  The problems share
 *      the conduction / viscosity flags; each keeps its own dt, time,
 *      boundaries, metric and reconstruction.  grim_batch_problem returns
 *      problem p's handle for set/get of its state and its statistics;
 *      that handle is owned by the batch (do not destroy it) and runs on
 *      the batch's stream. */
typedef struct grim_batch grim_batch;
int grim_batch_create(const grim_config* cfgs, int n, int device, grim_batch** out);
int grim_batch_destroy(grim_batch* b);
int grim_batch_size(const grim_batch* b);
int grim_batch_problem(grim_batch* b, int p, grim_handle** h);
int grim_batch_set_newton_mode(grim_batch* b, int mode, double rtol);
int grim_batch_enable_graph(grim_batch* b, int enable);
int grim_batch_time_steps(grim_batch* b, int nsteps);
int grim_batch_synchronize(grim_batch* b);
int grim_adjoint_forward(grim_handle* h, int nsteps, int every);
int grim_adjoint_backward(grim_handle* h, const double* lambda, double* grad, int memKind);
/* the transpose of the stencil alone, for tests: out = (d divF / d prim)^T
 * gbar for the interior zones of prim (ghosts taken as periodic images;
 * gbar read on the interior) */
int grim_adjoint_stencil(grim_handle* h, const double* prim, const double* gbar, double* out, int memKind);

/* ---- allocation-free divergence.  No counterpart in the reference: for
 *      callers that cannot call cudaMalloc (their device memory is owned by
 *      their own pool allocator, or they call in the middle of asynchronous
 *      work).  Same result as grim_compute_div_fluxes (interior zones of a
 *      dof x Z divF), on device pointers, enqueued on `stream` (a
 *      cudaStream_t, NULL = default stream) of the current device.  All
 *      scratch lives in one static 64 MiB device array per GPU that loads the
 *      library; grids needing more are rejected with GRIM_EINVAL.  Minkowski
 *      metric only.  The first call on a device looks up that array's address
 *      (make it before any stream capture), as does the first call after a
 *      device reset; calls that overlap on the GPU share the array and
 *      race. */
int grim_div_fluxes_noalloc(const grim_config* cfg, const double* prim, double* divF, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GRIM_B200_H_ */
