// stage.cuh -- device state and stage buffers shared by the kernels and the
// host runtime.
#pragma once
#include "common.cuh"

namespace grim {

// device-resident scalars of the stepper (dt, time and the Newton counters
// live here so a captured step needs no host round trip)
struct DevState {
  double dt, time, maxInvDt, dtOld;
  int first;
  int pad;
  unsigned long long count[2][16];   // unconverged zones per stage / iteration
  unsigned long long itersDone[2];
  unsigned long long nonFinite;
  unsigned long long finalUnconv[2];
  unsigned long long nanFlag;
  unsigned long long itHist[2][16];  // zones by Newton iterations used (fast path)
  unsigned long long listCount[2];   // compacted worklists: entries per ping-pong list
  unsigned long long waitTimeouts;   // bounded waits on asynchronous copies that gave up
  unsigned long long obsCount;       // torus observer records written (ring index = count % capacity)
  unsigned long long drainTimeouts;  // give-up paths whose wait for their own copies in flight gave up too
  unsigned* hostError;               // device alias of the handle's mapped host error word (null: none)
};

// the torus observers (ObserversTorus.hpp:6-253), in record order
enum {
  OBS_MASS = 0, OBS_EMAG, OBS_ETH, OBS_RHOMAX, OBS_BETAMIN, OBS_MDOT_IN, OBS_MDOT_OUT, OBS_UNBOUND_OUT,
  OBS_REL_UNBOUND_OUT, OBS_N
};
constexpr int kObsBlocks = 740;  // fixed partial count (5 blocks of 128 per SM): the sums' order does not depend on the launch

struct StageBufs {
  const double* ps;       // prims the stage's fluxes are computed from
  const double* pold;     // primOld
  double* prim;           // Newton guess / result
  const double* geoC;     // centre geometry (39 x Z) or null (Minkowski)
  const double* gamma;    // centre Christoffels (64 x Z) or null
  const double* geoF[3];  // face geometry per direction or null
  double* flux[3];        // face fluxes per direction, dof x Z
  double* uT;             // EMHD pre-pass: u_mu (4) + T (1), 5 x Z
  double* consOld;        // dof x Z (fluid rows then B rows)
  double* divF;           // dof x Z (fluid rows, then B rows)
  int divFB;              // the epilogue writes divF's B rows too (else the fluid rows only)
  int guessOld;           // half stage: the per-zone Newton reads its guess's fluid rows from
                          // pold, so the epilogue does not copy them into prim
  double* Sexp;           // nf x Z
  double* R;              // nf x Z  (Newton scratch)
  double* l2;             // 2 x Z   (l2, l2first)
  DevState* st;
  unsigned long long* nanCount;  // non-null: the per-zone Newton adds the zones whose result (fluid and field
                                 // rows) holds a NaN (fullStepDiagnostics' count of the full stage)
  int* list[2];           // compacted Newton worklists (interior zone indices)
};

// one problem of a ragged batch: its configuration, its stage buffers
// (half, full) and the offset of its first interior zone in the batch's
// concatenated index space
struct BatchEntry {
  DevCfg c;
  StageBufs b[2];
  long long offset;
};
// the batch's shared worklists (global interior indices) and their counts
struct BatchState {
  unsigned long long listCount[2];
  int* list[2];
};

}  // namespace grim
