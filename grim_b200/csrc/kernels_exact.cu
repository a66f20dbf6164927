// kernels_exact.cu -- kernel instantiations compiled with --fmad=false: the
// FP64 parity path, whose operation order matches the oracle bit for bit.
#define GRIM_KNS exact
#define GRIM_SKIP_FACES 1  // in faces_exact.cu
#include "kernels.cuh"
#include "launch.h"
