// kernels_exact.cu -- kernel instantiations compiled with --fmad=false: the
// FP64 parity path, whose operation order matches the oracle bit for bit.
#define GRIM_KNS exact
#include "kernels.cuh"
#include "launch.h"
