// kernels_fast.cu -- kernel instantiations compiled with FMA contraction on:
// the tangent / mixed-precision paths.
#define GRIM_KNS fast
#define GRIM_FAST_MATH 1
#define GRIM_SKIP_FACES 1  // in faces_fast.cu
#include "kernels.cuh"
#include "launch.h"
#include "opcount.cuh"
