// faces_exact.cu -- the face-flux kernels of the FP64 parity path
// (--fmad=false), in a unit of their own so their launch-shape variants
// compile in parallel with the rest.
#define GRIM_KNS exact
#define GRIM_ONLY_FACES 1
#include "kernels.cuh"
#include "launch.h"
