// faces_fast.cu -- the face-flux kernels of the tangent / mixed-precision
// path (FMA contraction on), in a unit of their own so their launch-shape
// variants compile in parallel with the rest.
#define GRIM_KNS fast
#define GRIM_FAST_MATH 1
#define GRIM_ONLY_FACES 1
#include "kernels.cuh"
#include "launch.h"
