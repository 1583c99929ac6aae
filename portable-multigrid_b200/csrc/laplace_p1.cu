// Slab-kernel launchers for FE_Q(1).
#define PMG_DEGREE 1
#include "laplace_launch.cuh"
