// Slab-kernel launchers for FE_Q(3).
#define PMG_DEGREE 3
#include "laplace_launch.cuh"
