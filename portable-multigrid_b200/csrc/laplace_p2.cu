// Slab-kernel launchers for FE_Q(2).
#define PMG_DEGREE 2
#include "laplace_launch.cuh"
