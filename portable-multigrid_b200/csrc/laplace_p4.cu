// Slab-kernel launchers for FE_Q(4).
#define PMG_DEGREE 4
#include "laplace_launch.cuh"
