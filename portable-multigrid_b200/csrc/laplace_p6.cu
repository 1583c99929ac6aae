// Slab-kernel launchers for FE_Q(6).
#define PMG_DEGREE 6
#include "laplace_launch.cuh"
