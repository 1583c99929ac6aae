// Slab-kernel launchers for FE_Q(5).
#define PMG_DEGREE 5
#include "laplace_launch.cuh"
