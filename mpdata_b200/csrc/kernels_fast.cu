// Kernels with nvcc's default FMA contraction (the production arithmetic).
#define MPD_NS fast
#include "kernels_all.cuh"
