// Kernels compiled with -fmad=false: every product and sum rounds on its own,
// as in a strict-IEEE CPU build of the reference.
#define MPD_NS strict
#include "kernels_all.cuh"
