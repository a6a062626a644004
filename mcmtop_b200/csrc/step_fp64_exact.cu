// FP64 step kernels, reference arithmetic: compiled with --fmad=false.
#define MCM_FLAVOUR_NS exact
#define MCM_EXACT 1
#include "step_fp64.cuh"
