// FP64 step kernels with fused multiply-add and reciprocals.
#define MCM_FLAVOUR_NS fast
#define MCM_EXACT 0
#include "step_fp64.cuh"
