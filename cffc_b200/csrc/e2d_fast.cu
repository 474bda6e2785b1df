// Fast FP64 kernels: the same source as e2d_exact.cu compiled with FMA
// contraction on; results differ from the reference only by FMA rounding.
#define E2D_NS fast
#include "e2d_stage.cuh"
