// FP64 variant built with -fmad=false: one rounding per operation, in the
// reference's operation order.
#define HLLD_NS v_exact
#define HLLD_EXACT_ARITH 1
#include "kernels_impl.cuh"
