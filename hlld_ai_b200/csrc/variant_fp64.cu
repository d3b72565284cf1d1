// FP64 variant with FMA contraction (the production FP64 form).
#define HLLD_NS v_fp64
#include "kernels_impl.cuh"
