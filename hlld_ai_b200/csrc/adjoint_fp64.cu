// Discrete adjoint of the FP64 step, in a translation unit of its own so
// that it compiles in parallel with the forward variants.  It takes the
// device code of the FP64 form (same flags as variant_fp64.cu) under its
// own namespace and recomputes the forward stages with the FP64 variant's
// launchers.
#define HLLD_NS v_adj
#define HLLD_DEVICE_ONLY
#include "kernels_impl.cuh"
#include "adjoint_impl.cuh"
