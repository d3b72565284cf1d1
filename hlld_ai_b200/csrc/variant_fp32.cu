// All-FP32 variant: primitives, reconstruction, fluxes, the HLLD p* solve and
// star states, the cell C2P, the conserved state, the staggered field and
// the RK accumulation all in float (the 2D step and the tube kernel; the
// flattened per-face and per-cell entry points stay FP64).  A precision
// study beside the FP64 and mixed forms: every constant comes from K<float>.
#define HLLD_NS v_fp32
#define HLLD_REAL float
#define HLLD_BRACKET_REAL float
#define HLLD_STATE_REAL float
#include "kernels_impl.cuh"
