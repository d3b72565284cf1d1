// Mixed-precision variant: FP32 primitives, reconstruction, physical
// fluxes, HLL state, HLL-state C2P (the p* bracket seed), corner EMF and flux
// divergence; FP64 HLLD p* bracket and iteration, HLLD star states, cell C2P
// and RK accumulation of the conserved state and the staggered field.
#define HLLD_NS v_mixed
#define HLLD_NR_RCP 1  // Newton reciprocal for the FP64 p* solve's shared denominators
// Newton square root for the FP64 p* residual and Kastaun master function
// (measured on B200, rotor 2048^2: x sweep 0.899 -> 0.886 ms)
#define HLLD_NR_SQRT 1
#define HLLD_REAL float
#ifndef HLLD_BRACKET_REAL
#define HLLD_BRACKET_REAL float
#endif
#include "kernels_impl.cuh"
