// Launchers exported by each arithmetic variant of kernels_impl.cuh.
// v_fp64: FP64 with FMA contraction; v_exact: FP64 with one rounding per
// operation (translation unit built with -fmad=false); v_mixed: FP32
// primitives, reconstruction, fluxes, EMF and divergence, FP64 cell C2P,
// HLLD p* iteration and RK accumulation; v_fp32: FP32 throughout.
#pragma once

#include <cuda_runtime.h>

#include "hlld_b200.h"

namespace hlld {

// Scratch arrays of one 2D step (carved out of the caller's buffer).
struct Scratch2D {
    void *Fx[7];  // x-face fluxes: D, Sx, Sy, Sz, tau, Bz, By (the variant's real type)
    void *Fy[7];  // y-face fluxes: D, Sx, Sy, Sz, tau, Bz, Bx
    void *Ez;     // corner EMF (the variant's real type)
    double *U0[6];  // RK stage-0 copy of the evolved cell variables (float in the FP32 form)
    double *Bx0, *By0;
    hlld_step_diag_t *diag;  // used when the caller passes none
    double *mu_warm;         // mixed form: each cell's last C2P root (warm start), or NULL
};

#define HLLD_DECLARE_VARIANT(NS)                                                                  \
    namespace NS {                                                                                \
    void launch_riemann_faces(int64_t n, const void *const *sL, const void *const *sR, int idir,  \
                              int solver, double gamma, void *const *F, void *const *U,           \
                              void *pstar, int32_t *err, int32_t *iters, uint8_t *flags,          \
                              hlld_flux_diag_t *diag, cudaStream_t st);                           \
    void launch_cons_to_prim(int64_t n, const void *const *cons, double gamma, double atmo_rho,   \
                             double atmo_eps, void *const *prim, uint8_t *status,                 \
                             cudaStream_t st);                                                    \
    void launch_prim_to_cons(int64_t n, const void *const *prim, void *const *cons,               \
                             cudaStream_t st);                                                    \
    void launch_sync_state(const hlld_grid2d_t *g, const hlld_state2d_t *s, uint8_t *status,      \
                           hlld_step_diag_t *diag, cudaStream_t st, double *mu_out = nullptr,     \
                           double *mu_warm = nullptr, bool start_from_prims = false,              \
                           cudaEvent_t after_cons = nullptr);                                     \
    void launch_rk_step_ct(const hlld_grid2d_t *g, const hlld_state2d_t *s, const Scratch2D &sc,  \
                           double dt_host, const double *dt_dev, int scheme,                      \
                           hlld_step_diag_t *diag, cudaStream_t st,                               \
                           cudaEvent_t cons_in = nullptr, cudaEvent_t cons_out = nullptr);        \
    void launch_compute_dt_2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, double cfl,        \
                              double *dt_dev, unsigned long long *work, cudaStream_t st);         \
    void launch_sweep2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, int axis,                \
                        void *const *F, hlld_flux_diag_t *fdiag, cudaStream_t st,                 \
                        double *pstar_out = nullptr, uint8_t *fail_out = nullptr);                \
    void launch_tubes_run(const hlld_tubes_t *b, void *const *cons, void *const *prims,           \
                          void *const *U0, void *const *F, double *t_out, int32_t *steps_out,     \
                          unsigned int *next, int threads, int blocks, cudaStream_t st);          \
    void launch_ct_update2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, const Scratch2D &sc,  \
                            const hlld_step_diag_t *diag, int stage, int scheme, double dt_host,  \
                            const double *dt_dev, cudaStream_t st);                               \
    }

// Records the detail string hlld_last_error_detail() returns; returns code.
int report_error(int code, const char *fmt, ...);

HLLD_DECLARE_VARIANT(v_fp64)
namespace v_adj {  // the discrete adjoint of the FP64 step (adjoint_fp64.cu)
size_t adjoint_scratch_bytes(const hlld_grid2d_t *g);
size_t adjoint_tape_bytes(const hlld_grid2d_t *g);
size_t adjoint_reverse_scratch_bytes(const hlld_grid2d_t *g);
void launch_adjoint_record(const hlld_grid2d_t *g, const hlld_state2d_t *s, double dt, int scheme,
                           void *tape, void *scratch, cudaStream_t st);
void launch_adjoint_reverse(const hlld_grid2d_t *g, const hlld_state2d_t *s_in,
                            const hlld_state2d_t *s_out, double dt, int scheme, const void *tape,
                            const hlld_state2d_t *lam, void *scratch, cudaStream_t st);
void launch_adjoint_rk_step_ct(const hlld_grid2d_t *g, const hlld_state2d_t *s_in,
                               const hlld_state2d_t *s_out, double dt, int scheme,
                               const hlld_state2d_t *lam, void *scratch, cudaStream_t st);
void launch_prim_to_cons_vjp(int64_t n, const void *const *prim, const void *const *lam_cons,
                             void *const *lam_prim, cudaStream_t st);
}
HLLD_DECLARE_VARIANT(v_exact)
HLLD_DECLARE_VARIANT(v_mixed)
HLLD_DECLARE_VARIANT(v_fp32)

}  // namespace hlld
