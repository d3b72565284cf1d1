/*
 * hlld_b200 C ABI: B200 (sm_100a) kernels for the special-relativistic MHD
 * finite-volume step of kemi2805/HLLD-AI (HLLE/HLLD fluxes, Kastaun C2P,
 * PLM/WENO5-Z/MP5 reconstruction, constrained transport, SSP-RK2/3).
 *
 * Conventions
 *   - All array arguments are DEVICE pointers to contiguous row-major
 *     arrays; no entry point allocates device memory except where stated.
 *   - Real arrays are double for HLLD_FP64 / HLLD_FP64_EXACT; for
 *     HLLD_MIXED the primitive arrays are float and everything else double;
 *     for HLLD_FP32 every state array (conserved, primitive, staggered
 *     field) is float (see each entry point).
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Every
 *     entry point only enqueues work; nothing synchronises the host.
 *   - Return value: HLLD_OK or a negative HLLD_ERR_* code;
 *     hlld_error_string() names it and hlld_last_error_detail() gives the
 *     last failure's message.  Numeric failures (non-converged roots,
 *     fallbacks) are never errors: they are reported in status/flag arrays
 *     and device counters, as the reference reports them in masks.
 *
 * 2D layout (src/physics/grid.py:146-207): cells (nxt, nyt) with
 * nxt = nx + 2 ng, x-major (y contiguous); Bxf (nxt+1, nyt) lower-x faces;
 * Byf (nxt, nyt+1) lower-y faces; corner EMF (nxt+1, nyt+1).
 */
#ifndef HLLD_B200_H
#define HLLD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HLLD_OK 0
#define HLLD_ERR_INVALID (-1)     /* bad argument: shape, enum, null pointer */
#define HLLD_ERR_CUDA (-2)        /* a CUDA launch or runtime call failed */
#define HLLD_ERR_UNSUPPORTED (-3) /* valid but not implemented here */
#define HLLD_ERR_SCRATCH (-4)     /* scratch buffer too small */

enum hlld_precision {
    HLLD_FP64 = 0,       /* FP64 throughout, FMA contraction on */
    HLLD_FP64_EXACT = 1, /* FP64, one rounding per operation (reference order) */
    HLLD_MIXED = 2,      /* FP32 reconstruction/fluxes/update, FP64 C2P, p*, RK state */
    HLLD_FP32 = 3        /* FP32 throughout: every array and every root solve in float
                          * (2D step and tube kernel only) */
};
/* HLLE: hlld.py:1005-1044; HLLD: :1202-1543; HLLC: :1549-1765 (flux plugin
 * and 2D step; the tube kernel and the adjoint take HLLE and HLLD) */
enum hlld_solver { HLLD_SOLVER_HLLE = 0, HLLD_SOLVER_HLLD = 1, HLLD_SOLVER_HLLC = 2 };
enum hlld_limiter {
    HLLD_LIM_PCM = 0, HLLD_LIM_MC = 1, HLLD_LIM_MINMOD = 2,
    HLLD_LIM_WENO5Z = 3, HLLD_LIM_MP5 = 4, HLLD_LIM_MP7 = 5
};
enum hlld_bc { HLLD_BC_OUTFLOW = 0, HLLD_BC_PERIODIC = 1 };

/* C2P status bits (src/physics/c2p.py:290-294, :360-362) */
#define HLLD_ST_BRACKET_OK 1u
#define HLLD_ST_CONVERGED 2u
#define HLLD_ST_V_CLAMPED 4u
#define HLLD_ST_ATMO 8u
#define HLLD_ST_BISECTED 16u
/* Riemann-solver flags (src/physics/hlld.py:1487-1513) */
#define HLLD_RF_WAVE_ORDER_BAD 1u
#define HLLD_RF_BN_ZERO 2u
#define HLLD_RF_FAILED 4u

/* Device-resident counters of one flux sweep: the numbers the reference
 * keeps in hlld.LAST_DIAG (src/physics/hlld.py:1516-1529).  In every form
 * but HLLD_FP64_EXACT the 2D sweep does not solve p* on faces with B_n = 0,
 * whose HLLE fallback result does not depend on it.  Those faces count in n_faces, n_bn_zero
 * and n_failed only, so n_not_converged, n_wave_order_bad, iters_sum_conv,
 * n_conv and max_iters cover the faces that were solved. */
typedef struct {
    unsigned long long n_faces;
    unsigned long long n_not_converged;
    unsigned long long n_wave_order_bad;
    unsigned long long n_bn_zero;
    unsigned long long n_failed;
    unsigned long long iters_sum_conv; /* sum of p* iterations over converged faces */
    unsigned long long n_conv;
    unsigned long long max_iters;
    unsigned long long fd_max_bits; /* bits of max |F_D| (non-negative double) */
} hlld_flux_diag_t;

/* Device-resident counters of one RK step (last stage's sweeps, as the
 * reference's rk_step_ct returns, src/physics/driver2d.py:242-249). */
typedef struct {
    hlld_flux_diag_t sweep[2];
    unsigned long long c2p_not_converged;
    unsigned long long c2p_bisected;
    unsigned long long c2p_atmo;
    unsigned long long c2p_bad_bracket;
    unsigned long long speed_max_bits[2]; /* bits of max(|v_d| + c_f), physical cells */
} hlld_step_diag_t;

/* Face EMF of the constrained transport (src/physics/ct.py:63-88
 * face_emf_x / face_emf_y; run_2d.py --emf-mode). */
enum hlld_emf_mode {
    /* the Riemann solver's transverse-B flux (the reference's default) */
    HLLD_EMF_SOLVER = 0,
    /* the HLL average of the transverse-B flux of the face states
     * (ct.py:91-96 _hll with sweep.py:106-119), whatever the solver */
    HLLD_EMF_HLL = 1
};

typedef struct {
    int32_t nx, ny, ng;
    double dx, dy;
    int32_t bc_x, bc_y;   /* enum hlld_bc */
    int32_t limiter;      /* enum hlld_limiter */
    int32_t solver;       /* enum hlld_solver */
    double gamma;         /* ideal gas: hybrid_eos(K=0, gamma, gamma_th=gamma) */
    double atmo_rho;
    int32_t upwind;       /* Gardiner-Stone upwinded corner EMF (1) or flux-CT (0) */
    int32_t precision;    /* enum hlld_precision */
    int32_t emf_mode;     /* enum hlld_emf_mode (0, the default, is the reference's default) */
} hlld_grid2d_t;

/* State2D (src/physics/state.py:54-74) as device pointers.
 * cons: D, Sx, Sy, Sz, tau, Bz (state.py:41 EVOLVED_KEYS), double.
 * prims: rho, vx, vy, vz, p, eps, Bx, By, Bz (double, float for HLLD_MIXED
 * and HLLD_FP32; in HLLD_FP32 cons, Bxf and Byf are float as well). */
typedef struct {
    void *cons[6];
    void *Bxf;
    void *Byf;
    void *prims[9];
} hlld_state2d_t;

/* How each tube of a batch is stepped (hlld_tubes_t.flavor). */
enum hlld_tube_flavor {
    /* src/physics/driver2d.py:110-156 rk_step on a ny = 1 grid: W v
     * reconstruction with the PCM positivity fallback, SSP-RK2/3 per
     * `scheme`, dt = compute_dt (driver.py:77-127) with the fast speed,
     * stepping while t < tend - 1e-14 */
    HLLD_TUBE_RK_STEP = 0,
    /* src/physics/driver.py:130-236 compute_rhs + rk2_step (the 1D
     * shock-tube driver): all nine primitives reconstructed as they are,
     * Heun RK2 with Bx held, dt = cfl dx (compute_dt with speed_of_light,
     * the driver's default, driver.py:390), stepping while t < tend */
    HLLD_TUBE_DRIVER1D_LIGHT = 1,
    /* as HLLD_TUBE_DRIVER1D_LIGHT with the fast-speed compute_dt
     * (run.dt_speed_of_light = false) */
    HLLD_TUBE_DRIVER1D_CFL = 2
};

/* A batch of independent 1D tubes (the batched-tube workload): tube i has
 * ncells[i] physical cells and ng ghosts per side, occupies cells
 * cell_off[i] .. cell_off[i] + ncells[i] + 2 ng - 1 of the concatenated cell
 * arrays and faces cell_off[i] + i .. cell_off[i] + i + ncells[i] + 2 ng of
 * the face arrays, and has cell width dx[i].  order (may be NULL) is the
 * processing order (e.g. longest tube first).  All pointers are device.
 * resume = 0: the conserved arrays are first computed from the primitives
 * (a fresh run); resume = 1: cons already holds the state that goes with
 * the primitives (a continued run, or the reference's rk2_step, which takes
 * both). */
typedef struct {
    int32_t ntubes, ng;
    const int32_t *ncells;
    const int64_t *cell_off;
    const double *dx;
    const int32_t *order;
    double cfl, tend;
    int32_t max_steps;
    int32_t limiter, solver, scheme, precision;
    double gamma, atmo_rho;
    int32_t flavor;       /* enum hlld_tube_flavor */
    int32_t resume;
} hlld_tubes_t;

int hlld_version(void);
const char *hlld_error_string(int code);
const char *hlld_last_error_detail(void);

/* Replaces src/physics/hlld.py:185-217 primitive_to_conserved.
 * prim: 9 arrays (rho, vx, vy, vz, p, eps, Bx, By, Bz); cons: 8 arrays
 * (D, Sx, Sy, Sz, tau, Bx, By, Bz); double (precision FP64 / FP64_EXACT). */
int hlld_prim_to_cons(int64_t n, const void *const *prim, int precision, void *const *cons,
                      void *stream);

/* Replaces src/physics/c2p.py:313-363 conservative_to_primitive (Kastaun
 * master function, mu_+ bisection, bracketed secant, bisection continuation,
 * atmosphere floor).  status (may be NULL): HLLD_ST_* bits per element. */
int hlld_cons_to_prim(int64_t n, const void *const *cons, double gamma, double atmo_rho,
                      double atmo_eps, int precision, void *const *prim, uint8_t *status,
                      void *stream);

/* Replaces the flux_fn plugin contract flux_fn(sL, sR, eos, idir) ->
 * (F, U, p_star): src/physics/hlld.py:1005-1044 hlle_flux and
 * src/physics/hlld.py:1202-1543 hlld_flux, on n flattened faces.
 * sL, sR: 9 primitive arrays each; F, U: 8 conserved arrays each (U may be
 * NULL); pstar (p* < 0 marks an HLLE fallback face, hlld.py:1531);
 * err / iters / flags may be NULL; diag (may be NULL) is zeroed and filled
 * with the LAST_DIAG counters. */
int hlld_riemann_faces(int64_t n, const void *const *sL, const void *const *sR, int idir,
                       int solver, double gamma, int precision, void *const *F, void *const *U,
                       void *pstar, int32_t *err, int32_t *iters, uint8_t *flags,
                       hlld_flux_diag_t *diag, void *stream);

/* Bytes of scratch hlld_rk_step_ct needs for grid g (face fluxes, corner
 * EMF, the RK stage-0 copy). */
int hlld_step2d_scratch_bytes(const hlld_grid2d_t *g, size_t *bytes);

/* Replaces src/physics/driver2d.py:221-249 rk_step_ct (with ct_stage
 * :162-193, sweep.py:30-135, ct.py:44-199, state.py:77-103 combine and
 * sync_state :196-218): one SSP-RK2 (scheme 2) or RK3 (scheme 3) step with
 * constrained transport, in place on s.  dt is read from dt_dev when it is
 * not NULL (device scalar, lets the step be graph-captured), else dt_host.
 * diag (device, may be NULL) is zeroed and filled. */
int hlld_rk_step_ct(const hlld_grid2d_t *g, const hlld_state2d_t *s, void *scratch,
                    size_t scratch_bytes, double dt_host, const double *dt_dev, int scheme,
                    hlld_step_diag_t *diag, void *stream);

/* No counterpart in the reference.  hlld_rk_step_ct for a state whose arrays
 * are copied between host and device memory on other streams while the step
 * runs (a host-resident state stepped on the device).  cons_in (a
 * cudaEvent_t, may be NULL): the stream waits for it before the first
 * stage's update, the first launch that reads the conserved cell arrays; the
 * primitives and the staggered field are read from the start, so they must
 * be in place before the call's work begins.  cons_out (a cudaEvent_t, may
 * be NULL) is recorded once the conserved arrays and the staggered field,
 * ghosts included, hold the step's result: the last stage's C2P and the
 * ghost fills of the primitives, which follow, read them but do not write
 * them.  The arithmetic is hlld_rk_step_ct's, bit for bit. */
int hlld_rk_step_ct_events(const hlld_grid2d_t *g, const hlld_state2d_t *s, void *scratch,
                           size_t scratch_bytes, double dt_host, const double *dt_dev, int scheme,
                           hlld_step_diag_t *diag, void *stream, void *cons_in, void *cons_out);

/* No counterpart in the reference.  hlld_rk_step_ct for callers that cannot
 * allocate device memory: hosts whose device memory belongs to a pool or
 * allocator they do not control (a framework's caching allocator, a
 * fixed-budget embedded runtime), plugin hosts that hand a solver only its
 * input and output arrays, and time-step loops that cannot afford the
 * device-wide synchronisation a cudaMalloc or cudaFree may cause.  The
 * scratch is a 64 MiB static device array inside the library (held on every
 * GPU that loads the library until the process exits); grids whose
 * hlld_step2d_scratch_bytes exceeds 64 MiB get HLLD_ERR_SCRATCH.  With ng = 2
 * that allows square grids up to 599^2 cells in HLLD_FP64 / HLLD_FP64_EXACT,
 * 708^2 in HLLD_MIXED and 849^2 in HLLD_FP32.  All calls share the one array
 * of a device: calls whose work overlaps on the GPU race, so serialise them
 * on one stream.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress, with that device current) and caches it.
 * Allocates nothing. */
int hlld_rk_step_ct_static(const hlld_grid2d_t *g, const hlld_state2d_t *s, double dt_host,
                           const double *dt_dev, int scheme, hlld_step_diag_t *diag,
                           void *stream);

/* Replaces src/physics/driver2d.py:196-218 sync_state: face BCs, cell BCs,
 * cell-centred B, C2P of the physical cells, primitive BCs, in place.
 * status (nxt*nyt, may be NULL) gets HLLD_ST_* bits of the physical cells. */
int hlld_sync_state(const hlld_grid2d_t *g, const hlld_state2d_t *s, uint8_t *status,
                    hlld_step_diag_t *diag, void *stream);

/* hlld_sync_state that also exposes the C2P roots (device, nxt*nyt doubles,
 * physical cells written): mu_out (may be NULL) receives each cell's root;
 * mu_start (HLLD_MIXED only, may be NULL) holds a previous root of each cell
 * to start the root search from, and is updated.  hlld_rk_step_ct does the
 * same internally in the mixed form: its first stage starts from the step's
 * input primitives (hlld_sync_state_from_prims) and its later stages start
 * from the first stage's roots.  (The reference always solves from the
 * bracket, c2p.py:188-236; a started search reaches the same |f| < 1e-15
 * root, and falls back to the bracketed solve if it does not within eight
 * steps.) */
int hlld_sync_state_roots(const hlld_grid2d_t *g, const hlld_state2d_t *s, uint8_t *status,
                          hlld_step_diag_t *diag, double *mu_out, double *mu_start, void *stream);

/* hlld_sync_state (HLLD_MIXED only) whose C2P starts each physical cell's
 * root search from the primitives the state holds on entry -- Kastaun's
 * root is mu = 1 / (h W), h = 1 + eps + p / rho -- which the call then
 * overwrites with the primitives of the current conserved state.  mu_out
 * (may be NULL) receives the roots.  This is the first RK stage's sync in
 * the mixed hlld_rk_step_ct: the primitives are the step's input, the
 * conserved state the stage's update.  Cells whose primitives are not
 * physical (v >= 1, rho <= 0) and starts that do not converge within eight
 * secant steps take the bracketed solve of c2p.py:188-236. */
int hlld_sync_state_from_prims(const hlld_grid2d_t *g, const hlld_state2d_t *s, uint8_t *status,
                               hlld_step_diag_t *diag, double *mu_out, void *stream);

/* Replaces src/physics/sweep.py:30-119 sweep() in the form the 2D step uses
 * it (reconstruct_prims, normal B taken from the staggered faces
 * sweep.py:82-89, flux_fn on every face, F[B_n] = 0 sweep.py:99-100), fused
 * into one launch.  F: 7 face arrays D, Sx, Sy, Sz, tau, Bz, B_t with B_t =
 * By for axis 0 and Bx for axis 1 ((nxt+1, nyt) or (nxt, nyt+1)); the zero
 * normal-B flux is not stored.  diag (device, required) is zeroed, then
 * receives the LAST_DIAG counters and max |F_D|. */
int hlld_sweep2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, int axis, void *const *F,
                 hlld_flux_diag_t *diag, void *stream);

/* Replaces the rest of ct_stage + combine for RK stage `stage` (0-based) of
 * `scheme` (src/physics/driver2d.py:183-192, :241-246; ct.py:57-185;
 * sweep.py:122-135; state.py:77-103): corner EMF, flux divergence, CT face
 * update and the SSP-RK combine, in place on s.  Fx, Fy: the two sweeps'
 * outputs; Ez: (nxt+1)(nyt+1) work array; U0 (6 cell arrays), Bx0, By0: the
 * RK stage-0 copy, written at stage 0 and read afterwards; diag: the step
 * counters whose sweep[0/1].fd_max_bits set the upwind deadband (ct.py:114). */
int hlld_ct_update2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, void *const *Fx,
                     void *const *Fy, void *Ez, void *const *U0, void *Bx0, void *By0,
                     const hlld_step_diag_t *diag, int stage, int scheme, double dt_host,
                     const double *dt_dev, void *stream);

/* Replaces src/physics/tube_seed.py:93-144 run_tubes for the batched-tube
 * workload, with a dt per tube: every tube runs src/physics/driver2d.py:110-156
 * rk_step on a ny = 1 grid (x sweep only -- the y sweep of a ny = 1 grid
 * contributes exactly zero), dt from src/physics/driver.py:77-127
 * compute_dt each step, until tend or max_steps (flavor HLLD_TUBE_RK_STEP),
 * or the 1D driver's loop (src/physics/driver.py:388-412 around rk2_step,
 * the other flavors), in ONE persistent launch of
 * `blocks` CTAs of `threads` threads (a multiple of 32, at most 512; 0 =
 * library defaults: 512 threads, one CTA per SM).  prims (9
 * arrays, ghosts filled) are read and updated in place; cons (8), U0 (8
 * cell arrays) and F (8 face arrays, slot Bx unused) are work arrays;
 * t_out / steps_out get each tube's final time and step count; next is one
 * device unsigned int (the work counter, zeroed by the call).  Primitives
 * and F are float for HLLD_MIXED and HLLD_FP32, double otherwise. */
int hlld_tubes_run(const hlld_tubes_t *b, void *const *cons, void *const *prims,
                   void *const *U0, void *const *F, double *t_out, int32_t *steps_out,
                   unsigned int *next, int threads, int blocks, void *stream);

/* The adjoint split in two, for checkpointed runs that recompute a segment
 * once: hlld_adjoint_record_step advances s by one step exactly as
 * hlld_rk_step_ct does and writes the step's tape (the stage-1 and stage-2
 * inputs and, per stage, F_D, the sweep counters and each face's p* and
 * HLLE fallback); hlld_adjoint_reverse_step then maps lambda of the output
 * to lambda of the input without recomputing the forward.  Sizes from
 * hlld_adjoint_tape_bytes (one tape per recorded step; the scratch can be
 * shared by all calls on one stream).  No counterpart in the reference.
 * FP64, HLLE or HLLD; buffers 256-byte aligned. */
int hlld_adjoint_tape_bytes(const hlld_grid2d_t *g, size_t *tape_bytes, size_t *scratch_bytes);
int hlld_adjoint_record_step(const hlld_grid2d_t *g, const hlld_state2d_t *s, double dt,
                             int scheme, void *tape, size_t tape_bytes, void *scratch,
                             size_t scratch_bytes, void *stream);
int hlld_adjoint_reverse_step(const hlld_grid2d_t *g, const hlld_state2d_t *s_in,
                              const hlld_state2d_t *s_out, double dt, int scheme, const void *tape,
                              size_t tape_bytes, const hlld_state2d_t *lam, void *scratch,
                              size_t scratch_bytes, void *stream);

/* Reverse of src/physics/hlld.py:185-217 primitive_to_conserved on n
 * elements (FP64): lam_prim[9] = (d cons / d prim)^T lam_cons[8], with eps
 * an independent input as it is there.  Entries of lam_cons may be NULL
 * (zero).  For gradients of an objective with respect to initial data. */
int hlld_prim_to_cons_vjp(int64_t n, const void *const *prim, const void *const *lam_cons,
                          void *const *lam_prim, void *stream);

/* Bytes of scratch hlld_adjoint_rk_step_ct needs for this grid (FP64 only). */
int hlld_adjoint_scratch_bytes(const hlld_grid2d_t *g, size_t *bytes);

/* Discrete adjoint of one hlld_rk_step_ct step.  No counterpart in the
 * reference, whose gradients would come from torch autograd through
 * src/physics/driver2d.py:221-249 rk_step_ct; this is that step's
 * transpose with its dt held fixed.  s_in is the step's input state and
 * s_out the output the forward step made from it with dt.  lam (device
 * arrays shaped like a state: cons[6], Bxf, Byf, prims[9], double) holds
 * on entry the gradient of the objective with respect to the output state
 * and on return its gradient with respect to the input state's cons and
 * faces (lam.prims returns zeroed: the input primitives are a function of
 * them).  Discrete decisions (limiter branches, HLLD region and fallback,
 * upwind signs, clamps) are frozen at their forward outcome; p* and the C2P
 * root are differentiated by the implicit-function theorem.  g->precision
 * must be HLLD_FP64; scratch (256-byte aligned) of
 * hlld_adjoint_scratch_bytes bytes. */
int hlld_adjoint_rk_step_ct(const hlld_grid2d_t *g, const hlld_state2d_t *s_in,
                            const hlld_state2d_t *s_out, double dt, int scheme,
                            const hlld_state2d_t *lam, void *scratch, size_t scratch_bytes,
                            void *stream);

/* Replaces src/physics/driver2d.py:52-82 compute_dt_2d: writes
 * dt = cfl / (max(|vx|+cf)/dx + max(|vy|+cf)/dy) to dt_dev (device double);
 * work (device, >= 2 unsigned long long) holds the running maxima. */
int hlld_compute_dt_2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, double cfl,
                       double *dt_dev, unsigned long long *work, void *stream);

#ifdef __cplusplus
}
#endif
#endif
