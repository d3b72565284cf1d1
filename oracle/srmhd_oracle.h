/*
 * CPU oracle for the SRMHD finite-volume step -- TEST INFRASTRUCTURE ONLY.
 *
 * A scalar, per-element C restatement of kemi2805/HLLD-AI's FP64 PyTorch
 * hot path (src/physics/{eos,hlld,c2p,reconstruction,sweep,ct,driver2d,
 * driver,state,grid}.py).  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it, and only as
 * the checker or the timed CPU baseline.  The product (hlld_ai_b200) never
 * links or calls it.
 *
 * Semantics pinned here (and the two known differences from the PyTorch
 * reference, both last-bit level):
 *   - every elementary operation is performed in the reference's order,
 *     one IEEE-754 rounding per operation (build with -ffp-contract=off);
 *   - sqrt is the correctly rounded libm sqrt.  torch's CPU sqrt (MKL vector
 *     math) is faithfully but not correctly rounded: about 1% of its results
 *     are one ulp away from this one;
 *   - iterations stop per element.  The reference's Kastaun secant
 *     (c2p.py:214-217) runs until EVERY cell of its batch has converged and
 *     keeps stepping converged cells meanwhile, so a reference result
 *     depends on its batch mates at round-off level; this oracle returns the
 *     reference's answer for a batch of one element.  All other reference
 *     loops (mu_+ bisection c2p.py:174-182, p* secant hlld.py:707-737 with
 *     frozen lanes, bracket widening hlld.py:1314-1321, bisection
 *     continuation c2p.py:257-262) are batch independent and reproduced
 *     exactly.
 *   - equation of state: the hot path's hybrid_eos(K=0, gamma, gamma_th=
 *     gamma) (scripts/run_2d.py:213), i.e. an ideal gas, written with the
 *     reference's operation order (eos.py:32-76).
 */
#ifndef SRMHD_ORACLE_H
#define SRMHD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* primitive component order (hlld.py:8-9) */
enum { ORC_RHO = 0, ORC_VX, ORC_VY, ORC_VZ, ORC_P, ORC_EPS, ORC_PBX, ORC_PBY, ORC_PBZ, ORC_NPRIM };
/* conserved component order (hlld.py:11-12) */
enum { ORC_D = 0, ORC_SX, ORC_SY, ORC_SZ, ORC_TAU, ORC_BX, ORC_BY, ORC_BZ, ORC_NCONS };

/* C2P status bits (c2p.py:290-294, :360-362) */
#define ORC_ST_BRACKET_OK 1u
#define ORC_ST_CONVERGED 2u
#define ORC_ST_V_CLAMPED 4u
#define ORC_ST_ATMO 8u
#define ORC_ST_BISECTED 16u

/* Riemann-solver flags (hlld.py:1487-1513) */
#define ORC_RF_WAVE_ORDER_BAD 1u
#define ORC_RF_BN_ZERO 2u
#define ORC_RF_FAILED 4u

enum { ORC_SOLVER_HLLE = 0, ORC_SOLVER_HLLD = 1, ORC_SOLVER_HLLC = 2 };
enum { ORC_LIM_PCM = 0, ORC_LIM_MC = 1, ORC_LIM_MINMOD = 2, ORC_LIM_WENO5Z = 3, ORC_LIM_MP5 = 4, ORC_LIM_MP7 = 5 };
enum { ORC_BC_OUTFLOW = 0, ORC_BC_PERIODIC = 1 };

int orc_version(void);
void orc_set_threads(int n);

/* hlld.py:185-217 primitive_to_conserved */
void orc_prim_to_cons(int64_t n, const double *const *prim, double *const *cons);

/* c2p.py:313-363 conservative_to_primitive; status may be NULL */
void orc_cons_to_prim(int64_t n, const double *const *cons, double gamma, double atmo_rho,
                      double atmo_eps, double *const *prim, uint8_t *status);

/* hlld.py:1005-1044 hlle_flux / hlld.py:1202-1543 hlld_flux on n faces.
 * err, iters, flags may be NULL. */
void orc_riemann(int64_t n, const double *const *sL, const double *const *sR, int idir,
                 int solver, double gamma, double *const *F, double *const *U,
                 double *pstar, int32_t *err, int32_t *iters, uint8_t *flags);

/* reconstruction.py:239-264 reconstruct() of one variable along one axis of
 * an (n0, n1) row-major array; QL, QR are (n0+1, n1) or (n0, n1+1). */
void orc_reconstruct(const double *q, int n0, int n1, int axis, int limiter, double *QL,
                     double *QR);

/* reconstruction.py:272-338 reconstruct_prims (vel_var "Wv" when wv != 0).
 * prim: the 9 primitives (eps unused), each (n0, n1).  L, R: 9 face arrays
 * each, in primitive order (eps recomputed from p, rho). */
void orc_reconstruct_prims(const double *const *prim, int n0, int n1, int axis, int limiter,
                           int wv, double gamma, double *const *L, double *const *R);

typedef struct {
    int nx, ny, ng;
    double dx, dy;
    int bc_x, bc_y;
    int limiter;
    int solver;
    double gamma;
    double atmo_rho;
    int upwind;
    /* face EMF (ct.py:63-88): 0 "solver", the Riemann solver's transverse-B
     * flux; 1 "hll", the HLL average of the transverse-B flux from the face
     * states (sweep.py:106-119) */
    int emf_mode;
} orc_grid2d;

typedef struct {
    int64_t n_faces[2];
    int64_t n_not_converged[2];
    int64_t n_wave_order_bad[2];
    int64_t n_bn_zero[2];
    int64_t n_failed[2];
    int64_t iters_sum_conv[2]; /* sum of iterations over converged faces */
    int64_t n_conv[2];
    int64_t max_iters[2];
    double fd_max[2]; /* max |F_D| of each sweep (ct.py:114) */
} orc_step_diag;

/* driver2d.py:196-218 sync_state: face BC, cell BC, cell-centred B, C2P,
 * primitive BC.  cons: 6 arrays D, Sx, Sy, Sz, tau, Bz (state.py:41).
 * prim: 9 arrays.  status (nxt*nyt) may be NULL. */
void orc_sync_state(const orc_grid2d *g, double *const *cons, double *Bxf, double *Byf,
                    double *const *prim, uint8_t *status);

/* driver2d.py:221-249 rk_step_ct: one SSP-RK2/3 step with CT; the state
 * (cons, faces, prims) is updated in place.  diag may be NULL (it reports
 * the last stage's sweeps, as the reference's returned diag does). */
int orc_rk_step_ct(const orc_grid2d *g, double dt, int scheme, double *const *cons,
                   double *Bxf, double *Byf, double *const *prim, orc_step_diag *diag);

/* driver2d.py:52-82 compute_dt_2d */
double orc_compute_dt_2d(const orc_grid2d *g, const double *const *prim, double cfl);

/* ct.py:119-177 corner_emf on (n0, n1) cells; Ez is (n0+1, n1+1) */
void orc_corner_emf(int n0, int n1, const double *Ec, const double *Efx, const double *Efy,
                    const double *Fx_rho, const double *Fy_rho, int upwind, double *Ez);

/* driver.py:192-236 rk2_step of the 1D shock-tube driver (outflow, Bx
 * frozen, all nine primitives reconstructed with `limiter`).  prim/cons:
 * 9 / 8 arrays of ntotal = ncells + 2 ng. */
void orc_rk2_step_1d(int ncells, int ng, double dx, double dt, int limiter, int solver,
                     double gamma, double atmo_rho, double *const *cons, double *const *prim);

/* One 1D tube run to tend (the batched-tube workload): driver2d.py:110-156
 * rk_step (no CT) on a ny = 1 grid, whose y sweep contributes exactly zero,
 * so only the x sweep is formed: reconstruct_prims of all eight work
 * variables (W v), flux_fn with idir 0, F[Bx] = 0, all eight conserved
 * variables evolved, outflow BCs, C2P, P[B] = U[B].  dt per step is
 * driver.py:77-127 compute_dt (max |vx| + c_f over the physical cells),
 * capped at tend - t.  prim: 9 arrays of L + 2 ng cells (ghosts filled),
 * updated in place.  Returns the number of steps taken. */
int orc_tube_run(int L, int ng, double dx, double cfl, double tend, int max_steps, int limiter,
                 int solver, double gamma, double atmo_rho, int scheme, double *const *prim,
                 double *t_out);

/* The same with the stepping flavor and the conserved state exposed:
 * flavor ORC_TUBE_RK_STEP is orc_tube_run; ORC_TUBE_DRIVER1D_LIGHT /
 * ORC_TUBE_DRIVER1D_CFL run driver.py:388-412 (rk2_step = orc_rk2_step_1d
 * each step, dt = cfl dx or compute_dt, while t < tend).  cons (8 arrays of
 * L + 2 ng, may be NULL): with resume = 1 it is the starting conserved
 * state (else it is computed from prim); on return it holds the final one. */
enum { ORC_TUBE_RK_STEP = 0, ORC_TUBE_DRIVER1D_LIGHT = 1, ORC_TUBE_DRIVER1D_CFL = 2 };
int orc_tube_run_ex(int L, int ng, double dx, double cfl, double tend, int max_steps, int limiter,
                    int solver, double gamma, double atmo_rho, int scheme, int flavor, int resume,
                    double *const *cons, double *const *prim, double *t_out);

#ifdef __cplusplus
}
#endif
#endif
