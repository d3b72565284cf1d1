// extern "C" entry points of libhlld_b200.so (declared in include/hlld_b200.h):
// argument checks, scratch layout and dispatch to the arithmetic variant.
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "variants.h"

namespace {

thread_local char g_detail[512] = "";

int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_detail, sizeof g_detail, fmt, ap);
    va_end(ap);
    return code;
}

// launch errors only (a kernel's own faults surface at the next sync)
int check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(HLLD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return HLLD_OK;
}

bool fp64_precision(int precision) {
    return precision == HLLD_FP64 || precision == HLLD_FP64_EXACT;
}

bool step_precision(int precision) {
    return fp64_precision(precision) || precision == HLLD_MIXED || precision == HLLD_FP32;
}

// bytes of one element of the step's primitive, flux and EMF arrays
size_t real_bytes(int precision) { return (precision == HLLD_MIXED || precision == HLLD_FP32) ? 4 : 8; }
// bytes of one element of the conserved state, the staggered field and the
// RK stage-0 copy
size_t state_bytes(int precision) { return precision == HLLD_FP32 ? 4 : 8; }

int check_grid(const hlld_grid2d_t *g) {
    if (!g) return fail(HLLD_ERR_INVALID, "grid is NULL");
    if (g->nx < 1 || g->ny < 1) return fail(HLLD_ERR_INVALID, "nx, ny must be >= 1");
    if (g->ng < 1) return fail(HLLD_ERR_INVALID, "ng must be >= 1");
    if (g->nx <= g->ng || g->ny <= g->ng)
        return fail(HLLD_ERR_INVALID, "nx and ny must exceed ng (periodic ghost sources)");
    if ((int64_t)(g->nx + 2 * g->ng + 1) * (g->ny + 2 * g->ng + 1) > (int64_t)1 << 31)
        return fail(HLLD_ERR_INVALID, "grid too large for 32-bit face indexing");
    if (g->bc_x < 0 || g->bc_x > 1 || g->bc_y < 0 || g->bc_y > 1)
        return fail(HLLD_ERR_INVALID, "bc must be HLLD_BC_OUTFLOW or HLLD_BC_PERIODIC");
    if (g->limiter < 0 || g->limiter > HLLD_LIM_MP7) return fail(HLLD_ERR_INVALID, "bad limiter");
    static const int need[6] = {1, 1, 1, 2, 2, 3};  // stencil half-width per limiter
    if (g->ng < need[g->limiter])
        return fail(HLLD_ERR_INVALID, "ng = %d is too narrow for the limiter (needs %d)", g->ng,
                    need[g->limiter]);
    if (g->solver != HLLD_SOLVER_HLLE && g->solver != HLLD_SOLVER_HLLD && g->solver != HLLD_SOLVER_HLLC)
        return fail(HLLD_ERR_INVALID, "solver must be HLLE, HLLD or HLLC");
    if (!(g->gamma > 1.0)) return fail(HLLD_ERR_INVALID, "gamma must be > 1");
    if (!(g->dx > 0.0) || !(g->dy > 0.0)) return fail(HLLD_ERR_INVALID, "dx, dy must be > 0");
    if (!step_precision(g->precision))
        return fail(HLLD_ERR_UNSUPPORTED, "precision %d not available for the 2D step", g->precision);
    if (g->emf_mode != HLLD_EMF_SOLVER && g->emf_mode != HLLD_EMF_HLL)
        return fail(HLLD_ERR_INVALID, "emf_mode must be HLLD_EMF_SOLVER or HLLD_EMF_HLL");
    return HLLD_OK;
}

int check_state(const hlld_state2d_t *s) {
    if (!s) return fail(HLLD_ERR_INVALID, "state is NULL");
    for (int k = 0; k < 6; ++k)
        if (!s->cons[k]) return fail(HLLD_ERR_INVALID, "state.cons[%d] is NULL", k);
    for (int k = 0; k < 9; ++k)
        if (!s->prims[k]) return fail(HLLD_ERR_INVALID, "state.prims[%d] is NULL", k);
    if (!s->Bxf || !s->Byf) return fail(HLLD_ERR_INVALID, "state faces are NULL");
    return HLLD_OK;
}

constexpr size_t kAlign = 256;
size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// scratch layout of one 2D step; returns the byte count and fills sc when base != NULL
size_t layout_scratch(const hlld_grid2d_t *g, char *base, hlld::Scratch2D *sc) {
    const size_t nxt = g->nx + 2 * g->ng, nyt = g->ny + 2 * g->ng;
    const size_t nfx = (nxt + 1) * nyt, nfy = nxt * (nyt + 1), ncr = (nxt + 1) * (nyt + 1),
                 nc = nxt * nyt;
    const size_t rb = real_bytes(g->precision), sb = state_bytes(g->precision);
    size_t off = 0;
    auto take = [&](size_t count, size_t elem) -> void * {
        void *p = base ? (void *)(base + off) : nullptr;
        off += align_up(count * elem);
        return p;
    };
    hlld::Scratch2D s{};
    for (int k = 0; k < 7; ++k) s.Fx[k] = take(nfx, rb);
    for (int k = 0; k < 7; ++k) s.Fy[k] = take(nfy, rb);
    s.Ez = take(ncr, rb);
    for (int k = 0; k < 6; ++k) s.U0[k] = (double *)take(nc, sb);
    s.Bx0 = (double *)take(nfx, sb);
    s.By0 = (double *)take(nfy, sb);
    s.diag = base ? (hlld_step_diag_t *)(base + off) : nullptr;
    off += align_up(sizeof(hlld_step_diag_t));
    // mixed form: the C2P roots of the step's first stage (warm start)
    s.mu_warm = g->precision == HLLD_MIXED ? (double *)take(nc, 8) : nullptr;
    if (sc) *sc = s;
    return off;
}

}  // namespace

int hlld::report_error(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_detail, sizeof g_detail, fmt, ap);
    va_end(ap);
    return code;
}

extern "C" {

int hlld_version(void) { return 1; }

const char *hlld_error_string(int code) {
    switch (code) {
    case HLLD_OK: return "ok";
    case HLLD_ERR_INVALID: return "invalid argument";
    case HLLD_ERR_CUDA: return "CUDA error";
    case HLLD_ERR_UNSUPPORTED: return "unsupported";
    case HLLD_ERR_SCRATCH: return "scratch buffer too small";
    default: return "unknown error";
    }
}

const char *hlld_last_error_detail(void) { return g_detail; }

int hlld_prim_to_cons(int64_t n, const void *const *prim, int precision, void *const *cons,
                      void *stream) {
    if (n < 0 || !prim || !cons) return fail(HLLD_ERR_INVALID, "bad arguments");
    if (!fp64_precision(precision)) return fail(HLLD_ERR_UNSUPPORTED, "precision %d", precision);
    if (n == 0) return HLLD_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == HLLD_FP64_EXACT) hlld::v_exact::launch_prim_to_cons(n, prim, cons, st);
    else hlld::v_fp64::launch_prim_to_cons(n, prim, cons, st);
    return check_launch("prim_to_cons");
}

int hlld_cons_to_prim(int64_t n, const void *const *cons, double gamma, double atmo_rho,
                      double atmo_eps, int precision, void *const *prim, uint8_t *status,
                      void *stream) {
    if (n < 0 || !cons || !prim) return fail(HLLD_ERR_INVALID, "bad arguments");
    if (!(gamma > 1.0)) return fail(HLLD_ERR_INVALID, "gamma must be > 1");
    if (!fp64_precision(precision)) return fail(HLLD_ERR_UNSUPPORTED, "precision %d", precision);
    if (n == 0) return HLLD_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == HLLD_FP64_EXACT)
        hlld::v_exact::launch_cons_to_prim(n, cons, gamma, atmo_rho, atmo_eps, prim, status, st);
    else
        hlld::v_fp64::launch_cons_to_prim(n, cons, gamma, atmo_rho, atmo_eps, prim, status, st);
    return check_launch("cons_to_prim");
}

int hlld_riemann_faces(int64_t n, const void *const *sL, const void *const *sR, int idir,
                       int solver, double gamma, int precision, void *const *F, void *const *U,
                       void *pstar, int32_t *err, int32_t *iters, uint8_t *flags,
                       hlld_flux_diag_t *diag, void *stream) {
    if (n < 0 || !sL || !sR || !F || !pstar) return fail(HLLD_ERR_INVALID, "bad arguments");
    if (idir < 0 || idir > 2) return fail(HLLD_ERR_INVALID, "idir must be 0, 1 or 2");
    if (solver != HLLD_SOLVER_HLLE && solver != HLLD_SOLVER_HLLD && solver != HLLD_SOLVER_HLLC)
        return fail(HLLD_ERR_INVALID, "solver must be HLLE, HLLD or HLLC");
    if (!(gamma > 1.0)) return fail(HLLD_ERR_INVALID, "gamma must be > 1");
    if (!fp64_precision(precision)) return fail(HLLD_ERR_UNSUPPORTED, "precision %d", precision);
    cudaStream_t st = (cudaStream_t)stream;
    if (diag && cudaMemsetAsync(diag, 0, sizeof(hlld_flux_diag_t), st) != cudaSuccess)
        return check_launch("riemann_faces diag reset");
    if (n == 0) return HLLD_OK;
    if (precision == HLLD_FP64_EXACT)
        hlld::v_exact::launch_riemann_faces(n, sL, sR, idir, solver, gamma, F, U, pstar, err, iters,
                                            flags, diag, st);
    else
        hlld::v_fp64::launch_riemann_faces(n, sL, sR, idir, solver, gamma, F, U, pstar, err, iters,
                                           flags, diag, st);
    return check_launch("riemann_faces");
}

int hlld_step2d_scratch_bytes(const hlld_grid2d_t *g, size_t *bytes) {
    int rc = check_grid(g);
    if (rc) return rc;
    if (!bytes) return fail(HLLD_ERR_INVALID, "bytes is NULL");
    *bytes = layout_scratch(g, nullptr, nullptr);
    return HLLD_OK;
}

int hlld_rk_step_ct(const hlld_grid2d_t *g, const hlld_state2d_t *s, void *scratch,
                    size_t scratch_bytes, double dt_host, const double *dt_dev, int scheme,
                    hlld_step_diag_t *diag, void *stream) {
    return hlld_rk_step_ct_events(g, s, scratch, scratch_bytes, dt_host, dt_dev, scheme, diag,
                                  stream, nullptr, nullptr);
}

int hlld_rk_step_ct_events(const hlld_grid2d_t *g, const hlld_state2d_t *s, void *scratch,
                           size_t scratch_bytes, double dt_host, const double *dt_dev, int scheme,
                           hlld_step_diag_t *diag, void *stream, void *cons_in, void *cons_out) {
    int rc = check_grid(g);
    if (rc) return rc;
    if ((rc = check_state(s))) return rc;
    if (scheme != 2 && scheme != 3) return fail(HLLD_ERR_INVALID, "scheme must be 2 or 3");
    if (!scratch) return fail(HLLD_ERR_INVALID, "scratch is NULL");
    if ((uintptr_t)scratch % kAlign) return fail(HLLD_ERR_INVALID, "scratch must be 256-byte aligned");
    hlld::Scratch2D sc;
    size_t need = layout_scratch(g, (char *)scratch, &sc);
    if (scratch_bytes < need)
        return fail(HLLD_ERR_SCRATCH, "scratch has %zu bytes, the step needs %zu", scratch_bytes, need);
    if (!dt_dev && !(dt_host == dt_host)) return fail(HLLD_ERR_INVALID, "dt is NaN");
    hlld_step_diag_t *d = diag ? diag : sc.diag;
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t ein = (cudaEvent_t)cons_in, eout = (cudaEvent_t)cons_out;
    if (g->precision == HLLD_FP64_EXACT)
        hlld::v_exact::launch_rk_step_ct(g, s, sc, dt_host, dt_dev, scheme, d, st, ein, eout);
    else if (g->precision == HLLD_MIXED)
        hlld::v_mixed::launch_rk_step_ct(g, s, sc, dt_host, dt_dev, scheme, d, st, ein, eout);
    else if (g->precision == HLLD_FP32)
        hlld::v_fp32::launch_rk_step_ct(g, s, sc, dt_host, dt_dev, scheme, d, st, ein, eout);
    else
        hlld::v_fp64::launch_rk_step_ct(g, s, sc, dt_host, dt_dev, scheme, d, st, ein, eout);
    return check_launch("rk_step_ct");
}

int hlld_sync_state(const hlld_grid2d_t *g, const hlld_state2d_t *s, uint8_t *status,
                    hlld_step_diag_t *diag, void *stream) {
    int rc = check_grid(g);
    if (rc) return rc;
    if ((rc = check_state(s))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (diag && cudaMemsetAsync(diag, 0, sizeof(hlld_step_diag_t), st) != cudaSuccess)
        return check_launch("sync_state diag reset");
    if (g->precision == HLLD_FP64_EXACT)
        hlld::v_exact::launch_sync_state(g, s, status, diag, st);
    else if (g->precision == HLLD_MIXED)
        hlld::v_mixed::launch_sync_state(g, s, status, diag, st);
    else if (g->precision == HLLD_FP32)
        hlld::v_fp32::launch_sync_state(g, s, status, diag, st);
    else
        hlld::v_fp64::launch_sync_state(g, s, status, diag, st);
    return check_launch("sync_state");
}

int hlld_sync_state_roots(const hlld_grid2d_t *g, const hlld_state2d_t *s, uint8_t *status,
                          hlld_step_diag_t *diag, double *mu_out, double *mu_start, void *stream) {
    int rc = check_grid(g);
    if (rc) return rc;
    if ((rc = check_state(s))) return rc;
    if (mu_start && g->precision != HLLD_MIXED)
        return fail(HLLD_ERR_UNSUPPORTED, "the C2P warm start belongs to the mixed form");
    cudaStream_t st = (cudaStream_t)stream;
    if (diag && cudaMemsetAsync(diag, 0, sizeof(hlld_step_diag_t), st) != cudaSuccess)
        return check_launch("sync_state diag reset");
    if (g->precision == HLLD_FP64_EXACT)
        hlld::v_exact::launch_sync_state(g, s, status, diag, st, mu_out, nullptr);
    else if (g->precision == HLLD_MIXED)
        hlld::v_mixed::launch_sync_state(g, s, status, diag, st, mu_out, mu_start);
    else if (g->precision == HLLD_FP32)
        hlld::v_fp32::launch_sync_state(g, s, status, diag, st, mu_out, mu_start);
    else
        hlld::v_fp64::launch_sync_state(g, s, status, diag, st, mu_out, nullptr);
    return check_launch("sync_state_roots");
}

int hlld_sync_state_from_prims(const hlld_grid2d_t *g, const hlld_state2d_t *s, uint8_t *status,
                               hlld_step_diag_t *diag, double *mu_out, void *stream) {
    int rc = check_grid(g);
    if (rc) return rc;
    if ((rc = check_state(s))) return rc;
    if (g->precision != HLLD_MIXED)
        return fail(HLLD_ERR_UNSUPPORTED, "the C2P warm start belongs to the mixed form");
    cudaStream_t st = (cudaStream_t)stream;
    if (diag && cudaMemsetAsync(diag, 0, sizeof(hlld_step_diag_t), st) != cudaSuccess)
        return check_launch("sync_state diag reset");
    hlld::v_mixed::launch_sync_state(g, s, status, diag, st, mu_out, nullptr, true);
    return check_launch("sync_state_from_prims");
}

int hlld_sweep2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, int axis, void *const *F,
                 hlld_flux_diag_t *diag, void *stream) {
    int rc = check_grid(g);
    if (rc) return rc;
    if ((rc = check_state(s))) return rc;
    if (axis != 0 && axis != 1) return fail(HLLD_ERR_INVALID, "axis must be 0 or 1");
    if (!F || !diag) return fail(HLLD_ERR_INVALID, "F and diag are required");
    for (int k = 0; k < 7; ++k)
        if (!F[k]) return fail(HLLD_ERR_INVALID, "F[%d] is NULL", k);
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(diag, 0, sizeof(hlld_flux_diag_t), st) != cudaSuccess)
        return check_launch("sweep2d diag reset");
    if (g->precision == HLLD_FP64_EXACT)
        hlld::v_exact::launch_sweep2d(g, s, axis, F, diag, st);
    else if (g->precision == HLLD_MIXED)
        hlld::v_mixed::launch_sweep2d(g, s, axis, F, diag, st);
    else if (g->precision == HLLD_FP32)
        hlld::v_fp32::launch_sweep2d(g, s, axis, F, diag, st);
    else
        hlld::v_fp64::launch_sweep2d(g, s, axis, F, diag, st);
    return check_launch("sweep2d");
}

int hlld_ct_update2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, void *const *Fx,
                     void *const *Fy, void *Ez, void *const *U0, void *Bx0, void *By0,
                     const hlld_step_diag_t *diag, int stage, int scheme, double dt_host,
                     const double *dt_dev, void *stream) {
    int rc = check_grid(g);
    if (rc) return rc;
    if ((rc = check_state(s))) return rc;
    if (scheme != 2 && scheme != 3) return fail(HLLD_ERR_INVALID, "scheme must be 2 or 3");
    if (stage < 0 || stage >= scheme) return fail(HLLD_ERR_INVALID, "stage out of range");
    if (!Fx || !Fy || !Ez || !U0 || !Bx0 || !By0 || !diag)
        return fail(HLLD_ERR_INVALID, "NULL array argument");
    hlld::Scratch2D sc{};
    for (int k = 0; k < 7; ++k) {
        sc.Fx[k] = Fx[k];
        sc.Fy[k] = Fy[k];
        if (!sc.Fx[k] || !sc.Fy[k]) return fail(HLLD_ERR_INVALID, "flux array %d is NULL", k);
    }
    for (int k = 0; k < 6; ++k) {
        sc.U0[k] = (double *)U0[k];
        if (!sc.U0[k]) return fail(HLLD_ERR_INVALID, "U0[%d] is NULL", k);
    }
    sc.Ez = Ez;
    sc.Bx0 = (double *)Bx0;
    sc.By0 = (double *)By0;
    cudaStream_t st = (cudaStream_t)stream;
    if (g->precision == HLLD_FP64_EXACT)
        hlld::v_exact::launch_ct_update2d(g, s, sc, diag, stage, scheme, dt_host, dt_dev, st);
    else if (g->precision == HLLD_MIXED)
        hlld::v_mixed::launch_ct_update2d(g, s, sc, diag, stage, scheme, dt_host, dt_dev, st);
    else if (g->precision == HLLD_FP32)
        hlld::v_fp32::launch_ct_update2d(g, s, sc, diag, stage, scheme, dt_host, dt_dev, st);
    else
        hlld::v_fp64::launch_ct_update2d(g, s, sc, diag, stage, scheme, dt_host, dt_dev, st);
    return check_launch("ct_update2d");
}

int hlld_tubes_run(const hlld_tubes_t *b, void *const *cons, void *const *prims,
                   void *const *U0, void *const *F, double *t_out, int32_t *steps_out,
                   unsigned int *next, int threads, int blocks, void *stream) {
    if (!b) return fail(HLLD_ERR_INVALID, "batch is NULL");
    if (b->ntubes < 0) return fail(HLLD_ERR_INVALID, "ntubes < 0");
    if (b->ntubes == 0) return HLLD_OK;
    if (!b->ncells || !b->cell_off || !b->dx || !cons || !prims || !U0 || !F || !t_out ||
        !steps_out || !next)
        return fail(HLLD_ERR_INVALID, "NULL array argument");
    if (b->limiter < 0 || b->limiter > HLLD_LIM_MP7) return fail(HLLD_ERR_INVALID, "bad limiter");
    static const int need[6] = {1, 1, 1, 2, 2, 3};
    if (b->ng < need[b->limiter]) return fail(HLLD_ERR_INVALID, "ng too narrow for the limiter");
    if (b->solver != HLLD_SOLVER_HLLE && b->solver != HLLD_SOLVER_HLLD)
        return fail(HLLD_ERR_INVALID, "the tube kernel takes HLLE or HLLD");
    if (b->scheme != 2 && b->scheme != 3) return fail(HLLD_ERR_INVALID, "scheme must be 2 or 3");
    if (b->flavor < HLLD_TUBE_RK_STEP || b->flavor > HLLD_TUBE_DRIVER1D_CFL)
        return fail(HLLD_ERR_INVALID, "unknown tube flavor %d", b->flavor);
    if (!(b->gamma > 1.0) || !(b->cfl > 0.0)) return fail(HLLD_ERR_INVALID, "gamma, cfl");
    if (!step_precision(b->precision)) return fail(HLLD_ERR_UNSUPPORTED, "precision %d", b->precision);
    for (int k = 0; k < 8; ++k)
        if (!cons[k] || !U0[k] || (k != 5 && !F[k]))
            return fail(HLLD_ERR_INVALID, "NULL work array %d", k);
    for (int k = 0; k < 9; ++k)
        if (!prims[k]) return fail(HLLD_ERR_INVALID, "prims[%d] is NULL", k);
    if (threads <= 0) threads = 512;
    if (threads % 32 || threads > 512)
        return fail(HLLD_ERR_INVALID, "threads must be a multiple of 32, at most 512");
    if (blocks <= 0) {
        // as many CTAs as fit at 128 registers per thread: 512 threads per SM
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        blocks = sms * (512 / threads > 0 ? 512 / threads : 1);
    }
    if (blocks > b->ntubes) blocks = b->ntubes;
    cudaStream_t st = (cudaStream_t)stream;
    if (b->precision == HLLD_FP64_EXACT)
        hlld::v_exact::launch_tubes_run(b, cons, prims, U0, F, t_out, steps_out, next, threads, blocks, st);
    else if (b->precision == HLLD_MIXED)
        hlld::v_mixed::launch_tubes_run(b, cons, prims, U0, F, t_out, steps_out, next, threads, blocks, st);
    else if (b->precision == HLLD_FP32)
        hlld::v_fp32::launch_tubes_run(b, cons, prims, U0, F, t_out, steps_out, next, threads, blocks, st);
    else
        hlld::v_fp64::launch_tubes_run(b, cons, prims, U0, F, t_out, steps_out, next, threads, blocks, st);
    return check_launch("tubes_run");
}

int hlld_compute_dt_2d(const hlld_grid2d_t *g, const hlld_state2d_t *s, double cfl,
                       double *dt_dev, unsigned long long *work, void *stream) {
    int rc = check_grid(g);
    if (rc) return rc;
    if ((rc = check_state(s))) return rc;
    if (!dt_dev || !work) return fail(HLLD_ERR_INVALID, "dt_dev and work must be device pointers");
    if (!(cfl > 0.0)) return fail(HLLD_ERR_INVALID, "cfl must be > 0");
    cudaStream_t st = (cudaStream_t)stream;
    if (g->precision == HLLD_FP64_EXACT)
        hlld::v_exact::launch_compute_dt_2d(g, s, cfl, dt_dev, work, st);
    else if (g->precision == HLLD_MIXED)
        hlld::v_mixed::launch_compute_dt_2d(g, s, cfl, dt_dev, work, st);
    else if (g->precision == HLLD_FP32)
        hlld::v_fp32::launch_compute_dt_2d(g, s, cfl, dt_dev, work, st);
    else
        hlld::v_fp64::launch_compute_dt_2d(g, s, cfl, dt_dev, work, st);
    return check_launch("compute_dt_2d");
}

int hlld_prim_to_cons_vjp(int64_t n, const void *const *prim, const void *const *lam_cons,
                          void *const *lam_prim, void *stream) {
    if (n < 0) return fail(HLLD_ERR_INVALID, "n < 0");
    if (n == 0) return HLLD_OK;
    if (!prim || !lam_cons || !lam_prim) return fail(HLLD_ERR_INVALID, "NULL array argument");
    for (int k = 0; k < 9; ++k)
        if (!prim[k] || !lam_prim[k]) return fail(HLLD_ERR_INVALID, "prim / lam_prim[%d] is NULL", k);
    hlld::v_adj::launch_prim_to_cons_vjp(n, prim, lam_cons, lam_prim, (cudaStream_t)stream);
    return check_launch("prim_to_cons_vjp");
}

int hlld_adjoint_scratch_bytes(const hlld_grid2d_t *g, size_t *bytes) {
    int rc = check_grid(g);
    if (rc) return rc;
    if (!bytes) return fail(HLLD_ERR_INVALID, "bytes is NULL");
    if (g->precision != HLLD_FP64)
        return fail(HLLD_ERR_UNSUPPORTED, "the adjoint is implemented for HLLD_FP64");
    *bytes = hlld::v_adj::adjoint_scratch_bytes(g);
    return HLLD_OK;
}

static int check_adjoint_grid(const hlld_grid2d_t *g) {
    int rc = check_grid(g);
    if (rc) return rc;
    if (g->precision != HLLD_FP64)
        return fail(HLLD_ERR_UNSUPPORTED, "the adjoint is implemented for HLLD_FP64");
    if (g->solver == HLLD_SOLVER_HLLC)
        return fail(HLLD_ERR_UNSUPPORTED, "the adjoint is implemented for HLLE and HLLD");
    if (g->emf_mode != HLLD_EMF_SOLVER)
        return fail(HLLD_ERR_UNSUPPORTED, "the adjoint is implemented for emf_mode HLLD_EMF_SOLVER");
    return HLLD_OK;
}

static int check_buffer(const void *p, size_t have, size_t need, const char *what) {
    if (!p) return fail(HLLD_ERR_INVALID, "%s is NULL", what);
    if ((uintptr_t)p % kAlign) return fail(HLLD_ERR_INVALID, "%s must be 256-byte aligned", what);
    if (have < need) return fail(HLLD_ERR_SCRATCH, "%s has %zu bytes, %zu needed", what, have, need);
    return HLLD_OK;
}

int hlld_adjoint_tape_bytes(const hlld_grid2d_t *g, size_t *tape_bytes, size_t *scratch_bytes) {
    int rc = check_adjoint_grid(g);
    if (rc) return rc;
    if (!tape_bytes || !scratch_bytes) return fail(HLLD_ERR_INVALID, "size outputs are NULL");
    *tape_bytes = hlld::v_adj::adjoint_tape_bytes(g);
    *scratch_bytes = hlld::v_adj::adjoint_reverse_scratch_bytes(g);
    return HLLD_OK;
}

int hlld_adjoint_record_step(const hlld_grid2d_t *g, const hlld_state2d_t *s, double dt,
                             int scheme, void *tape, size_t tape_bytes, void *scratch,
                             size_t scratch_bytes, void *stream) {
    int rc = check_adjoint_grid(g);
    if (rc) return rc;
    if ((rc = check_state(s))) return rc;
    if (scheme != 2 && scheme != 3) return fail(HLLD_ERR_INVALID, "scheme must be 2 or 3");
    if (!(dt > 0.0)) return fail(HLLD_ERR_INVALID, "dt must be > 0");
    if ((rc = check_buffer(tape, tape_bytes, hlld::v_adj::adjoint_tape_bytes(g), "tape"))) return rc;
    if ((rc = check_buffer(scratch, scratch_bytes, hlld::v_adj::adjoint_reverse_scratch_bytes(g),
                           "scratch")))
        return rc;
    hlld::v_adj::launch_adjoint_record(g, s, dt, scheme, tape, scratch, (cudaStream_t)stream);
    return check_launch("adjoint_record_step");
}

int hlld_adjoint_reverse_step(const hlld_grid2d_t *g, const hlld_state2d_t *s_in,
                              const hlld_state2d_t *s_out, double dt, int scheme, const void *tape,
                              size_t tape_bytes, const hlld_state2d_t *lam, void *scratch,
                              size_t scratch_bytes, void *stream) {
    int rc = check_adjoint_grid(g);
    if (rc) return rc;
    if ((rc = check_state(s_in)) || (rc = check_state(s_out)) || (rc = check_state(lam))) return rc;
    if (scheme != 2 && scheme != 3) return fail(HLLD_ERR_INVALID, "scheme must be 2 or 3");
    if (!(dt > 0.0)) return fail(HLLD_ERR_INVALID, "dt must be > 0");
    if ((rc = check_buffer(tape, tape_bytes, hlld::v_adj::adjoint_tape_bytes(g), "tape"))) return rc;
    if ((rc = check_buffer(scratch, scratch_bytes, hlld::v_adj::adjoint_reverse_scratch_bytes(g),
                           "scratch")))
        return rc;
    hlld::v_adj::launch_adjoint_reverse(g, s_in, s_out, dt, scheme, tape, lam, scratch,
                                        (cudaStream_t)stream);
    return check_launch("adjoint_reverse_step");
}

int hlld_adjoint_rk_step_ct(const hlld_grid2d_t *g, const hlld_state2d_t *s_in,
                            const hlld_state2d_t *s_out, double dt, int scheme,
                            const hlld_state2d_t *lam, void *scratch, size_t scratch_bytes,
                            void *stream) {
    int rc = check_grid(g);
    if (rc) return rc;
    if (g->precision != HLLD_FP64)
        return fail(HLLD_ERR_UNSUPPORTED, "the adjoint is implemented for HLLD_FP64");
    if (g->solver == HLLD_SOLVER_HLLC)
        return fail(HLLD_ERR_UNSUPPORTED, "the adjoint is implemented for HLLE and HLLD");
    if ((rc = check_state(s_in)) || (rc = check_state(s_out)) || (rc = check_state(lam))) return rc;
    if (scheme != 2 && scheme != 3) return fail(HLLD_ERR_INVALID, "scheme must be 2 or 3");
    if (!(dt > 0.0)) return fail(HLLD_ERR_INVALID, "dt must be > 0");
    if (!scratch) return fail(HLLD_ERR_INVALID, "scratch is NULL");
    if ((uintptr_t)scratch % kAlign) return fail(HLLD_ERR_INVALID, "scratch must be 256-byte aligned");
    const size_t need = hlld::v_adj::adjoint_scratch_bytes(g);
    if (scratch_bytes < need)
        return fail(HLLD_ERR_SCRATCH, "scratch has %zu bytes, the adjoint needs %zu", scratch_bytes, need);
    hlld::v_adj::launch_adjoint_rk_step_ct(g, s_in, s_out, dt, scheme, lam, scratch,
                                             (cudaStream_t)stream);
    return check_launch("adjoint_rk_step_ct");
}

}  // extern "C"
