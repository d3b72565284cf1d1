/*
 * CPU oracle for the SRMHD finite-volume step -- TEST INFRASTRUCTURE ONLY.
 * See srmhd_oracle.h for the semantics and the list of permitted callers.
 *
 * Every expression follows the cited reference line, operation by
 * operation, so that each intermediate rounds exactly as in the reference's
 * element-wise PyTorch code.  Build with -O2 -ffp-contract=off (no FMA
 * contraction, no fast-math).
 */
#include "srmhd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TINY 1e-300 /* hlld.py:29, c2p.py:29 */

int orc_version(void) { return 1; }

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ── element-wise helpers with torch's semantics ───────────────────────── */

/* torch.maximum / torch.minimum: NaN-propagating; ties keep the first operand */
static inline double tmax(double a, double b) {
    if (isnan(a)) return a;
    if (isnan(b)) return b;
    return (a < b) ? b : a;
}
static inline double tmin(double a, double b) {
    if (isnan(a)) return a;
    if (isnan(b)) return b;
    return (b < a) ? b : a;
}
/* torch.clamp(x, min=lo) / torch.clamp(x, max=hi) with a scalar bound */
static inline double clamp_lo(double x, double lo) { return (x < lo) ? lo : x; }
static inline double clamp_hi(double x, double hi) { return (x > hi) ? hi : x; }
/* torch.sign: -1, 0, +1; sign(NaN) = 0 */
static inline double tsign(double x) { return (x > 0.0) ? 1.0 : ((x < 0.0) ? -1.0 : 0.0); }

/* hlld.py:45-54 _sdiv (identical to c2p.py:32-36) */
static inline double sdiv(double num, double den) {
    if (fabs(den) < TINY) {
        double s = tsign(den);
        if (s == 0.0) s = 1.0;
        return num / (s * TINY);
    }
    return num / den;
}

/* ── EOS: hybrid_eos(K=0, gamma, gamma_th=gamma) (eos.py:32-76) ────────── */

/* eos.py:32-39 press__eps_rho with press_cold = eps_cold = 0 */
static inline double eos_press(double eps, double rho, double gamma) {
    double e = tmax(eps, 0.0);
    return 0.0 + (e - 0.0) * rho * (gamma - 1.0);
}
/* eos.py:41-46 eps__press_rho */
static inline double eos_eps(double press, double rho, double gamma) {
    return 0.0 + (press - 0.0) / (rho * (gamma - 1.0));
}
/* eos.py:65-76 press_and_cs2 (not cold: gamma_th = gamma != 1) */
static inline void eos_press_cs2(double eps, double rho, double gamma, double *p, double *cs2) {
    double press = eos_press(eps, rho, gamma);
    double h = 1.0 + eps + press / rho;
    double press_th = press - 0.0;
    *p = press;
    *cs2 = (gamma * 0.0 + gamma * press_th) / (rho * h);
}

/* ── primitive -> conserved (hlld.py:185-217) ─────────────────────────── */

static void p2c_one(const double *P, double *C) {
    double rho = P[ORC_RHO], vx = P[ORC_VX], vy = P[ORC_VY], vz = P[ORC_VZ];
    double p = P[ORC_P], eps = P[ORC_EPS];
    double Bx = P[ORC_PBX], By = P[ORC_PBY], Bz = P[ORC_PBZ];
    double v2 = vx * vx + vy * vy + vz * vz;
    double W = 1.0 / sqrt(clamp_lo(1.0 - v2, 1e-10));
    double vB = vx * Bx + vy * By + vz * Bz;
    double B2 = Bx * Bx + By * By + Bz * Bz;
    double h = 1.0 + eps + p / rho;
    double rHW2 = rho * h * (W * W);
    double D = rho * W;
    C[ORC_D] = D;
    C[ORC_SX] = (rHW2 + B2) * vx - vB * Bx;
    C[ORC_SY] = (rHW2 + B2) * vy - vB * By;
    C[ORC_SZ] = (rHW2 + B2) * vz - vB * Bz;
    C[ORC_TAU] = rHW2 - p - D + 0.5 * (B2 + B2 * v2 - vB * vB);
    C[ORC_BX] = Bx;
    C[ORC_BY] = By;
    C[ORC_BZ] = Bz;
}

void orc_prim_to_cons(int64_t n, const double *const *prim, double *const *cons) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double P[ORC_NPRIM], C[ORC_NCONS];
        for (int k = 0; k < ORC_NPRIM; ++k) P[k] = prim[k][i];
        p2c_one(P, C);
        for (int k = 0; k < ORC_NCONS; ++k) cons[k][i] = C[k];
    }
}

/* ── Kastaun C2P (c2p.py:41-363) ──────────────────────────────────────── */

typedef struct {
    double D, tau, S[3], B[3];
    double S2, B2, BdotS;
    double q, r[3], rNorm2;
    double Bt[3], BtNorm2;
    double B_dot_r, B2_rPerp2;
    double v02;
    double gamma;
} kastaun_t;

/* c2p.py:48-106 */
static void kastaun_init(kastaun_t *k, const double *C, double gamma) {
    double D = C[ORC_D];
    double Sx = C[ORC_SX], Sy = C[ORC_SY], Sz = C[ORC_SZ];
    double tau = C[ORC_TAU];
    double Bx = C[ORC_BX], By = C[ORC_BY], Bz = C[ORC_BZ];
    tau = clamp_lo(tau, 0.0);
    double S2 = Sx * Sx + Sy * Sy + Sz * Sz;
    double Snorm = sqrt(S2);
    double S_max = D + tau;
    int too_large = Snorm > S_max;
    double fac = too_large ? 0.9999 * S_max / (Snorm + TINY) : 1.0;
    Sx = Sx * fac;
    Sy = Sy * fac;
    Sz = Sz * fac;
    S2 = Sx * Sx + Sy * Sy + Sz * Sz;
    double B2 = Bx * Bx + By * By + Bz * Bz;
    double BdotS = Bx * Sx + By * Sy + Bz * Sz;
    k->D = D;
    k->tau = tau;
    k->S[0] = Sx; k->S[1] = Sy; k->S[2] = Sz;
    k->B[0] = Bx; k->B[1] = By; k->B[2] = Bz;
    k->S2 = S2;
    k->B2 = B2;
    k->BdotS = BdotS;
    k->q = tau / (D + TINY);
    k->r[0] = Sx / (D + TINY);
    k->r[1] = Sy / (D + TINY);
    k->r[2] = Sz / (D + TINY);
    k->rNorm2 = S2 / (D * D + TINY);
    double sqrtD = sqrt(D + TINY);
    k->Bt[0] = Bx / sqrtD;
    k->Bt[1] = By / sqrtD;
    k->Bt[2] = Bz / sqrtD;
    k->BtNorm2 = B2 / (D + TINY);
    k->B_dot_r = BdotS / (D * sqrtD + TINY);
    k->B2_rPerp2 = k->rNorm2 * k->BtNorm2 - k->B_dot_r * k->B_dot_r;
    k->v02 = k->rNorm2 / (k->rNorm2 + 1.0);
    k->gamma = gamma;
}

/* c2p.py:110-111 */
static inline double k_chi(const kastaun_t *k, double mu) { return 1.0 / (1.0 + mu * k->BtNorm2); }
/* c2p.py:113-116 */
static inline double k_rbar2(const kastaun_t *k, double mu) {
    double chi = k_chi(k, mu);
    return k->rNorm2 * (chi * chi) + mu * chi * (1.0 + chi) * (k->B_dot_r * k->B_dot_r);
}
/* c2p.py:118-122 */
static inline double k_qbar(const kastaun_t *k, double mu) {
    double chi = k_chi(k, mu);
    double mc = mu * chi;
    return k->q - 0.5 * k->BtNorm2 - 0.5 * (mc * mc) * k->B2_rPerp2;
}
/* c2p.py:124-127 */
static inline double k_fa(const kastaun_t *k, double mu) {
    return mu * sqrt(1.0 + k_rbar2(k, mu)) - 1.0;
}

typedef struct {
    double f, rho, eps, W, vhat2;
} master_t;

/* c2p.py:129-158 */
static master_t k_master(const kastaun_t *k, double mu) {
    master_t m;
    double qbar = k_qbar(k, mu);
    double rbar2 = k_rbar2(k, mu);
    double vhat2 = tmin((mu * mu) * rbar2, k->v02);
    double What = 1.0 / sqrt(clamp_lo(1.0 - vhat2, 1e-10));
    double rhohat0 = k->D / What;
    double rhohat = tmin(tmax(rhohat0, 1e-12), 1e15);
    double epshat0 = What * (qbar - mu * rbar2) + vhat2 * (What * What) / (1.0 + What);
    double epshat = tmin(tmax(epshat0, 0.0), 1e5);
    double phat = eos_press(epshat, rhohat, k->gamma);
    double ahat = phat / (rhohat * (1.0 + epshat) + TINY);
    double h_eff = (1.0 + ahat) * (1.0 + epshat);
    double nu_A = h_eff / What;
    double nu_B = (1 + ahat) * (1.0 + qbar - mu * rbar2);
    double nu = tmax(nu_A, nu_B);
    m.f = mu - sdiv(1.0, nu + mu * rbar2);
    m.rho = rhohat;
    m.eps = epshat;
    m.W = What;
    m.vhat2 = vhat2;
    return m;
}

/* c2p.py:162-184: 50 halvings of [0, 1]; the bracket width is exactly
 * 2^-k, so the batch-wide early stop never fires before the last step. */
static double k_mu_plus(const kastaun_t *k) {
    double lo = 0.0, hi = 1.0 / (1.0 + TINY);
    for (int it = 0; it < 50; ++it) {
        double mid = 0.5 * (lo + hi);
        double f_mid = k_fa(k, mid);
        double f_lo = k_fa(k, lo);
        int lft = (f_lo * f_mid) <= 0.0;
        if (lft) hi = mid;
        else lo = mid;
    }
    return hi;
}

typedef struct {
    double rho, v[3], p, eps;
    int bracket_ok, converged, v_clamped;
} c2p_out_t;

/* c2p.py:268-310 */
static void k_finish(const kastaun_t *k, double mu, int converged, int good_bracket,
                     c2p_out_t *o) {
    master_t m = k_master(k, mu);
    double chi = k_chi(k, mu);
    double mc = mu * chi;
    double mB = mu * k->B_dot_r;
    double v[3];
    for (int i = 0; i < 3; ++i) v[i] = mc * (k->r[i] + mB * k->Bt[i]);
    double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    double v2c = clamp_hi(v2, 1.0 - 1e-10);
    double norm = (v2 > 1.0 - 1e-10) ? sqrt(v2c / (v2 + TINY)) : 1.0;
    for (int i = 0; i < 3; ++i) o->v[i] = v[i] * norm;
    o->bracket_ok = good_bracket;
    o->converged = converged;
    o->v_clamped = v2 > 1.0 - 1e-10;
    o->p = eos_press(m.eps, m.rho, k->gamma);
    o->rho = m.rho;
    o->eps = m.eps;
}

/* c2p.py:188-236 invert, per element */
static void k_invert(const kastaun_t *k, c2p_out_t *o) {
    const double tol = 1e-15;
    double mu_plus = k_mu_plus(k);
    double mu_lo = 0.0;
    double mu_hi = mu_plus * (1.0 - 1e-10);
    double f_lo = k_master(k, mu_lo).f;
    double f_hi = k_master(k, mu_hi).f;
    int good_bracket = (f_lo * f_hi) < 0.0;
    double x0 = mu_lo, x1 = mu_hi, f0 = f_lo, f1 = f_hi;
    for (int it = 0; it < 60; ++it) {
        if (fabs(f1) < tol) break;
        double df = f1 - f0;
        int safe = fabs(df) > 1e-30;
        double x2s = safe ? x1 - f1 * (x1 - x0) / df : 0.5 * (x0 + x1);
        int inb = (x2s - x0) * (x2s - x1) < 0.0;
        double x2 = inb ? x2s : 0.5 * (x0 + x1);
        double f2 = k_master(k, x2).f;
        int lft = (f0 * f2) <= 0.0;
        if (!lft) {
            x0 = x1;
            f0 = f1;
        }
        x1 = x2;
        f1 = f2;
    }
    k_finish(k, x1, fabs(f1) < tol, good_bracket, o);
}

/* c2p.py:238-266 invert_bisection.  Once the bracket has collapsed onto
 * adjacent doubles every further halving maps the state onto itself, so
 * stopping at the first unchanged iteration returns the 200-step result. */
static void k_invert_bisection(const kastaun_t *k, c2p_out_t *o) {
    const double tol = 1e-15;
    double mu_plus = k_mu_plus(k);
    double x0 = 0.0;
    double x1 = mu_plus * (1.0 - 1e-10);
    double f0 = k_master(k, x0).f;
    double f1 = k_master(k, x1).f;
    int good_bracket = (f0 * f1) < 0.0;
    for (int it = 0; it < 200; ++it) {
        double xm = 0.5 * (x0 + x1);
        double fm = k_master(k, xm).f;
        int left = (f0 * fm) <= 0.0;
        double nx0 = left ? x0 : xm, nf0 = left ? f0 : fm;
        double nx1 = left ? xm : x1, nf1 = left ? fm : f1;
        int same = (memcmp(&nx0, &x0, 8) == 0) && (memcmp(&nx1, &x1, 8) == 0) &&
                   (memcmp(&nf0, &f0, 8) == 0) && (memcmp(&nf1, &f1, 8) == 0);
        x0 = nx0; f0 = nf0; x1 = nx1; f1 = nf1;
        if (same) break;
    }
    int pick = fabs(f0) < fabs(f1);
    double mu = pick ? x0 : x1;
    double fmu = pick ? f0 : f1;
    k_finish(k, mu, fabs(fmu) < tol, good_bracket, o);
}

/* c2p.py:313-363 conservative_to_primitive for one element */
static void c2p_one(const double *C, double gamma, double atmo_rho, double atmo_eps, double *P,
                    uint8_t *status) {
    kastaun_t k;
    kastaun_init(&k, C, gamma);
    c2p_out_t o;
    k_invert(&k, &o);
    uint8_t st = 0;
    int bisected = 0;
    if (!o.converged && o.bracket_ok) {
        int bo = o.bracket_ok;
        k_invert_bisection(&k, &o);
        o.bracket_ok = bo;
        bisected = 1;
    }
    double rho = o.rho, eps = o.eps, vx = o.v[0], vy = o.v[1], vz = o.v[2];
    int atmo = rho < atmo_rho;
    if (atmo) {
        rho = atmo_rho;
        eps = atmo_eps;
        vx = 0.0;
        vy = 0.0;
        vz = 0.0;
    }
    P[ORC_RHO] = rho;
    P[ORC_VX] = vx;
    P[ORC_VY] = vy;
    P[ORC_VZ] = vz;
    P[ORC_P] = eos_press(eps, rho, gamma);
    P[ORC_EPS] = eps;
    P[ORC_PBX] = C[ORC_BX];
    P[ORC_PBY] = C[ORC_BY];
    P[ORC_PBZ] = C[ORC_BZ];
    if (o.bracket_ok) st |= ORC_ST_BRACKET_OK;
    if (o.converged) st |= ORC_ST_CONVERGED;
    if (o.v_clamped) st |= ORC_ST_V_CLAMPED;
    if (atmo) st |= ORC_ST_ATMO;
    if (bisected) st |= ORC_ST_BISECTED;
    if (status) *status = st;
}

void orc_cons_to_prim(int64_t n, const double *const *cons, double gamma, double atmo_rho,
                      double atmo_eps, double *const *prim, uint8_t *status) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
        double C[ORC_NCONS], P[ORC_NPRIM];
        for (int k = 0; k < ORC_NCONS; ++k) C[k] = cons[k][i];
        c2p_one(C, gamma, atmo_rho, atmo_eps, P, status ? status + i : NULL);
        for (int k = 0; k < ORC_NPRIM; ++k) prim[k][i] = P[k];
    }
}

/* ── physical fluxes (hlld.py:57-113, :223-334) ───────────────────────── */

typedef struct {
    double u[ORC_NCONS], f[ORC_NCONS];
} side_t;

/* hlld.py:100-113 compute_cp_cm with one_over_alp2 = 1, betad = 0, gupdd = 1 */
static void cp_cm(double v02, double u0, double vd, double *cp, double *cm) {
    double u0_sq = u0 * u0;
    double a = u0_sq * (1.0 - v02) + v02 * 1.0;
    double b = 2.0 * (0.0 * 1.0 * v02 - u0_sq * vd * (1.0 - v02));
    double c = u0_sq * (vd * vd) * (1.0 - v02) - v02 * (1.0 - 0.0 * 0.0 * 1.0);
    double det = sqrt(clamp_lo(b * b - 4.0 * a * c, 0.0));
    double a_safe = clamp_lo(a, TINY);
    double c1 = 0.5 * (det - b) / a_safe;
    double c2 = -0.5 * (det + b) / a_safe;
    *cp = tmax(c1, c2);
    *cm = tmin(c1, c2);
}

/* hlld.py:57-62 lorentz */
static inline double lorentz_W(const double *P) {
    double v2 = P[ORC_VX] * P[ORC_VX] + P[ORC_VY] * P[ORC_VY] + P[ORC_VZ] * P[ORC_VZ];
    double v2s = clamp_hi(v2, 1.0 - 1e-10);
    return 1.0 / sqrt(1.0 - v2s);
}

/* hlld.py:84-90 compute_b2 */
static inline double comp_b2(const double *P, double W) {
    double B2 = P[ORC_PBX] * P[ORC_PBX] + P[ORC_PBY] * P[ORC_PBY] + P[ORC_PBZ] * P[ORC_PBZ];
    double vdotB = P[ORC_VX] * P[ORC_PBX] + P[ORC_VY] * P[ORC_PBY] + P[ORC_VZ] * P[ORC_PBZ];
    return B2 / (W * W) + vdotB * vdotB;
}

/* one side of compute_srmhd_fluxes (hlld.py:234-332); returns cp, cm */
static void phys_side(const double *P, int idir, double gamma, side_t *s, double *cp,
                      double *cm) {
    double W = lorentz_W(P);
    double p, cs2;
    eos_press_cs2(P[ORC_EPS], P[ORC_RHO], gamma, &p, &cs2);
    double b2 = comp_b2(P, W);
    /* hlld.py:65-81 compute_smallb */
    double v[3] = {P[ORC_VX], P[ORC_VY], P[ORC_VZ]};
    double B[3] = {P[ORC_PBX], P[ORC_PBY], P[ORC_PBZ]};
    double vdotB = v[0] * B[0] + v[1] * B[1] + v[2] * B[2];
    double bt = W * vdotB;
    double bs[3];
    for (int i = 0; i < 3; ++i) bs[i] = B[i] / W + vdotB * v[i] * W;
    /* hlld.py:93-97 */
    double rho = P[ORC_RHO], eps = P[ORC_EPS];
    double h = 1.0 + eps + p / rho;
    double v02 = cs2 + (b2 / (rho * h + b2)) * (1.0 - cs2);
    cp_cm(v02, W, v[idir], cp, cm);
    double d = rho * W;
    double uD[3] = {W * v[0], W * v[1], W * v[2]};
    double rhb2 = rho * h + b2;
    double Pb2 = p + 0.5 * b2;
    double vd = v[idir];
    double bdir = bs[idir];
    s->u[ORC_D] = d;
    s->f[ORC_D] = d * vd;
    double Tt = rhb2 * (W * W) + Pb2 * (-1.0) - bt * bt;
    s->u[ORC_TAU] = Tt - d;
    s->f[ORC_TAU] = (rhb2 * (W * W) * vd - bt * bdir) - d * vd;
    for (int i = 0; i < 3; ++i) {
        double delta = (i == idir) ? 1.0 : 0.0;
        s->u[ORC_SX + i] = rhb2 * W * uD[i] - bt * bs[i];
        s->f[ORC_SX + i] = rhb2 * (W * vd) * uD[i] + Pb2 * delta - bdir * bs[i];
    }
    double Bdir = B[idir];
    for (int i = 0; i < 3; ++i) {
        s->u[ORC_BX + i] = B[i];
        s->f[ORC_BX + i] = vd * B[i] - v[i] * Bdir;
    }
}

typedef struct {
    side_t L, R;
    double cmax, cmin;
} phys_t;

static void compute_srmhd_fluxes(const double *PL, const double *PR, int idir, double gamma,
                                 phys_t *ph) {
    double cp_l, cm_l, cp_r, cm_r;
    phys_side(PL, idir, gamma, &ph->L, &cp_l, &cm_l);
    phys_side(PR, idir, gamma, &ph->R, &cp_r, &cm_r);
    double cmax = clamp_lo(tmax(cp_l, cp_r), 0.0);
    double cmin = clamp_lo(tmax(-cm_l, -cm_r), 0.0);
    int both_small = (cmax < 1e-12) && (cmin < 1e-12);
    if (both_small) {
        cmax = 1.0;
        cmin = 1.0;
    }
    ph->cmax = cmax;
    ph->cmin = cmin;
}

/* hlld.py:161-168 _hf, _hu */
static inline double hf(double fL, double fR, double uL, double uR, double cm, double cx) {
    return (cx * fL + cm * fR - cx * cm * (uR - uL)) / (cx + cm);
}
static inline double hu(double fL, double fR, double uL, double uR, double cm, double cx) {
    return (cx * uR + cm * uL + fL - fR) / (cx + cm);
}

/* hlld.py:1036-1042: the HLL total-pressure estimate returned by hlle_flux */
static double hlle_p_estimate(const double *PL, const double *PR, double gamma) {
    double pl, pr, c;
    eos_press_cs2(PL[ORC_EPS], PL[ORC_RHO], gamma, &pl, &c);
    eos_press_cs2(PR[ORC_EPS], PR[ORC_RHO], gamma, &pr, &c);
    double wl = lorentz_W(PL), wr = lorentz_W(PR);
    double b2l = comp_b2(PL, wl), b2r = comp_b2(PR, wr);
    return clamp_lo(0.5 * (pl + 0.5 * b2l + pr + 0.5 * b2r), 1e-30);
}

/* hlld.py:1005-1044 hlle_flux for one face */
static void hlle_one(const double *PL, const double *PR, int idir, double gamma, double *F,
                     double *U, double *pstar) {
    phys_t ph;
    compute_srmhd_fluxes(PL, PR, idir, gamma, &ph);
    double cm = ph.cmin, cx = ph.cmax;
    for (int k = 0; k < ORC_NCONS; ++k) {
        double fL = ph.L.f[k], fR = ph.R.f[k], uL = ph.L.u[k], uR = ph.R.u[k];
        double fH = hf(fL, fR, uL, uR, cm, cx);
        double uH = hu(fL, fR, uL, uR, cm, cx);
        F[k] = (cx <= 0) ? fR : ((cm <= 0) ? fL : fH);
        U[k] = (cm <= 0) ? uL : ((cx <= 0) ? uR : uH);
    }
    *pstar = hlle_p_estimate(PL, PR, gamma);
}

/* ── HLLD (hlld.py:366-605, :669-746, :1202-1543) ─────────────────────── */

typedef struct {
    /* R vectors (hlld.py:401-428), energy form */
    double RSiL, RSiR, RS1L, RS1R, RS2L, RS2R;
    double RBiL, RBiR, RB1L, RB1R, RB2L, RB2R;
    double RTL, RTR, RDL, RDR;
    double S_L, S_R, BnL, BnR, cm, cx;
} hlld_calc_t;

typedef struct {
    double vaL, vaR, vt1aL, vt2aL, vt1aR, vt2aR;
    double Bt1aL, Bt2aL, Bt1aR, Bt2aR;
    double waL, waR, sqL, sqR, DaL, DaR, TauaL, TauaR;
    double SaL, SaR, St1aL, St2aL, St1aR, St2aR;
    double laL, laR, Kt1aL, Kt2aL, Kt1aR, Kt2aR;
    double Bic, Bt1c, Bt2c, KaL2, KaR2, KaLBc, KaRBc;
} hlld_vars_t;

/* hlld.py:431-583 compute_all_variables */
static void hlld_vars(const hlld_calc_t *c, double p, hlld_vars_t *o) {
    double cm = c->cm, cx = c->cx;
    double RSiL = c->RSiL, RSiR = c->RSiR, RS1L = c->RS1L, RS1R = c->RS1R;
    double RS2L = c->RS2L, RS2R = c->RS2R;
    double RB1L = c->RB1L, RB1R = c->RB1R, RB2L = c->RB2L, RB2R = c->RB2R;
    double RTL = c->RTL, RTR = c->RTR;
    double BnL = c->BnL, BnR = c->BnR;
    double ncm = -cm;

    double AL = RSiL - ncm * RTL + p * (1 - cm * cm);
    double AR = RSiR - cx * RTR + p * (1 - cx * cx);
    double GL = RB1L * RB1L + RB2L * RB2L;
    double GR = RB1R * RB1R + RB2R * RB2R;
    double CL = RS1L * RB1L + RS2L * RB2L;
    double CR = RS1R * RB1R + RS2R * RB2R;
    double QL = -AL - GL + (BnL * BnL) * (1 - cm * cm);
    double QR = -AR - GR + (BnR * BnR) * (1 - cx * cx);
    double XL = BnL * (AL * ncm * BnL + CL) - (AL + GL) * (ncm * p + RTL);
    double XR = BnR * (AR * cx * BnR + CR) - (AR + GR) * (cx * p + RTR);

    double vaL = sdiv(BnL * (AL * BnL + ncm * CL) - (AL + GL) * (p + RSiL), XL);
    double vaR = sdiv(BnR * (AR * BnR + cx * CR) - (AR + GR) * (p + RSiR), XR);
    double vt1aL = sdiv(QL * RS1L + RB1L * (CL + BnL * (ncm * RSiL - RTL)), XL);
    double vt1aR = sdiv(QR * RS1R + RB1R * (CR + BnR * (cx * RSiR - RTR)), XR);
    double vt2aL = sdiv(QL * RS2L + RB2L * (CL + BnL * (ncm * RSiL - RTL)), XL);
    double vt2aR = sdiv(QR * RS2R + RB2R * (CR + BnR * (cx * RSiR - RTR)), XR);

    double Bt1aL = sdiv(RB1L - BnL * vt1aL, ncm - vaL);
    double Bt1aR = sdiv(RB1R - BnR * vt1aR, cx - vaR);
    double Bt2aL = sdiv(RB2L - BnL * vt2aL, ncm - vaL);
    double Bt2aR = sdiv(RB2R - BnR * vt2aR, cx - vaR);

    double vRS_AL = vaL * RSiL + vt1aL * RS1L + vt2aL * RS2L;
    double vRS_AR = vaR * RSiR + vt1aR * RS1R + vt2aR * RS2R;

    double waL = p + sdiv(RTL - vRS_AL, ncm - vaL);
    double waR = p + sdiv(RTR - vRS_AR, cx - vaR);
    double DaL = sdiv(c->RDL, ncm - vaL);
    double DaR = sdiv(c->RDR, cx - vaR);

    double vBaL = vaL * BnL + vt1aL * Bt1aL + vt2aL * Bt2aL;
    double vBaR = vaR * BnR + vt1aR * Bt1aR + vt2aR * Bt2aR;

    double TauaL = sdiv(RTL + p * vaL - vBaL * BnL, ncm - vaL) - DaL;
    double TauaR = sdiv(RTR + p * vaR - vBaR * BnR, cx - vaR) - DaR;

    double SaL = (TauaL + DaL + p) * vaL - vBaL * BnL;
    double SaR = (TauaR + DaR + p) * vaR - vBaR * BnR;
    double St1aL = (TauaL + DaL + p) * vt1aL - vBaL * Bt1aL;
    double St1aR = (TauaR + DaR + p) * vt1aR - vBaR * Bt1aR;
    double St2aL = (TauaL + DaL + p) * vt2aL - vBaL * Bt2aL;
    double St2aR = (TauaR + DaR + p) * vt2aR - vBaR * Bt2aR;

    double sqL = sqrt(clamp_lo(waL, 0.0));
    double sqR = sqrt(clamp_lo(waR, 0.0));

    double S_L = c->S_L, S_R = c->S_R;
    double dL = ncm * p + RTL - BnL * S_L * sqL;
    double dR = cx * p + RTR + BnR * S_R * sqR;

    double KaL = sdiv(RSiL + p - c->RBiL * S_L * sqL, dL);
    double KaR = sdiv(RSiR + p + c->RBiR * S_R * sqR, dR);
    double Kt1aL = sdiv(RS1L - RB1L * S_L * sqL, dL);
    double Kt1aR = sdiv(RS1R + RB1R * S_R * sqR, dR);
    double Kt2aL = sdiv(RS2L - RB2L * S_L * sqL, dL);
    double Kt2aR = sdiv(RS2R + RB2R * S_R * sqR, dR);

    double laL = KaL, laR = KaR;
    double denom_ll = laR - laL;
    double Bic = BnR;
    double Bt1c = sdiv((Bt1aR * (laR - vaR) + BnR * vt1aR) - (Bt1aL * (laL - vaL) + BnL * vt1aL),
                       denom_ll);
    double Bt2c = sdiv((Bt2aR * (laR - vaR) + BnR * vt2aR) - (Bt2aL * (laL - vaL) + BnL * vt2aL),
                       denom_ll);

    o->vaL = vaL; o->vaR = vaR;
    o->vt1aL = vt1aL; o->vt2aL = vt2aL; o->vt1aR = vt1aR; o->vt2aR = vt2aR;
    o->Bt1aL = Bt1aL; o->Bt2aL = Bt2aL; o->Bt1aR = Bt1aR; o->Bt2aR = Bt2aR;
    o->waL = waL; o->waR = waR; o->sqL = sqL; o->sqR = sqR;
    o->DaL = DaL; o->DaR = DaR; o->TauaL = TauaL; o->TauaR = TauaR;
    o->SaL = SaL; o->SaR = SaR; o->St1aL = St1aL; o->St2aL = St2aL;
    o->St1aR = St1aR; o->St2aR = St2aR;
    o->laL = laL; o->laR = laR;
    o->Kt1aL = Kt1aL; o->Kt2aL = Kt2aL; o->Kt1aR = Kt1aR; o->Kt2aR = Kt2aR;
    o->Bic = Bic; o->Bt1c = Bt1c; o->Bt2c = Bt2c;
    o->KaL2 = KaL * KaL + Kt1aL * Kt1aL + Kt2aL * Kt2aL;
    o->KaR2 = KaR * KaR + Kt1aR * Kt1aR + Kt2aR * Kt2aR;
    o->KaLBc = KaL * Bic + Kt1aL * Bt1c + Kt2aL * Bt2c;
    o->KaRBc = KaR * Bic + Kt1aR * Bt1c + Kt2aR * Bt2c;
}

/* hlld.py:586-602 residual */
static double hlld_residual(const hlld_calc_t *c, double p) {
    hlld_vars_t v;
    hlld_vars(c, p, &v);
    double denom_R = c->S_R * v.sqR - v.KaRBc;
    double denom_L = c->S_L * v.sqL + v.KaLBc;
    return (v.laL - v.laR) + c->BnL * (sdiv(1.0 - v.KaR2, denom_R) + sdiv(1.0 - v.KaL2, denom_L));
}

/* hlld.py:1202-1543 hlld_flux for one face */
static void hlld_one(const double *PL, const double *PR, int idir, double gamma, double *F,
                     double *U, double *pstar_out, int32_t *err_out, int32_t *iters_out,
                     uint8_t *flags_out) {
    const int i = idir, t1 = (idir + 1) % 3, t2 = (idir + 2) % 3;
    phys_t ph;
    compute_srmhd_fluxes(PL, PR, idir, gamma, &ph);
    const double cm = ph.cmin, cx = ph.cmax;
    const double *uL = ph.L.u, *uR = ph.R.u, *fL = ph.L.f, *fR = ph.R.f;
    double fH[ORC_NCONS], uH[ORC_NCONS];
    for (int k = 0; k < ORC_NCONS; ++k) {
        fH[k] = hf(fL[k], fR[k], uL[k], uR[k], cm, cx);
        uH[k] = hu(fL[k], fR[k], uL[k], uR[k], cm, cx);
    }
    /* energy form (hlld.py:337-360): tau -> tau + D */
    double UiL[ORC_NCONS], UiR[ORC_NCONS], FiL[ORC_NCONS], FiR[ORC_NCONS];
    memcpy(UiL, uL, sizeof UiL);
    memcpy(UiR, uR, sizeof UiR);
    memcpy(FiL, fL, sizeof FiL);
    memcpy(FiR, fR, sizeof FiR);
    UiL[ORC_TAU] = uL[ORC_TAU] + uL[ORC_D];
    UiR[ORC_TAU] = uR[ORC_TAU] + uR[ORC_D];
    FiL[ORC_TAU] = fL[ORC_TAU] + fL[ORC_D];
    FiR[ORC_TAU] = fR[ORC_TAU] + fR[ORC_D];

    /* legacy bracket (hlld.py:1253-1263): total pressure of the HLL state */
    double Phll[ORC_NPRIM];
    c2p_one(uH, gamma, 1e-10, 1e-10, Phll, NULL);
    double p_hll, cs2_hll;
    eos_press_cs2(Phll[ORC_EPS], Phll[ORC_RHO], gamma, &p_hll, &cs2_hll);
    double w_hll = lorentz_W(Phll);
    double b2_hll = comp_b2(Phll, w_hll);
    p_hll = p_hll + 0.5 * b2_hll;

    /* p0 from the Bn = 0 limit (hlld.py:1265-1287) */
    const int Sn = ORC_SX + i, Bn = ORC_BX + i;
    double a = fH[ORC_TAU] + fH[ORC_D];
    double b = -fH[Sn] - uH[ORC_TAU] - uH[ORC_D];
    double c = uH[Sn];
    double disc = b * b - 4.0 * a * c;
    disc = clamp_lo(disc, 0.0);
    int abig = fabs(a) > 1e-14;
    double safe_a = abig ? a : 1.0;
    double safe_b = abig ? b : 1.0;
    double v_star = abig ? (-b - sqrt(disc)) / (2.0 * safe_a) : -c / safe_b;
    v_star = clamp_hi(clamp_lo(v_star, -(1.0 - 1e-10)), 1.0 - 1e-10);
    double p0 = fH[Sn] - (fH[ORC_TAU] + fH[ORC_D]) * v_star;
    p0 = clamp_lo(p0, 1e-30);

    /* bracket (hlld.py:1292-1303) */
    double BnL = uL[Bn], BnR = uR[Bn];
    double Bn2 = 0.5 * (BnL * BnL + BnR * BnR);
    int use_p0 = (Bn2 / p_hll) < 0.1;
    double p_lo = use_p0 ? p0 * 0.99 : p_hll * 0.99;
    double p_hi = use_p0 ? p0 * 1.01 : p_hll * 1.01;
    int bn_zero = (fabs(BnL) < 1e-14) && (fabs(BnR) < 1e-14);

    /* HLLDComputation._build_R (hlld.py:401-428) on the energy-form state */
    hlld_calc_t C;
    C.cm = cm;
    C.cx = cx;
    C.RSiL = -cm * UiL[ORC_SX + i] - FiL[ORC_SX + i];
    C.RSiR = cx * UiR[ORC_SX + i] - FiR[ORC_SX + i];
    C.RS1L = -cm * UiL[ORC_SX + t1] - FiL[ORC_SX + t1];
    C.RS1R = cx * UiR[ORC_SX + t1] - FiR[ORC_SX + t1];
    C.RS2L = -cm * UiL[ORC_SX + t2] - FiL[ORC_SX + t2];
    C.RS2R = cx * UiR[ORC_SX + t2] - FiR[ORC_SX + t2];
    C.RBiL = -cm * UiL[ORC_BX + i] - FiL[ORC_BX + i];
    C.RBiR = cx * UiR[ORC_BX + i] - FiR[ORC_BX + i];
    C.RB1L = -cm * UiL[ORC_BX + t1] - FiL[ORC_BX + t1];
    C.RB1R = cx * UiR[ORC_BX + t1] - FiR[ORC_BX + t1];
    C.RB2L = -cm * UiL[ORC_BX + t2] - FiL[ORC_BX + t2];
    C.RB2R = cx * UiR[ORC_BX + t2] - FiR[ORC_BX + t2];
    C.RTL = -cm * UiL[ORC_TAU] - FiL[ORC_TAU];
    C.RTR = cx * UiR[ORC_TAU] - FiR[ORC_TAU];
    C.RDL = -cm * UiL[ORC_D] - FiL[ORC_D];
    C.RDR = cx * UiR[ORC_D] - FiR[ORC_D];
    C.S_L = tsign(UiL[ORC_BX + i]);
    C.S_R = tsign(UiR[ORC_BX + i]);
    C.BnL = UiL[ORC_BX + i];
    C.BnR = UiR[ORC_BX + i];

    double f_lo = hlld_residual(&C, p_lo);
    double f_hi = hlld_residual(&C, p_hi);
    /* bracket widening (hlld.py:1314-1321) */
    for (int w = 0; w < 5; ++w) {
        if (!((f_lo * f_hi) > 0.0)) break;
        p_lo = p_lo / 2.0;
        p_hi = p_hi * 2.0;
        f_lo = hlld_residual(&C, p_lo);
        f_hi = hlld_residual(&C, p_hi);
    }

    /* safe_secant_bisection (hlld.py:669-746), tol 1e-10, 30 iterations */
    const double tol = 1.0e-10;
    const int max_iter = 30;
    double x0 = p_lo, x1 = p_hi, f0 = f_lo, f1 = f_hi;
    int32_t err = max_iter, iters_used = max_iter;
    int done = 0;
    for (int it = 1; it <= max_iter; ++it) {
        if (fabs(f1) < tol) {
            err = 0;
            iters_used = it - 1;
            done = 1;
            break;
        }
        double df = f1 - f0;
        int safe = fabs(df) > 1e-30 * fabs(f1);
        double dx = safe ? f1 * (x1 - x0) / df : 0.0;
        double x2 = x1 - dx;
        x2 = clamp_lo(x2, 1e-30);
        double f2 = hlld_residual(&C, x2);
        x0 = x1;
        f0 = f1;
        x1 = x2;
        f1 = f2;
    }
    if (!done && fabs(f1) < tol) {
        err = 0;
        iters_used = max_iter;
    }
    double p_star = x1;

    hlld_vars_t V;
    hlld_vars(&C, p_star, &V);

    /* star states (hlld.py:1359-1445) */
    double uaL[ORC_NCONS], uaR[ORC_NCONS], faL[ORC_NCONS], faR[ORC_NCONS];
    double ucL[ORC_NCONS], ucR[ORC_NCONS];
    uaL[ORC_BX + i] = BnL; uaL[ORC_BX + t1] = V.Bt1aL; uaL[ORC_BX + t2] = V.Bt2aL;
    uaL[ORC_D] = V.DaL; uaL[ORC_TAU] = V.TauaL;
    uaL[ORC_SX + i] = V.SaL; uaL[ORC_SX + t1] = V.St1aL; uaL[ORC_SX + t2] = V.St2aL;
    uaR[ORC_BX + i] = BnR; uaR[ORC_BX + t1] = V.Bt1aR; uaR[ORC_BX + t2] = V.Bt2aR;
    uaR[ORC_D] = V.DaR; uaR[ORC_TAU] = V.TauaR;
    uaR[ORC_SX + i] = V.SaR; uaR[ORC_SX + t1] = V.St1aR; uaR[ORC_SX + t2] = V.St2aR;
    for (int k = 0; k < ORC_NCONS; ++k) {
        faL[k] = fL[k] + (-cm) * (uaL[k] - uL[k]);
        faR[k] = fR[k] + (cx) * (uaR[k] - uR[k]);
    }
    double fac = sdiv(1.0 - V.KaL2, -C.S_L * V.sqL - V.KaLBc);
    double vc = V.laL - V.Bic * fac;
    double vt1 = V.Kt1aL - V.Bt1c * fac;
    double vt2 = V.Kt2aL - V.Bt2c * fac;
    double lC = vc, laL = V.laL, laR = V.laR;
    double vcomp[3], Bc[3];
    vcomp[i] = vc; vcomp[t1] = vt1; vcomp[t2] = vt2;
    Bc[i] = V.Bic; Bc[t1] = V.Bt1c; Bc[t2] = V.Bt2c;
    ucL[ORC_BX + i] = V.Bic; ucL[ORC_BX + t1] = V.Bt1c; ucL[ORC_BX + t2] = V.Bt2c;
    ucR[ORC_BX + i] = V.Bic; ucR[ORC_BX + t1] = V.Bt1c; ucR[ORC_BX + t2] = V.Bt2c;
    double vBc = vc * V.Bic + vt1 * V.Bt1c + vt2 * V.Bt2c;
    ucL[ORC_D] = uaL[ORC_D] * sdiv(laL - V.vaL, laL - vc);
    ucR[ORC_D] = uaR[ORC_D] * sdiv(laR - V.vaR, laR - vc);
    ucL[ORC_TAU] = sdiv(laL * uaL[ORC_TAU] - faL[ORC_TAU] + p_star * vc - vBc * V.Bic, laL - vc);
    ucR[ORC_TAU] = sdiv(laR * uaR[ORC_TAU] - faR[ORC_TAU] + p_star * vc - vBc * V.Bic, laR - vc);
    /* components in the order normal, t1, t2 (hlld.py:1438-1445) */
    int comp_order[3] = {i, t1, t2};
    for (int q = 0; q < 3; ++q) {
        int cc = comp_order[q];
        ucL[ORC_SX + cc] = (ucL[ORC_TAU] + p_star + ucL[ORC_D]) * vcomp[cc] - vBc * Bc[cc];
    }
    for (int q = 0; q < 3; ++q) {
        int cc = comp_order[q];
        ucR[ORC_SX + cc] = (ucR[ORC_TAU] + p_star + ucR[ORC_D]) * vcomp[cc] - vBc * Bc[cc];
    }

    /* region selection at xi = 0 (hlld.py:1447-1480) */
    double vi = 0.0;
    int cL_mask = vi <= -cm;
    int caL_mask = (-cm < vi) && (vi <= laL);
    int ccL_mask = (laL < vi) && (vi < lC);
    int ccR_mask = (lC <= vi) && (vi < laR);
    int caR_mask = (laR <= vi) && (vi < cx);
    int cR_mask = vi >= cx;
    for (int k = 0; k < ORC_NCONS; ++k) {
        double fcL = faL[k] + laL * (ucL[k] - uaL[k]);
        double fcR = faR[k] + laR * (ucR[k] - uaR[k]);
        double f = fH[k];
        if (cL_mask) f = fL[k];
        if (caL_mask) f = faL[k];
        if (ccL_mask) f = fcL;
        if (ccR_mask) f = fcR;
        if (caR_mask) f = faR[k];
        if (cR_mask) f = fR[k];
        double u = uH[k];
        if (cL_mask) u = uL[k];
        if (caL_mask) u = uaL[k];
        if (ccL_mask) u = ucL[k];
        if (ccR_mask) u = ucR[k];
        if (caR_mask) u = uaR[k];
        if (cR_mask) u = uR[k];
        F[k] = f;
        U[k] = u;
    }
    /* degenerate states and fallback (hlld.py:1487-1534) */
    int wave_order_bad = (V.vaR > cx) || (V.vaL < -cm) || (vc < V.laL) || (vc > V.laR);
    int failed = (err > 0) || wave_order_bad || bn_zero;
    if (failed) {
        p_star = -fabs(p_hll) - 1e-10;
        for (int k = 0; k < ORC_NCONS; ++k) {
            F[k] = fH[k];
            U[k] = uH[k];
        }
    }
    *pstar_out = p_star;
    if (err_out) *err_out = err;
    if (iters_out) *iters_out = iters_used;
    if (flags_out)
        *flags_out = (uint8_t)((wave_order_bad ? ORC_RF_WAVE_ORDER_BAD : 0) |
                               (bn_zero ? ORC_RF_BN_ZERO : 0) | (failed ? ORC_RF_FAILED : 0));
}

/* hlld.py:1549-1765 hllc_flux for one face; pstar gets the p_hll the
 * reference returns in that slot */
static void hllc_one(const double *PL, const double *PR, int idir, double gamma, double *F,
                     double *U, double *pstar) {
    phys_t ph;
    compute_srmhd_fluxes(PL, PR, idir, gamma, &ph);
    const int t1 = (idir + 1) % 3, t2 = (idir + 2) % 3;
    const int Sn = ORC_SX + idir, S1 = ORC_SX + t1, S2 = ORC_SX + t2;
    const int Bn = ORC_BX + idir, B1 = ORC_BX + t1, B2 = ORC_BX + t2;
    const double cmin = ph.cmin, cmax = ph.cmax;
    const double S_L = -cmin, S_R = cmax;
    double fH[ORC_NCONS], uH[ORC_NCONS];
    for (int k = 0; k < ORC_NCONS; ++k) {
        fH[k] = hf(ph.L.f[k], ph.R.f[k], ph.L.u[k], ph.R.u[k], cmin, cmax);
        uH[k] = hu(ph.L.f[k], ph.R.f[k], ph.L.u[k], ph.R.u[k], cmin, cmax);
    }
    const double BG = ph.L.u[Bn];
    const int has_B = fabs(BG) > 1e-15;
    /* contact speed (quadratic, minus root) */
    const double cross = has_B ? uH[B1] * fH[B1] + uH[B2] * fH[B2] : 0.0;
    const double bt2 = has_B ? uH[B1] * uH[B1] + uH[B2] * uH[B2] : 0.0;
    const double fbt2 = has_B ? fH[B1] * fH[B1] + fH[B2] * fH[B2] : 0.0;
    const double E_hll = uH[ORC_TAU] + uH[ORC_D];
    const double fE_hll = fH[ORC_TAU] + fH[ORC_D];
    const double qa = fE_hll - cross;
    const double qb = -fH[Sn] - E_hll + bt2 + fbt2;
    const double qc = uH[Sn] - cross;
    const double disc = sqrt(clamp_lo(qb * qb - 4.0 * qa * qc, 0.0));
    const double vc_quad = sdiv(-0.5 * (qb + disc), qa);
    const double vc_lin = sdiv(-qc, qb);
    const double vc = fabs(qa) < 1e-15 ? (fabs(qb) < 1e-15 ? 0.0 : vc_lin) : vc_quad;
    /* star-region transverse velocities, Lorentz factor, v*.B* */
    const double vt1 = has_B ? sdiv(uH[B1] * vc - fH[B1], BG) : 0.0;
    const double vt2 = has_B ? sdiv(uH[B2] * vc - fH[B2], BG) : 0.0;
    const double v2 = vc * vc + vt1 * vt1 + vt2 * vt2;
    const double v2s = clamp_hi(v2, 1.0 - 1e-10);
    const double gs = 1.0 / sqrt(1.0 - v2s);
    const double vsBs = has_B ? vc * uH[Bn] + vt1 * uH[B1] + vt2 * uH[B2] : 0.0;
    const double bgs = BG / gs;
    const double p_star = has_B ? fH[Sn] + bgs * bgs - vc * (fH[ORC_TAU] + fH[ORC_D] - BG * vsBs)
                                : fH[Sn] - vc * (fH[ORC_TAU] + fH[ORC_D]);
    /* star states */
    double uc[2][ORC_NCONS], fs[2][ORC_NCONS];
    for (int side = 0; side < 2; ++side) {
        const side_t *sd = side == 0 ? &ph.L : &ph.R;
        const double SK = side == 0 ? S_L : S_R;
        const double vdK = (side == 0 ? PL : PR)[ORC_VX + idir];
        const double denom = SK - vc;
        double *c = uc[side];
        c[Bn] = BG;
        c[B1] = uH[B1];
        c[B2] = uH[B2];
        c[ORC_D] = sdiv(sd->u[ORC_D] * (SK - vdK), denom);
        c[ORC_TAU] = sdiv(SK * sd->u[ORC_TAU] - sd->f[ORC_TAU] + p_star * vc - vsBs * BG, denom);
        c[Sn] = (c[ORC_TAU] + c[ORC_D] + p_star) * vc - vsBs * BG;
        const double gs2 = gs * gs;
        const double St1B = sdiv(-BG * (uH[B1] / gs2 + vsBs * vt1) - sd->f[S1] + SK * sd->u[S1], denom);
        const double St2B = sdiv(-BG * (uH[B2] / gs2 + vsBs * vt2) - sd->f[S2] + SK * sd->u[S2], denom);
        const double St10 = sdiv(sd->u[S1] * (SK - vdK), denom);
        const double St20 = sdiv(sd->u[S2] * (SK - vdK), denom);
        c[S1] = has_B ? St1B : St10;
        c[S2] = has_B ? St2B : St20;
        for (int k = 0; k < ORC_NCONS; ++k) fs[side][k] = sd->f[k] + SK * (c[k] - sd->u[k]);
    }
    /* region at xi = 0, then the degenerate / superluminal and non-finite
     * fallbacks to the HLL state */
    const int degen = (vc <= S_L) || (vc >= S_R) || (v2 >= 1.0);
    for (int k = 0; k < ORC_NCONS; ++k) {
        double f = fH[k], u = uH[k];
        if (0.0 <= S_L) { f = ph.L.f[k]; u = ph.L.u[k]; }
        if (S_L < 0.0 && 0.0 < vc) { f = fs[0][k]; u = uc[0][k]; }
        if (vc <= 0.0 && 0.0 < S_R) { f = fs[1][k]; u = uc[1][k]; }
        if (0.0 >= S_R) { f = ph.R.f[k]; u = ph.R.u[k]; }
        if (degen) { f = fH[k]; u = uH[k]; }
        if (!isfinite(f) || !isfinite(u)) { f = fH[k]; u = uH[k]; }
        F[k] = f;
        U[k] = u;
    }
    *pstar = hlle_p_estimate(PL, PR, gamma);
}

static void riemann_one(const double *PL, const double *PR, int idir, int solver, double gamma,
                        double *F, double *U, double *pstar, int32_t *err, int32_t *iters,
                        uint8_t *flags) {
    if (solver == ORC_SOLVER_HLLD) {
        hlld_one(PL, PR, idir, gamma, F, U, pstar, err, iters, flags);
    } else if (solver == ORC_SOLVER_HLLC) {
        hllc_one(PL, PR, idir, gamma, F, U, pstar);
        if (err) *err = 0;
        if (iters) *iters = 0;
        if (flags) *flags = 0;
    } else {
        hlle_one(PL, PR, idir, gamma, F, U, pstar);
        if (err) *err = 0;
        if (iters) *iters = 0;
        if (flags) *flags = 0;
    }
}

void orc_riemann(int64_t n, const double *const *sL, const double *const *sR, int idir,
                 int solver, double gamma, double *const *F, double *const *U, double *pstar,
                 int32_t *err, int32_t *iters, uint8_t *flags) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t e = 0; e < n; ++e) {
        double PL[ORC_NPRIM], PR[ORC_NPRIM], f[ORC_NCONS], u[ORC_NCONS], ps;
        int32_t er, itn;
        uint8_t fl;
        for (int k = 0; k < ORC_NPRIM; ++k) {
            PL[k] = sL[k][e];
            PR[k] = sR[k][e];
        }
        riemann_one(PL, PR, idir, solver, gamma, f, u, &ps, &er, &itn, &fl);
        for (int k = 0; k < ORC_NCONS; ++k) {
            F[k][e] = f[k];
            U[k][e] = u[k];
        }
        pstar[e] = ps;
        if (err) err[e] = er;
        if (iters) iters[e] = itn;
        if (flags) flags[e] = fl;
    }
}

/* ── reconstruction (reconstruction.py) ───────────────────────────────── */

/* reconstruction.py:60-66 */
static inline double minmod(double a, double b) {
    return (a * b > 0.0) ? ((fabs(a) < fabs(b)) ? a : b) : 0.0;
}
/* reconstruction.py:69-77 */
static inline double mc_lim(double a, double b) {
    double c = 0.5 * (a + b);
    return (a * b > 0.0) ? tsign(c) * tmin(2.0 * fabs(a), tmin(2.0 * fabs(b), fabs(c))) : 0.0;
}

/* reconstruction.py:111-128, value at the right face of the centre cell */
static double weno5z(double vm2, double vm1, double v0, double vp1, double vp2) {
    double p0 = (2.0 * vm2 - 7.0 * vm1 + 11.0 * v0) / 6.0;
    double p1 = (-vm1 + 5.0 * v0 + 2.0 * vp1) / 6.0;
    double p2 = (2.0 * v0 + 5.0 * vp1 - vp2) / 6.0;
    double c1 = 13.0 / 12.0, c2 = 0.25;
    double t;
    double b0 = (t = vm2 - 2.0 * vm1 + v0, c1 * (t * t));
    double u = vm2 - 4.0 * vm1 + 3.0 * v0;
    b0 = b0 + c2 * (u * u);
    double b1 = (t = vm1 - 2.0 * v0 + vp1, c1 * (t * t));
    u = vm1 - vp1;
    b1 = b1 + c2 * (u * u);
    double b2 = (t = v0 - 2.0 * vp1 + vp2, c1 * (t * t));
    u = 3.0 * v0 - 4.0 * vp1 + vp2;
    b2 = b2 + c2 * (u * u);
    double tau5 = fabs(b0 - b2);
    double eps = 1e-40;
    double r0 = tau5 / (b0 + eps), r1 = tau5 / (b1 + eps), r2 = tau5 / (b2 + eps);
    double a0 = 0.1 * (1.0 + r0 * r0);
    double a1 = 0.6 * (1.0 + r1 * r1);
    double a2 = 0.3 * (1.0 + r2 * r2);
    return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2);
}

/* reconstruction.py:136-162 */
static double mp_limit(double vl, double vm2, double vm1, double v0, double vp1, double vp2) {
    const double alpha = 4.0;
    double vmp = v0 + minmod(vp1 - v0, alpha * (v0 - vm1));
    int need = (vl - v0) * (vl - vmp) > 1e-40;
    double d_m1 = vm2 - 2.0 * vm1 + v0;
    double d_0 = vm1 - 2.0 * v0 + vp1;
    double d_p1 = v0 - 2.0 * vp1 + vp2;
    double dm4_p = minmod(minmod(4.0 * d_0 - d_p1, 4.0 * d_p1 - d_0), minmod(d_0, d_p1));
    double dm4_m = minmod(minmod(4.0 * d_m1 - d_0, 4.0 * d_0 - d_m1), minmod(d_m1, d_0));
    double v_ul = v0 + alpha * (v0 - vm1);
    double v_av = 0.5 * (v0 + vp1);
    double v_md = v_av - 0.5 * dm4_p;
    double v_lc = v0 + 0.5 * (v0 - vm1) + (4.0 / 3.0) * dm4_m;
    double vmin = tmax(tmin(tmin(v0, vp1), v_md), tmin(tmin(v0, v_ul), v_lc));
    double vmax = tmin(tmax(tmax(v0, vp1), v_md), tmax(tmax(v0, v_ul), v_lc));
    /* _median(a, b, c) = a + minmod(b - a, c - a) (reconstruction.py:131-133) */
    return need ? vl + minmod(vmin - vl, vmax - vl) : vl;
}

/* reconstruction.py:165-168 */
static double mp5(double vm2, double vm1, double v0, double vp1, double vp2) {
    double vl = (2.0 * vm2 - 13.0 * vm1 + 47.0 * v0 + 27.0 * vp1 - 3.0 * vp2) / 60.0;
    return mp_limit(vl, vm2, vm1, v0, vp1, vp2);
}
/* reconstruction.py:171-176 */
static double mp7(double vm3, double vm2, double vm1, double v0, double vp1, double vp2,
                  double vp3) {
    double vl = (-3.0 * vm3 + 25.0 * vm2 - 101.0 * vm1 + 319.0 * v0 + 214.0 * vp1 - 38.0 * vp2 +
                 4.0 * vp3) /
                420.0;
    return mp_limit(vl, vm2, vm1, v0, vp1, vp2);
}

static int lim_stencil(int limiter) {
    switch (limiter) {
    case ORC_LIM_PCM: return 0;
    case ORC_LIM_MC:
    case ORC_LIM_MINMOD: return 1;
    case ORC_LIM_WENO5Z:
    case ORC_LIM_MP5: return 2;
    default: return 3;
    }
}

/* cell edges of one line of n values q[0..n) with stride s:
 * re[c] = value at the right face of cell c, le[c] at its left face
 * (reconstruction.py:182-213, :225-264) */
static void line_edges(const double *q, int64_t s, int n, int limiter, double *re, double *le) {
    if (limiter == ORC_LIM_PCM) {
        /* slope = zeros_like(Q): left = Q + 0.5*0, right = Q - 0.5*0 */
        for (int c = 0; c < n; ++c) {
            re[c] = q[c * s] + 0.5 * 0.0;
            le[c] = q[c * s] - 0.5 * 0.0;
        }
        return;
    }
    int plm_lim = (limiter == ORC_LIM_MINMOD) ? ORC_LIM_MINMOD : ORC_LIM_MC;
    /* PLM (MC for the high-order edge fallback, reconstruction.py:201) */
    for (int c = 0; c < n; ++c) {
        double slope = 0.0;
        if (c >= 1 && c <= n - 2) {
            double a = q[c * s] - q[(c - 1) * s];
            double b = q[(c + 1) * s] - q[c * s];
            slope = (plm_lim == ORC_LIM_MINMOD) ? minmod(a, b) : mc_lim(a, b);
        }
        re[c] = q[c * s] + 0.5 * slope;
        le[c] = q[c * s] - 0.5 * slope;
    }
    if (limiter == ORC_LIM_MC || limiter == ORC_LIM_MINMOD) return;
    int w = lim_stencil(limiter);
    if (n <= 2 * w) return;
    for (int c = w; c < n - w; ++c) {
#define Q(k) q[(int64_t)(c + (k)) * s]
        if (limiter == ORC_LIM_WENO5Z) {
            re[c] = weno5z(Q(-2), Q(-1), Q(0), Q(1), Q(2));
            le[c] = weno5z(Q(2), Q(1), Q(0), Q(-1), Q(-2));
        } else if (limiter == ORC_LIM_MP5) {
            re[c] = mp5(Q(-2), Q(-1), Q(0), Q(1), Q(2));
            le[c] = mp5(Q(2), Q(1), Q(0), Q(-1), Q(-2));
        } else {
            re[c] = mp7(Q(-3), Q(-2), Q(-1), Q(0), Q(1), Q(2), Q(3));
            le[c] = mp7(Q(3), Q(2), Q(1), Q(0), Q(-1), Q(-2), Q(-3));
        }
#undef Q
    }
}

void orc_reconstruct(const double *q, int n0, int n1, int axis, int limiter, double *QL,
                     double *QR) {
    int n = axis == 0 ? n0 : n1;
    int nlines = axis == 0 ? n1 : n0;
    int64_t s = axis == 0 ? n1 : 1;
    /* face arrays: axis 0 -> (n0+1, n1); axis 1 -> (n0, n1+1) */
    int64_t fs = axis == 0 ? n1 : 1;
#pragma omp parallel
    {
        double *re = (double *)malloc(sizeof(double) * (size_t)n);
        double *le = (double *)malloc(sizeof(double) * (size_t)n);
#pragma omp for schedule(static)
        for (int l = 0; l < nlines; ++l) {
            const double *ql = axis == 0 ? q + l : q + (int64_t)l * n1;
            int64_t fo = axis == 0 ? l : (int64_t)l * (n1 + 1);
            line_edges(ql, s, n, limiter, re, le);
            for (int f = 0; f <= n; ++f) {
                QL[fo + f * fs] = (f == 0) ? re[0] : re[f - 1];
                QR[fo + f * fs] = (f == n) ? le[n - 1] : le[f];
            }
        }
        free(re);
        free(le);
    }
}

/* reconstruction.py:272-338 on whole arrays */
void orc_reconstruct_prims(const double *const *prim, int n0, int n1, int axis, int limiter,
                           int wv, double gamma, double *const *L, double *const *R) {
    int64_t nc = (int64_t)n0 * n1;
    int64_t nf = axis == 0 ? (int64_t)(n0 + 1) * n1 : (int64_t)n0 * (n1 + 1);
    /* work variables in reconstruction.py:269 order */
    static const int wk[8] = {ORC_RHO, ORC_P, ORC_VX, ORC_VY, ORC_VZ, ORC_PBX, ORC_PBY, ORC_PBZ};
    double *work[8];
    for (int k = 0; k < 8; ++k) work[k] = (double *)malloc(sizeof(double) * (size_t)nc);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < nc; ++e) {
        double vx = prim[ORC_VX][e], vy = prim[ORC_VY][e], vz = prim[ORC_VZ][e];
        double W = 1.0;
        if (wv) {
            double v2 = vx * vx + vy * vy + vz * vz;
            W = 1.0 / sqrt(clamp_lo(1.0 - v2, 1e-14));
        }
        for (int k = 0; k < 8; ++k) {
            double x = prim[wk[k]][e];
            if (wv && (wk[k] == ORC_VX || wk[k] == ORC_VY || wk[k] == ORC_VZ)) x = W * x;
            work[k][e] = x;
        }
    }
    double *l8[8], *r8[8];
    for (int k = 0; k < 8; ++k) {
        l8[k] = L[wk[k]];
        r8[k] = R[wk[k]];
        orc_reconstruct(work[k], n0, n1, axis, limiter, l8[k], r8[k]);
    }
    if (limiter != ORC_LIM_PCM) {
        double *cl = (double *)malloc(sizeof(double) * (size_t)nf);
        double *cr = (double *)malloc(sizeof(double) * (size_t)nf);
        uint8_t *bad = (uint8_t *)malloc((size_t)nf);
        for (int64_t f = 0; f < nf; ++f)
            bad[f] = (l8[0][f] <= 1e-12) || (r8[0][f] <= 1e-12) || (l8[1][f] <= 1e-14) ||
                     (r8[1][f] <= 1e-14);
        for (int k = 0; k < 8; ++k) {
            orc_reconstruct(work[k], n0, n1, axis, ORC_LIM_PCM, cl, cr);
            for (int64_t f = 0; f < nf; ++f)
                if (bad[f]) {
                    l8[k][f] = cl[f];
                    r8[k][f] = cr[f];
                }
        }
        free(cl);
        free(cr);
        free(bad);
    }
    for (int side = 0; side < 2; ++side) {
        double *const *S = side == 0 ? L : R;
#pragma omp parallel for schedule(static)
        for (int64_t f = 0; f < nf; ++f) {
            if (wv) {
                double zx = S[ORC_VX][f], zy = S[ORC_VY][f], zz = S[ORC_VZ][f];
                double z2 = zx * zx + zy * zy + zz * zz;
                double fac = 1.0 / sqrt(1.0 + z2);
                S[ORC_VX][f] = zx * fac;
                S[ORC_VY][f] = zy * fac;
                S[ORC_VZ][f] = zz * fac;
            }
            S[ORC_RHO][f] = clamp_lo(S[ORC_RHO][f], 1e-12);
            S[ORC_P][f] = clamp_lo(S[ORC_P][f], 1e-14);
            S[ORC_EPS][f] = eos_eps(S[ORC_P][f], S[ORC_RHO][f], gamma);
        }
    }
    for (int k = 0; k < 8; ++k) free(work[k]);
}

/* ── constrained transport (ct.py) ────────────────────────────────────── */

/* ct.py:96-116 with the sweep-global scale */
static inline double upwind_sign(double F, double scale) {
    return (fabs(F) > 1e-9 * scale) ? tsign(F) : 0.0;
}

static double absmax(const double *a, int64_t n) {
    double m = 0.0;
    int first = 1;
    for (int64_t i = 0; i < n; ++i) {
        double v = fabs(a[i]);
        if (isnan(v)) return v;
        if (first || v > m) m = v;
        first = 0;
    }
    return m;
}

void orc_corner_emf(int n0, int n1, const double *Ec, const double *Efx, const double *Efy,
                    const double *Fx_rho, const double *Fy_rho, int upwind, double *Ez) {
    int64_t N1 = n1 + 1;
    memset(Ez, 0, sizeof(double) * (size_t)(n0 + 1) * (size_t)N1);
    double sx = upwind ? absmax(Fx_rho, (int64_t)(n0 + 1) * n1) : 0.0;
    double sy = upwind ? absmax(Fy_rho, (int64_t)n0 * (n1 + 1)) : 0.0;
#pragma omp parallel for schedule(static)
    for (int i = 1; i < n0; ++i)
        for (int j = 1; j < n1; ++j) {
            /* Efy (n0, n1+1); Efx (n0+1, n1); Ec (n0, n1) */
            double Ezyf = Efy[(int64_t)i * N1 + j];
            double Ezyfm = Efy[(int64_t)(i - 1) * N1 + j];
            double Ezxf = Efx[(int64_t)i * n1 + j];
            double Ezxfm = Efx[(int64_t)i * n1 + j - 1];
            double EzNE = Ec[(int64_t)i * n1 + j];
            double EzNW = Ec[(int64_t)(i - 1) * n1 + j];
            double EzSE = Ec[(int64_t)i * n1 + j - 1];
            double EzSW = Ec[(int64_t)(i - 1) * n1 + j - 1];
            double Eavg = 0.25 * ((Ezyf + Ezyfm) + (Ezxf + Ezxfm));
            double val;
            if (upwind) {
                double Sx = upwind_sign(Fx_rho[(int64_t)i * n1 + j], sx);
                double Sxm = upwind_sign(Fx_rho[(int64_t)i * n1 + j - 1], sx);
                double dEdyN = (1.0 - Sx) * (EzNE - Ezyf) + (1.0 + Sx) * (EzNW - Ezyfm);
                double dEdyS = (1.0 - Sxm) * (Ezyf - EzSE) + (1.0 + Sxm) * (Ezyfm - EzSW);
                double dEdy = 0.125 * (dEdyS - dEdyN);
                double Sy = upwind_sign(Fy_rho[(int64_t)i * N1 + j], sy);
                double Sym = upwind_sign(Fy_rho[(int64_t)(i - 1) * N1 + j], sy);
                double dEdxE = (1.0 - Sy) * (EzNE - Ezxf) + (1.0 + Sy) * (EzSE - Ezxfm);
                double dEdxW = (1.0 - Sym) * (Ezxf - EzNW) + (1.0 + Sym) * (Ezxfm - EzSW);
                double dEdx = 0.125 * (dEdxW - dEdxE);
                val = Eavg + (dEdy + dEdx);
            } else {
                val = Eavg;
            }
            Ez[(int64_t)i * N1 + j] = val;
        }
}

/* ── grid boundary conditions (grid.py:93-143, :229-255) ──────────────── */

/* source index along an axis of a cell-centred array (grid.py:93-113) */
static inline int bc_cc_src(int idx, int n, int ng, int kind) {
    if (idx >= ng && idx < ng + n) return idx;
    if (kind == ORC_BC_OUTFLOW) return idx < ng ? ng : ng + n - 1;
    /* periodic: v[:ng] = v[n:n+ng]; v[n+ng:] = v[ng:2ng] */
    return idx < ng ? idx + n : idx - n;
}
/* source index along the normal axis of a face array (grid.py:116-143) */
static inline int bc_face_src(int idx, int n, int ng, int kind) {
    if (kind == ORC_BC_OUTFLOW) {
        if (idx < ng) return ng;
        if (idx > ng + n) return ng + n;
        return idx;
    }
    if (idx == ng + n) return ng; /* seam collapse */
    if (idx < ng) return idx + n;
    if (idx > ng + n) return idx - n;
    return idx;
}

/* apply a separable ghost map to an (n0, n1) array in place */
static void apply_map(double *v, int n0, int n1, const int *m0, const int *m1) {
    double *tmp = (double *)malloc(sizeof(double) * (size_t)n0 * (size_t)n1);
    memcpy(tmp, v, sizeof(double) * (size_t)n0 * (size_t)n1);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n0; ++i)
        for (int j = 0; j < n1; ++j) v[(int64_t)i * n1 + j] = tmp[(int64_t)m0[i] * n1 + m1[j]];
    free(tmp);
}

static void bc_cc(const orc_grid2d *g, double *v) {
    int nxt = g->nx + 2 * g->ng, nyt = g->ny + 2 * g->ng;
    int *mx = (int *)malloc(sizeof(int) * nxt), *my = (int *)malloc(sizeof(int) * nyt);
    for (int i = 0; i < nxt; ++i) mx[i] = bc_cc_src(i, g->nx, g->ng, g->bc_x);
    for (int j = 0; j < nyt; ++j) my[j] = bc_cc_src(j, g->ny, g->ng, g->bc_y);
    apply_map(v, nxt, nyt, mx, my);
    free(mx);
    free(my);
}

static void bc_face(const orc_grid2d *g, double *Bxf, double *Byf) {
    int nxt = g->nx + 2 * g->ng, nyt = g->ny + 2 * g->ng;
    int *mx = (int *)malloc(sizeof(int) * (nxt + 1)), *my = (int *)malloc(sizeof(int) * (nyt + 1));
    for (int i = 0; i <= nxt; ++i) mx[i] = bc_face_src(i, g->nx, g->ng, g->bc_x);
    for (int j = 0; j < nyt; ++j) my[j] = bc_cc_src(j, g->ny, g->ng, g->bc_y);
    apply_map(Bxf, nxt + 1, nyt, mx, my);
    for (int i = 0; i < nxt; ++i) mx[i] = bc_cc_src(i, g->nx, g->ng, g->bc_x);
    for (int j = 0; j <= nyt; ++j) my[j] = bc_face_src(j, g->ny, g->ng, g->bc_y);
    apply_map(Byf, nxt, nyt + 1, mx, my);
    free(mx);
    free(my);
}

/* ct.py:44-54 */
static void cell_centred_B(int nxt, int nyt, const double *Bxf, const double *Byf, double *Bcx,
                           double *Bcy) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nxt; ++i)
        for (int j = 0; j < nyt; ++j) {
            Bcx[(int64_t)i * nyt + j] = 0.5 * (Bxf[(int64_t)i * nyt + j] + Bxf[(int64_t)(i + 1) * nyt + j]);
            Bcy[(int64_t)i * nyt + j] =
                0.5 * (Byf[(int64_t)i * (nyt + 1) + j] + Byf[(int64_t)i * (nyt + 1) + j + 1]);
        }
}

/* state.py:41 EVOLVED_KEYS -> conserved component */
static const int EVOLVED[6] = {ORC_D, ORC_SX, ORC_SY, ORC_SZ, ORC_TAU, ORC_BZ};

void orc_sync_state(const orc_grid2d *g, double *const *cons, double *Bxf, double *Byf,
                    double *const *prim, uint8_t *status) {
    int nxt = g->nx + 2 * g->ng, nyt = g->ny + 2 * g->ng;
    int64_t nc = (int64_t)nxt * nyt;
    bc_face(g, Bxf, Byf);
    for (int k = 0; k < 6; ++k) bc_cc(g, cons[k]);
    double *Bcx = (double *)malloc(sizeof(double) * (size_t)nc);
    double *Bcy = (double *)malloc(sizeof(double) * (size_t)nc);
    cell_centred_B(nxt, nyt, Bxf, Byf, Bcx, Bcy);
    const double *C8[ORC_NCONS] = {cons[0], cons[1], cons[2], cons[3], cons[4], Bcx, Bcy, cons[5]};
    orc_cons_to_prim(nc, C8, g->gamma, g->atmo_rho, 1e-10, prim, status);
    memcpy(prim[ORC_PBX], Bcx, sizeof(double) * (size_t)nc);
    memcpy(prim[ORC_PBY], Bcy, sizeof(double) * (size_t)nc);
    memcpy(prim[ORC_PBZ], cons[5], sizeof(double) * (size_t)nc);
    for (int k = 0; k < ORC_NPRIM; ++k) bc_cc(g, prim[k]);
    free(Bcx);
    free(Bcy);
}

/* one directional sweep (sweep.py:30-119): face fluxes for all faces */
/* sweep.py:30-119; Fbt_hll (may be NULL): the HLL average of the
 * transverse-B flux per face for emf_mode "hll" (sweep.py:106-119 with
 * ct.py:63-96 _hll) */
static void sweep2d(const orc_grid2d *g, const double *const *prims, const double *Bnf, int axis,
                    double *const *F, orc_step_diag *diag, double *Fbt_hll) {
    int nxt = g->nx + 2 * g->ng, nyt = g->ny + 2 * g->ng;
    int64_t nf = axis == 0 ? (int64_t)(nxt + 1) * nyt : (int64_t)nxt * (nyt + 1);
    double *L[ORC_NPRIM], *R[ORC_NPRIM], *U[ORC_NCONS];
    for (int k = 0; k < ORC_NPRIM; ++k) {
        L[k] = (double *)malloc(sizeof(double) * (size_t)nf);
        R[k] = (double *)malloc(sizeof(double) * (size_t)nf);
    }
    for (int k = 0; k < ORC_NCONS; ++k) U[k] = (double *)malloc(sizeof(double) * (size_t)nf);
    orc_reconstruct_prims(prims, nxt, nyt, axis, g->limiter, 1, g->gamma, L, R);
    int bk = axis == 0 ? ORC_PBX : ORC_PBY;
    memcpy(L[bk], Bnf, sizeof(double) * (size_t)nf);
    memcpy(R[bk], Bnf, sizeof(double) * (size_t)nf);
    double *ps = (double *)malloc(sizeof(double) * (size_t)nf);
    int32_t *er = (int32_t *)malloc(sizeof(int32_t) * (size_t)nf);
    int32_t *it = (int32_t *)malloc(sizeof(int32_t) * (size_t)nf);
    uint8_t *fl = (uint8_t *)malloc((size_t)nf);
    orc_riemann(nf, (const double *const *)L, (const double *const *)R, axis, g->solver, g->gamma,
                F, U, ps, er, it, fl);
    /* sweep.py:99-100 freeze_normal_B */
    memset(F[ORC_BX + axis], 0, sizeof(double) * (size_t)nf);
    if (Fbt_hll) {
        const int kb = axis == 0 ? ORC_BY : ORC_BX;
        for (int64_t f = 0; f < nf; ++f) {
            double PL[ORC_NPRIM], PR[ORC_NPRIM];
            for (int k = 0; k < ORC_NPRIM; ++k) {
                PL[k] = L[k][f];
                PR[k] = R[k][f];
            }
            phys_t ph;
            compute_srmhd_fluxes(PL, PR, axis, g->gamma, &ph);
            Fbt_hll[f] = hf(ph.L.f[kb], ph.R.f[kb], ph.L.u[kb], ph.R.u[kb], ph.cmin, ph.cmax);
        }
    }
    if (diag) {
        int64_t nnc = 0, nwb = 0, nbz = 0, nfl = 0, isum = 0, nconv = 0, imax = 0;
        for (int64_t f = 0; f < nf; ++f) {
            if (er[f] > 0) nnc++;
            else {
                nconv++;
                isum += it[f];
            }
            if (fl[f] & ORC_RF_WAVE_ORDER_BAD) nwb++;
            if (fl[f] & ORC_RF_BN_ZERO) nbz++;
            if (fl[f] & ORC_RF_FAILED) nfl++;
            if (it[f] > imax) imax = it[f];
        }
        diag->n_faces[axis] = nf;
        diag->n_not_converged[axis] = nnc;
        diag->n_wave_order_bad[axis] = nwb;
        diag->n_bn_zero[axis] = nbz;
        diag->n_failed[axis] = nfl;
        diag->iters_sum_conv[axis] = isum;
        diag->n_conv[axis] = nconv;
        diag->max_iters[axis] = imax;
        diag->fd_max[axis] = absmax(F[ORC_D], nf);
    }
    for (int k = 0; k < ORC_NPRIM; ++k) {
        free(L[k]);
        free(R[k]);
    }
    for (int k = 0; k < ORC_NCONS; ++k) free(U[k]);
    free(ps);
    free(er);
    free(it);
    free(fl);
}

/* driver2d.py:104-105 */
static const double RK3[3][3] = {{1.0, 0.0, 1.0}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
static const double RK2[2][3] = {{1.0, 0.0, 1.0}, {0.5, 0.5, 0.5}};

int orc_rk_step_ct(const orc_grid2d *g, double dt, int scheme, double *const *cons, double *Bxf,
                   double *Byf, double *const *prim, orc_step_diag *diag) {
    if (scheme != 2 && scheme != 3) return -1;
    int nxt = g->nx + 2 * g->ng, nyt = g->ny + 2 * g->ng;
    int64_t nc = (int64_t)nxt * nyt, nfx = (int64_t)(nxt + 1) * nyt, nfy = (int64_t)nxt * (nyt + 1);
    int64_t ncr = (int64_t)(nxt + 1) * (nyt + 1);
    int nst = scheme;
    const double(*tab)[3] = scheme == 3 ? RK3 : RK2;
    /* S0 = clone (driver2d.py:235-237) */
    double *U0[6], *Fx[ORC_NCONS], *Fy[ORC_NCONS];
    for (int k = 0; k < 6; ++k) {
        U0[k] = (double *)malloc(sizeof(double) * (size_t)nc);
        memcpy(U0[k], cons[k], sizeof(double) * (size_t)nc);
    }
    double *Bx0 = (double *)malloc(sizeof(double) * (size_t)nfx);
    double *By0 = (double *)malloc(sizeof(double) * (size_t)nfy);
    memcpy(Bx0, Bxf, sizeof(double) * (size_t)nfx);
    memcpy(By0, Byf, sizeof(double) * (size_t)nfy);
    for (int k = 0; k < ORC_NCONS; ++k) {
        Fx[k] = (double *)malloc(sizeof(double) * (size_t)nfx);
        Fy[k] = (double *)malloc(sizeof(double) * (size_t)nfy);
    }
    double *Bcx = (double *)malloc(sizeof(double) * (size_t)nc);
    double *Bcy = (double *)malloc(sizeof(double) * (size_t)nc);
    double *Ec = (double *)malloc(sizeof(double) * (size_t)nc);
    double *Efx = (double *)malloc(sizeof(double) * (size_t)nfx);
    double *Efy = (double *)malloc(sizeof(double) * (size_t)nfy);
    double *Ez = (double *)malloc(sizeof(double) * (size_t)ncr);
    double *pw[ORC_NPRIM];
    for (int k = 0; k < ORC_NPRIM; ++k) pw[k] = (double *)malloc(sizeof(double) * (size_t)nc);

    for (int st = 0; st < nst; ++st) {
        double a = tab[st][0], b = tab[st][1], c = tab[st][2];
        /* ct_stage (driver2d.py:162-193) */
        cell_centred_B(nxt, nyt, Bxf, Byf, Bcx, Bcy);
        for (int k = 0; k < ORC_NPRIM; ++k) memcpy(pw[k], prim[k], sizeof(double) * (size_t)nc);
        memcpy(pw[ORC_PBX], Bcx, sizeof(double) * (size_t)nc);
        memcpy(pw[ORC_PBY], Bcy, sizeof(double) * (size_t)nc);
        for (int64_t e = 0; e < nc; ++e) Ec[e] = Bcx[e] * pw[ORC_VY][e] - Bcy[e] * pw[ORC_VX][e];
        /* ct.py:63-88 face_emf_x / face_emf_y */
        const int hll = g->emf_mode == 1;
        sweep2d(g, (const double *const *)pw, Bxf, 0, Fx, diag, hll ? Efx : NULL);
        sweep2d(g, (const double *const *)pw, Byf, 1, Fy, diag, hll ? Efy : NULL);
        for (int64_t e = 0; e < nfx; ++e) Efx[e] = -(hll ? Efx[e] : Fx[ORC_BY][e]);
        if (!hll)
            for (int64_t e = 0; e < nfy; ++e) Efy[e] = Fy[ORC_BX][e];
        orc_corner_emf(nxt, nyt, Ec, Efx, Efy, Fx[ORC_D], Fy[ORC_D], g->upwind, Ez);
        /* flux divergence + ct_rhs + combine (sweep.py:122-135, ct.py:180-185,
         * state.py:77-103); L is computed on the fly */
        double w2 = c * dt;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nxt; ++i)
            for (int j = 0; j < nyt; ++j) {
                int64_t e = (int64_t)i * nyt + j;
                for (int k = 0; k < 6; ++k) {
                    int ck = EVOLVED[k];
                    double rx = -(Fx[ck][(int64_t)(i + 1) * nyt + j] - Fx[ck][e]) / g->dx;
                    double ry = -(Fy[ck][(int64_t)i * (nyt + 1) + j + 1] -
                                  Fy[ck][(int64_t)i * (nyt + 1) + j]) /
                                g->dy;
                    double L = rx + ry;
                    double v = a * U0[k][e];
                    v = v + b * cons[k][e];
                    v = v + w2 * L;
                    cons[k][e] = v;
                }
            }
#pragma omp parallel for schedule(static)
        for (int i = 0; i <= nxt; ++i)
            for (int j = 0; j < nyt; ++j) {
                int64_t e = (int64_t)i * nyt + j;
                double dB = (Ez[(int64_t)i * (nyt + 1) + j] - Ez[(int64_t)i * (nyt + 1) + j + 1]) / g->dy;
                double v = a * Bx0[e];
                v = v + b * Bxf[e];
                v = v + w2 * dB;
                Bxf[e] = v;
            }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nxt; ++i)
            for (int j = 0; j <= nyt; ++j) {
                int64_t e = (int64_t)i * (nyt + 1) + j;
                double dB = (Ez[(int64_t)(i + 1) * (nyt + 1) + j] - Ez[(int64_t)i * (nyt + 1) + j]) / g->dx;
                double v = a * By0[e];
                v = v + b * Byf[e];
                v = v + w2 * dB;
                Byf[e] = v;
            }
        orc_sync_state(g, cons, Bxf, Byf, prim, NULL);
    }
    for (int k = 0; k < 6; ++k) free(U0[k]);
    for (int k = 0; k < ORC_NCONS; ++k) {
        free(Fx[k]);
        free(Fy[k]);
    }
    for (int k = 0; k < ORC_NPRIM; ++k) free(pw[k]);
    free(Bx0); free(By0); free(Bcx); free(Bcy); free(Ec); free(Efx); free(Efy); free(Ez);
    return 0;
}

double orc_compute_dt_2d(const orc_grid2d *g, const double *const *prim, double cfl) {
    int nyt = g->ny + 2 * g->ng;
    double mx = 0.0, my = 0.0;
    int first = 1, nan_seen = 0;
    for (int i = g->ng; i < g->ng + g->nx; ++i)
        for (int j = g->ng; j < g->ng + g->ny; ++j) {
            int64_t e = (int64_t)i * nyt + j;
            double rho = prim[ORC_RHO][e], eps = prim[ORC_EPS][e];
            double vx = prim[ORC_VX][e], vy = prim[ORC_VY][e], vz = prim[ORC_VZ][e];
            double Bx = prim[ORC_PBX][e], By = prim[ORC_PBY][e], Bz = prim[ORC_PBZ][e];
            double p, cs2;
            eos_press_cs2(eps, rho, g->gamma, &p, &cs2);
            double v2 = vx * vx + vy * vy + vz * vz;
            double W = 1.0 / sqrt(clamp_lo(1.0 - v2, 1e-10));
            double B2 = Bx * Bx + By * By + Bz * Bz;
            double vdotB = vx * Bx + vy * By + vz * Bz;
            double b2 = (B2 + vdotB * vdotB) / (W * W);
            double h = 1.0 + eps + p / rho;
            double v02 = cs2 + (b2 / (rho * h + b2)) * (1.0 - cs2);
            double cf = sqrt(clamp_hi(clamp_lo(v02, 0.0), 1.0));
            double sxv = fabs(vx) + cf, syv = fabs(vy) + cf;
            if (isnan(sxv) || isnan(syv)) nan_seen = 1;
            if (first || sxv > mx) mx = sxv;
            if (first || syv > my) my = syv;
            first = 0;
        }
    if (nan_seen) return NAN;
    double sx = clamp_lo(mx, 1e-14), sy = clamp_lo(my, 1e-14);
    /* `cfl / tensor` is torch's reciprocal(tensor) * cfl */
    return (1.0 / (sx / g->dx + sy / g->dy)) * cfl;
}

/* ── 1D shock-tube driver (driver.py:135-236) ─────────────────────────── */

static void rhs_1d(int ncells, int ng, double dx, int limiter, int solver, double gamma,
                   const double *const *prim, double *const *rhs) {
    int nt = ncells + 2 * ng;
    int nf = ncells + 1;
    /* get_interface_states (reconstruction.py:354-373): all nine primitives */
    double *QL[ORC_NPRIM], *QR[ORC_NPRIM], *sl[ORC_NPRIM], *sr[ORC_NPRIM];
    for (int k = 0; k < ORC_NPRIM; ++k) {
        QL[k] = (double *)malloc(sizeof(double) * (nt + 1));
        QR[k] = (double *)malloc(sizeof(double) * (nt + 1));
        orc_reconstruct(prim[k], nt, 1, 0, limiter, QL[k], QR[k]);
        sl[k] = QL[k] + ng;
        sr[k] = QR[k] + ng;
    }
    double *F[ORC_NCONS], *U[ORC_NCONS];
    for (int k = 0; k < ORC_NCONS; ++k) {
        F[k] = (double *)malloc(sizeof(double) * nf);
        U[k] = (double *)malloc(sizeof(double) * nf);
    }
    double *ps = (double *)malloc(sizeof(double) * nf);
    orc_riemann(nf, (const double *const *)sl, (const double *const *)sr, 0, solver, gamma, F, U,
                ps, NULL, NULL, NULL);
    for (int e = 0; e < nf; ++e) F[ORC_BX][e] = 0.0; /* driver.py:171 */
    for (int k = 0; k < ORC_NCONS; ++k) {
        for (int e = 0; e < nt; ++e) rhs[k][e] = 0.0;
        for (int c = 0; c < ncells; ++c) rhs[k][ng + c] = +((F[k][c] - F[k][c + 1]) / dx);
    }
    for (int k = 0; k < ORC_NPRIM; ++k) {
        free(QL[k]);
        free(QR[k]);
    }
    for (int k = 0; k < ORC_NCONS; ++k) {
        free(F[k]);
        free(U[k]);
    }
    free(ps);
}

/* grid.py:49-62 apply_outflow_bc */
static void outflow_1d(double *v, int ncells, int ng) {
    for (int e = 0; e < ng; ++e) v[e] = v[ng];
    for (int e = ng + ncells; e < ncells + 2 * ng; ++e) v[e] = v[ng + ncells - 1];
}

void orc_rk2_step_1d(int ncells, int ng, double dx, double dt, int limiter, int solver,
                     double gamma, double atmo_rho, double *const *cons, double *const *prim) {
    int nt = ncells + 2 * ng;
    double *k1[ORC_NCONS], *c1[ORC_NCONS], *p1[ORC_NPRIM];
    for (int k = 0; k < ORC_NCONS; ++k) {
        k1[k] = (double *)malloc(sizeof(double) * nt);
        c1[k] = (double *)malloc(sizeof(double) * nt);
    }
    for (int k = 0; k < ORC_NPRIM; ++k) p1[k] = (double *)malloc(sizeof(double) * nt);
    /* stage 1 */
    rhs_1d(ncells, ng, dx, limiter, solver, gamma, (const double *const *)prim, k1);
    for (int k = 0; k < ORC_NCONS; ++k) {
        for (int e = 0; e < nt; ++e) c1[k][e] = cons[k][e] + dt * k1[k][e];
        outflow_1d(c1[k], ncells, ng);
    }
    memcpy(c1[ORC_BX], cons[ORC_BX], sizeof(double) * nt);
    orc_cons_to_prim(nt, (const double *const *)c1, gamma, atmo_rho, 1e-10, p1, NULL);
    for (int k = 0; k < ORC_NPRIM; ++k) outflow_1d(p1[k], ncells, ng);
    /* stage 2 */
    rhs_1d(ncells, ng, dx, limiter, solver, gamma, (const double *const *)p1, k1);
    double *bx = (double *)malloc(sizeof(double) * nt);
    memcpy(bx, cons[ORC_BX], sizeof(double) * nt);
    for (int k = 0; k < ORC_NCONS; ++k) {
        for (int e = 0; e < nt; ++e) cons[k][e] = 0.5 * (cons[k][e] + c1[k][e] + dt * k1[k][e]);
        outflow_1d(cons[k], ncells, ng);
    }
    memcpy(cons[ORC_BX], bx, sizeof(double) * nt);
    orc_cons_to_prim(nt, (const double *const *)cons, gamma, atmo_rho, 1e-10, prim, NULL);
    for (int k = 0; k < ORC_NPRIM; ++k) outflow_1d(prim[k], ncells, ng);
    free(bx);
    for (int k = 0; k < ORC_NCONS; ++k) {
        free(k1[k]);
        free(c1[k]);
    }
    for (int k = 0; k < ORC_NPRIM; ++k) free(p1[k]);
}

/* ── batched-tube workload: one 1D tube (driver2d.py:110-156 on ny = 1) ─ */

/* driver.py:77-127 compute_dt with speed_of_light = False; `(cfl*dx) /
 * tensor` is torch's reciprocal(tensor) * (cfl*dx) */
static double tube_dt(int L, int ng, double dx, double cfl, double gamma,
                      const double *const *prim) {
    double mx = 0.0;
    int first = 1, nan_seen = 0;
    for (int i = ng; i < ng + L; ++i) {
        double rho = prim[ORC_RHO][i], eps = prim[ORC_EPS][i];
        double vx = prim[ORC_VX][i], vy = prim[ORC_VY][i], vz = prim[ORC_VZ][i];
        double Bx = prim[ORC_PBX][i], By = prim[ORC_PBY][i], Bz = prim[ORC_PBZ][i];
        double p, cs2;
        eos_press_cs2(eps, rho, gamma, &p, &cs2);
        double v2 = vx * vx + vy * vy + vz * vz;
        double W = 1.0 / sqrt(clamp_lo(1.0 - v2, 1e-10));
        double B2 = Bx * Bx + By * By + Bz * Bz;
        double vdotB = vx * Bx + vy * By + vz * Bz;
        double b2 = (B2 + vdotB * vdotB) / (W * W);
        double h = 1.0 + eps + p / rho;
        double v02 = cs2 + (b2 / (rho * h + b2)) * (1.0 - cs2);
        double vf = sqrt(clamp_hi(clamp_lo(v02, 0.0), 1.0));
        double s = fabs(vx) + vf;
        if (isnan(s)) nan_seen = 1;
        if (first || s > mx) mx = s;
        first = 0;
    }
    if (nan_seen) return NAN;
    mx = clamp_lo(mx, 1e-14);
    return (1.0 / mx) * (cfl * dx);
}

/* driver.py:388-412: the 1D driver's loop around rk2_step; dt from
 * compute_dt (speed_of_light -> max speed 1, i.e. (1/1) (cfl dx)) */
static int driver1d_run(int L, int ng, double dx, double cfl, double tend, int max_steps,
                        int limiter, int solver, double gamma, double atmo_rho, int light,
                        double *const *cons, double *const *prim, double *t_out) {
    double t = 0.0;
    int steps = 0;
    while (t < tend && steps < max_steps) {
        double dt = light ? (1.0 / 1.0) * (cfl * dx)
                          : tube_dt(L, ng, dx, cfl, gamma, (const double *const *)prim);
        if (dt > tend - t) dt = tend - t;
        if (!(dt > 0.0)) break;
        orc_rk2_step_1d(L, ng, dx, dt, limiter, solver, gamma, atmo_rho, cons, prim);
        t += dt;
        steps++;
    }
    if (t_out) *t_out = t;
    return steps;
}

int orc_tube_run(int L, int ng, double dx, double cfl, double tend, int max_steps, int limiter,
                 int solver, double gamma, double atmo_rho, int scheme, double *const *prim,
                 double *t_out) {
    return orc_tube_run_ex(L, ng, dx, cfl, tend, max_steps, limiter, solver, gamma, atmo_rho,
                           scheme, ORC_TUBE_RK_STEP, 0, NULL, prim, t_out);
}

int orc_tube_run_ex(int L, int ng, double dx, double cfl, double tend, int max_steps, int limiter,
                    int solver, double gamma, double atmo_rho, int scheme, int flavor, int resume,
                    double *const *cons, double *const *prim, double *t_out) {
    const int nt = L + 2 * ng, nf = nt + 1;
    if (flavor != ORC_TUBE_RK_STEP) {
        double *C[ORC_NCONS];
        for (int k = 0; k < ORC_NCONS; ++k)
            C[k] = cons ? cons[k] : (double *)malloc(sizeof(double) * nt);
        if (!resume) orc_prim_to_cons(nt, (const double *const *)prim, C);
        int steps = driver1d_run(L, ng, dx, cfl, tend, max_steps, limiter, solver, gamma, atmo_rho,
                                 flavor == ORC_TUBE_DRIVER1D_LIGHT, C, prim, t_out);
        if (!cons)
            for (int k = 0; k < ORC_NCONS; ++k) free(C[k]);
        return steps;
    }
    const double(*tab)[3] = scheme == 3 ? RK3 : RK2;
    const int nst = scheme == 3 ? 3 : 2;
    double *U[ORC_NCONS], *U0[ORC_NCONS], *F[ORC_NCONS], *Uf[ORC_NCONS];
    double *Lp[ORC_NPRIM], *Rp[ORC_NPRIM];
    for (int k = 0; k < ORC_NCONS; ++k) {
        U[k] = (double *)malloc(sizeof(double) * nt);
        U0[k] = (double *)malloc(sizeof(double) * nt);
        F[k] = (double *)malloc(sizeof(double) * nf);
        Uf[k] = (double *)malloc(sizeof(double) * nf);
    }
    for (int k = 0; k < ORC_NPRIM; ++k) {
        Lp[k] = (double *)malloc(sizeof(double) * nf);
        Rp[k] = (double *)malloc(sizeof(double) * nf);
    }
    double *ps = (double *)malloc(sizeof(double) * nf);
    if (resume && cons)
        for (int k = 0; k < ORC_NCONS; ++k) memcpy(U[k], cons[k], sizeof(double) * nt);
    else
        orc_prim_to_cons(nt, (const double *const *)prim, U);
    double t = 0.0;
    int steps = 0;
    while (t < tend - 1e-14 && steps < max_steps) {
        double dt = tube_dt(L, ng, dx, cfl, gamma, (const double *const *)prim);
        if (dt > tend - t) dt = tend - t;
        if (!(dt > 0.0)) break;
        for (int k = 0; k < ORC_NCONS; ++k) memcpy(U0[k], U[k], sizeof(double) * nt);
        for (int st = 0; st < nst; ++st) {
            double a = tab[st][0], b = tab[st][1], c = tab[st][2];
            /* sweep.py:30-119 with Bnf = None: all eight work variables */
            orc_reconstruct_prims((const double *const *)prim, nt, 1, 0, limiter, 1, gamma, Lp, Rp);
            orc_riemann(nf, (const double *const *)Lp, (const double *const *)Rp, 0, solver, gamma,
                        F, Uf, ps, NULL, NULL, NULL);
            for (int e = 0; e < nf; ++e) F[ORC_BX][e] = 0.0;
            double w2 = c * dt;
            for (int k = 0; k < ORC_NCONS; ++k)
                for (int i = 0; i < nt; ++i) {
                    /* rx + ry with ry = -0.0 exactly (identical y faces) */
                    double rhs = -(F[k][i + 1] - F[k][i]) / dx + (-0.0);
                    double v = a * U0[k][i] + b * U[k][i];
                    U[k][i] = v + w2 * rhs;
                }
            for (int k = 0; k < ORC_NCONS; ++k) outflow_1d(U[k], L, ng);
            orc_cons_to_prim(nt, (const double *const *)U, gamma, atmo_rho, 1e-10, prim, NULL);
            for (int k = 0; k < ORC_NPRIM; ++k) outflow_1d(prim[k], L, ng);
        }
        t += dt;
        steps++;
    }
    if (t_out) *t_out = t;
    if (cons)
        for (int k = 0; k < ORC_NCONS; ++k) memcpy(cons[k], U[k], sizeof(double) * nt);
    for (int k = 0; k < ORC_NCONS; ++k) {
        free(U[k]); free(U0[k]); free(F[k]); free(Uf[k]);
    }
    for (int k = 0; k < ORC_NPRIM; ++k) {
        free(Lp[k]); free(Rp[k]);
    }
    free(ps);
    return steps;
}
