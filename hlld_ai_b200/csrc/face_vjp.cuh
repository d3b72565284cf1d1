// Reverse mode (vector-Jacobian products) of one Riemann face in FP64:
// given the adjoint of the face flux, the adjoint of the two face states.
//
// The forward quantities are recomputed here in the order of
// srmhd_phys.cuh (phys_side / srmhd_fluxes / hlle_face / hlld_face) and
// each statement is then reversed.  Decisions (clamps, max/min, region
// masks, the HLLD fallback) are taken from the recomputed values, so they are
// the forward's.  For HLLD the solved p* is an input: its derivative is the
// implicit-function theorem's, dp* = -(d_C r . dC) / (d_p r), with r the
// residual (hlld.py:586-602); reversing it adds -(p*bar / r_p) * d_C r to the
// adjoint of the residual's inputs.
//
// The results equal the dual-number tangents of the same functions
// contracted with the flux adjoint, at a fraction of their cost.
#pragma once

#include "srmhd_phys.cuh"

namespace hlld {
namespace vjp {

// ── one side of compute_srmhd_fluxes (hlld.py:234-332) ───────────────────

struct SideFwd {
    double P[NPRIM];
    double v2, v2s, W, e, press, he, cs2, B2, vdotB, b2, bt, bs[3], h, X, Y, v02;
    // cp_cm
    double u0sq, omv, a, b, c, disc, det, as, c1, c2, cp, cm;
    double d, rhb2, Pb2, W2;
    double u[NCONS], f[NCONS];
};

template <int IDIR>
__device__ __forceinline__ void side_fwd(const double *P, double g, SideFwd &s) {
    for (int k = 0; k < NPRIM; ++k) s.P[k] = P[k];
    const double vx = P[P_VX], vy = P[P_VY], vz = P[P_VZ];
    const double rho = P[P_RHO], eps = P[P_EPS];
    const double v[3] = {vx, vy, vz}, B[3] = {P[P_BX], P[P_BY], P[P_BZ]};
    s.v2 = vx * vx + vy * vy + vz * vz;
    s.v2s = clamp_hi(s.v2, 1.0 - 1e-10);
    s.W = 1.0 / sqrt(1.0 - s.v2s);
    const double W = s.W;
    // (the intermediates of the reverse only: shared reciprocals)
    const double iW = 1.0 / W, irho = 1.0 / rho;
    s.e = tmax(eps, 0.0);
    s.press = 0.0 + (s.e - 0.0) * rho * (g - 1.0);
    s.he = 1.0 + eps + s.press * irho;
    s.cs2 = (g * 0.0 + g * (s.press - 0.0)) * irho / s.he;
    s.B2 = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
    s.vdotB = v[0] * B[0] + v[1] * B[1] + v[2] * B[2];
    s.b2 = s.B2 * (iW * iW) + s.vdotB * s.vdotB;
    s.bt = W * s.vdotB;
    for (int i = 0; i < 3; ++i) s.bs[i] = B[i] * iW + s.vdotB * v[i] * W;
    s.h = 1.0 + eps + s.press * irho;
    s.Y = rho * s.h + s.b2;
    s.X = s.b2 / s.Y;
    s.v02 = s.cs2 + s.X * (1.0 - s.cs2);
    // cp_cm(v02, W, v[IDIR])
    const double vd = v[IDIR];
    s.u0sq = W * W;
    s.omv = 1.0 - s.v02;
    s.a = s.u0sq * s.omv + s.v02 * 1.0;
    s.b = 2.0 * (0.0 * 1.0 * s.v02 - s.u0sq * vd * s.omv);
    s.c = s.u0sq * (vd * vd) * s.omv - s.v02 * (1.0 - 0.0 * 0.0 * 1.0);
    s.disc = s.b * s.b - 4.0 * s.a * s.c;
    s.det = sqrt(clamp_lo(s.disc, 0.0));
    s.as = clamp_lo(s.a, K<double>::tiny);
    const double ias = 1.0 / s.as;
    s.c1 = 0.5 * (s.det - s.b) * ias;
    s.c2 = -0.5 * (s.det + s.b) * ias;
    s.cp = tmax(s.c1, s.c2);
    s.cm = tmin(s.c1, s.c2);
    s.d = rho * W;
    s.rhb2 = rho * s.h + s.b2;
    s.Pb2 = s.press + 0.5 * s.b2;
    s.W2 = W * W;
    const double bdir = s.bs[IDIR];
    s.u[C_D] = s.d;
    s.f[C_D] = s.d * vd;
    s.u[C_TAU] = s.rhb2 * s.W2 + s.Pb2 * -1.0 - s.bt * s.bt - s.d;
    s.f[C_TAU] = (s.rhb2 * s.W2 * vd - s.bt * bdir) - s.d * vd;
    for (int i = 0; i < 3; ++i) {
        const double uDi = W * v[i];
        s.u[C_SX + i] = s.rhb2 * W * uDi - s.bt * s.bs[i];
        s.f[C_SX + i] = s.rhb2 * (W * vd) * uDi + s.Pb2 * (i == IDIR ? 1.0 : 0.0) - bdir * s.bs[i];
    }
    for (int i = 0; i < 3; ++i) {
        s.u[C_BX + i] = B[i];
        s.f[C_BX + i] = vd * B[i] - v[i] * B[IDIR];
    }
}

// adjoints of u, f, cp, cm -> adjoints of the side's nine primitives (added)
template <int IDIR>
__device__ __forceinline__ void side_rev(const SideFwd &s, double g, const double *au,
                                         const double *af, double acp, double acm, double *aP) {
    const double *P = s.P;
    const double rho = P[P_RHO], eps = P[P_EPS];
    const double v[3] = {P[P_VX], P[P_VY], P[P_VZ]}, B[3] = {P[P_BX], P[P_BY], P[P_BZ]};
    const double W = s.W, vd = v[IDIR], bdir = s.bs[IDIR];
    // reciprocals of the shared denominators
    const double ias = 1.0 / s.as, irho = 1.0 / rho, iW = 1.0 / W, iY = 1.0 / s.Y;
    double a_v[3] = {0, 0, 0}, a_B[3] = {0, 0, 0}, a_bs[3] = {0, 0, 0};
    double a_W = 0, a_rho = 0, a_eps = 0, a_vd = 0, a_bdir = 0, a_d = 0, a_rhb2 = 0, a_W2 = 0;
    double a_Pb2 = 0, a_bt = 0, a_press = 0, a_b2 = 0, a_h = 0, a_vdotB = 0, a_B2 = 0;
    // B components
    for (int i = 0; i < 3; ++i) {
        const double l = af[C_BX + i];
        a_vd += l * B[i];
        a_B[i] += l * vd + au[C_BX + i];
        a_v[i] -= l * B[IDIR];
        a_B[IDIR] -= l * v[i];
    }
    // momenta
    for (int i = 0; i < 3; ++i) {
        const double uDi = W * v[i];
        double a_uDi = 0;
        const double lf = af[C_SX + i];
        const double q = W * vd;
        a_rhb2 += lf * q * uDi;
        const double a_q = lf * s.rhb2 * uDi;
        a_uDi += lf * s.rhb2 * q;
        if (i == IDIR) a_Pb2 += lf;
        a_bdir -= lf * s.bs[i];
        a_bs[i] -= lf * bdir;
        a_W += a_q * vd;
        a_vd += a_q * W;
        const double lu = au[C_SX + i];
        a_rhb2 += lu * W * uDi;
        a_W += lu * s.rhb2 * uDi;
        a_uDi += lu * s.rhb2 * W;
        a_bt -= lu * s.bs[i];
        a_bs[i] -= lu * s.bt;
        a_W += a_uDi * v[i];
        a_v[i] += a_uDi * W;
    }
    // energy
    {
        const double l = af[C_TAU];
        a_rhb2 += l * s.W2 * vd;
        a_W2 += l * s.rhb2 * vd;
        a_vd += l * s.rhb2 * s.W2;
        a_bt -= l * bdir;
        a_bdir -= l * s.bt;
        a_d -= l * vd;
        a_vd -= l * s.d;
        const double m = au[C_TAU];
        a_rhb2 += m * s.W2;
        a_W2 += m * s.rhb2;
        a_Pb2 -= m;
        a_bt -= 2.0 * m * s.bt;
        a_d -= m;
    }
    // density
    a_d += af[C_D] * vd + au[C_D];
    a_vd += af[C_D] * s.d;
    a_W += 2.0 * W * a_W2;
    a_bs[IDIR] += a_bdir;
    a_press += a_Pb2;
    a_b2 += 0.5 * a_Pb2;
    a_rho += a_rhb2 * s.h;
    a_h += a_rhb2 * rho;
    a_b2 += a_rhb2;
    a_rho += a_d * W;
    a_W += a_d * rho;
    // cp_cm
    {
        double a_c1 = 0, a_c2 = 0;
        if (s.c1 < s.c2) a_c2 += acp; else a_c1 += acp;
        if (s.c2 < s.c1) a_c2 += acm; else a_c1 += acm;
        double a_det = 0, a_b = 0, a_as = 0, a_a = 0, a_c = 0, a_u0sq = 0, a_omv = 0, a_v02 = 0;
        a_det += a_c1 * 0.5 * ias;
        a_b -= a_c1 * 0.5 * ias;
        a_as -= a_c1 * s.c1 * ias;
        a_det -= a_c2 * 0.5 * ias;
        a_b -= a_c2 * 0.5 * ias;
        a_as -= a_c2 * s.c2 * ias;
        if (!(s.a < K<double>::tiny)) a_a += a_as;
        const double a_dc = s.det > 0.0 ? a_det * 0.5 / s.det : 0.0;
        const double a_disc = s.disc < 0.0 ? 0.0 : a_dc;
        a_b += 2.0 * s.b * a_disc;
        a_a -= 4.0 * s.c * a_disc;
        a_c -= 4.0 * s.a * a_disc;
        a_u0sq += a_c * (vd * vd) * s.omv;
        a_vd += a_c * s.u0sq * 2.0 * vd * s.omv;
        a_omv += a_c * s.u0sq * (vd * vd);
        a_v02 -= a_c;
        a_u0sq -= a_b * 2.0 * vd * s.omv;
        a_vd -= a_b * 2.0 * s.u0sq * s.omv;
        a_omv -= a_b * 2.0 * s.u0sq * vd;
        a_u0sq += a_a * s.omv;
        a_omv += a_a * s.u0sq;
        a_v02 += a_a;
        a_v02 -= a_omv;
        a_W += 2.0 * W * a_u0sq;
        // v02 = cs2 + X (1 - cs2), X = b2 / Y, Y = rho h + b2
        double a_cs2 = a_v02 * (1.0 - s.X);
        const double a_X = a_v02 * (1.0 - s.cs2);
        a_b2 += a_X * iY;
        const double a_Y = -a_X * s.X * iY;
        a_rho += a_Y * s.h;
        a_h += a_Y * rho;
        a_b2 += a_Y;
        // cs2 = g press / (rho he), he = 1 + eps + press / rho
        a_press += a_cs2 * g * irho / s.he;
        a_rho -= a_cs2 * s.cs2 * irho;
        const double a_he = -a_cs2 * s.cs2 / s.he;
        a_eps += a_he;
        a_press += a_he * irho;
        a_rho -= a_he * s.press * irho * irho;
    }
    // h = 1 + eps + press / rho
    a_eps += a_h;
    a_press += a_h * irho;
    a_rho -= a_h * s.press * irho * irho;
    // bs, bt, b2
    for (int i = 0; i < 3; ++i) {
        a_B[i] += a_bs[i] * iW;
        a_W += -a_bs[i] * B[i] * iW * iW + a_bs[i] * s.vdotB * v[i];
        a_vdotB += a_bs[i] * v[i] * W;
        a_v[i] += a_bs[i] * s.vdotB * W;
    }
    a_W += a_bt * s.vdotB;
    a_vdotB += a_bt * W;
    a_B2 += a_b2 * iW * iW;
    a_W -= a_b2 * 2.0 * s.B2 * iW * iW * iW;
    a_vdotB += 2.0 * a_b2 * s.vdotB;
    for (int i = 0; i < 3; ++i) {
        a_B[i] += 2.0 * a_B2 * B[i] + a_vdotB * v[i];
        a_v[i] += a_vdotB * B[i];
    }
    // press = e rho (g - 1), e = max(eps, 0)
    if (!(eps < 0.0)) a_eps += a_press * rho * (g - 1.0);
    a_rho += a_press * s.e * (g - 1.0);
    // W = (1 - v2s)^(-1/2), v2s = min(v2, 1 - 1e-10)
    const double a_v2 = s.v2 > 1.0 - 1e-10 ? 0.0 : a_W * 0.5 * W * W * W;
    a_v[IDIR] += a_vd;
    for (int i = 0; i < 3; ++i) a_v[i] += 2.0 * a_v2 * v[i];
    aP[P_RHO] += a_rho;
    aP[P_VX] += a_v[0];
    aP[P_VY] += a_v[1];
    aP[P_VZ] += a_v[2];
    aP[P_EPS] += a_eps;
    aP[P_BX] += a_B[0];
    aP[P_BY] += a_B[1];
    aP[P_BZ] += a_B[2];
}

// a side chosen at compile time (left = true)
template <bool LEFT>
struct SideTag {
    static constexpr bool value = LEFT;
};

// what the face solvers read of a side after side_fwd: its conserved
// state, flux and characteristic speeds (18 words instead of SideFwd's 60,
// so that the face's reverse does not hold both sides' intermediates)
struct SideOut {
    double u[NCONS], f[NCONS], cp, cm;
};

// taken from the forward solver's own phys_side, so that u, f and the wave
// speeds -- and through them every decision of the face -- are bit-identical
// to the forward step's
template <int IDIR>
__device__ __forceinline__ void side_out(const double *P, double g, SideOut &o) {
    Side<double> s;
    phys_side<IDIR, double>(P, g, s, o.cp, o.cm);
    for (int k = 0; k < NCONS; ++k) {
        o.u[k] = s.u[k];
        o.f[k] = s.f[k];
    }
}

// a copy the optimiser cannot see through, so that a recomputation from it
// is not merged with the earlier evaluation (whose intermediates would then
// stay live in between)
__device__ __forceinline__ double opaque(double x) {
#ifdef __CUDA_ARCH__
    asm volatile("mov.b64 %0, %0;" : "+d"(x));
#endif
    return x;
}

// side_rev with the side's intermediates recomputed from its primitives
template <int IDIR>
__device__ __forceinline__ void side_rev_from(const double *P, double g, const double *au,
                                              const double *af, double acp, double acm,
                                              double *aP) {
    double Pc[NPRIM];
    for (int k = 0; k < NPRIM; ++k) Pc[k] = opaque(P[k]);
    SideFwd s;
    side_fwd<IDIR>(Pc, g, s);
    side_rev<IDIR>(s, g, au, af, acp, acm, aP);
}

// srmhd_fluxes' wave speeds: adjoints of cmax / cmin -> the sides' cp / cm
struct Speeds {
    double cmax, cmin;
    bool small;
};

__device__ __forceinline__ Speeds speeds(const SideOut &L, const SideOut &R) {
    Speeds s;
    s.cmax = clamp_lo(tmax(L.cp, R.cp), 0.0);
    s.cmin = clamp_lo(tmax(-L.cm, -R.cm), 0.0);
    s.small = (s.cmax < 1e-12) && (s.cmin < 1e-12);
    if (s.small) {
        s.cmax = 1.0;
        s.cmin = 1.0;
    }
    return s;
}

__device__ __forceinline__ void speeds_rev(const SideOut &L, const SideOut &R, const Speeds &s,
                                           double acmax, double acmin, double &acpL,
                                           double &acpR, double &acmL, double &acmR) {
    acpL = acpR = acmL = acmR = 0.0;
    if (s.small) return;
    const double mx = tmax(L.cp, R.cp);
    if (!(mx < 0.0)) {
        if (L.cp < R.cp) acpR += acmax; else acpL += acmax;
    }
    const double mn = tmax(-L.cm, -R.cm);
    if (!(mn < 0.0)) {
        if (-L.cm < -R.cm) acmR -= acmin; else acmL -= acmin;
    }
}

// hf (hlld.py:161-164) in reverse: adjoints of fL, fR, uL, uR, cm, cx.
// (S = cx + cm is the same for every component; its reciprocal is one
// common subexpression of the unrolled component loop.)
__device__ __forceinline__ void hf_rev(double fL, double fR, double uL, double uR, double cm,
                                       double cx, double g, double &afL, double &afR,
                                       double &auL, double &auR, double &acm, double &acx) {
    const double iS = 1.0 / (cx + cm);
    const double N = cx * fL + cm * fR - cx * cm * (uR - uL), q = N * iS;
    const double gi = g * iS;
    afL += gi * cx;
    afR += gi * cm;
    auR -= gi * cx * cm;
    auL += gi * cx * cm;
    acx += gi * ((fL - cm * (uR - uL)) - q);
    acm += gi * ((fR - cx * (uR - uL)) - q);
}

// ── HLLE (hlld.py:1005-1044) ──────────────────────────────────────────────

template <int IDIR>
__device__ __forceinline__ void hlle_face_vjp(const double *PL, const double *PR, double gamma,
                                              const double *aF, double *aPL, double *aPR) {
    SideOut L, R;
    side_out<IDIR>(PL, gamma, L);
    side_out<IDIR>(PR, gamma, R);
    const Speeds sp = speeds(L, R);
    const double cm = sp.cmin, cx = sp.cmax;
    double auL[NCONS] = {}, afL[NCONS] = {}, auR[NCONS] = {}, afR[NCONS] = {};
    double acm = 0, acx = 0;
    for (int k = 0; k < NCONS; ++k) {
        const double g = aF[k];
        if (cx <= 0.0) afR[k] += g;
        else if (cm <= 0.0) afL[k] += g;
        else hf_rev(L.f[k], R.f[k], L.u[k], R.u[k], cm, cx, g, afL[k], afR[k], auL[k], auR[k], acm, acx);
    }
    double acpL, acpR, acmL, acmR;
    speeds_rev(L, R, sp, acx, acm, acpL, acpR, acmL, acmR);
    side_rev_from<IDIR>(PL, gamma, auL, afL, acpL, acmL, aPL);
    side_rev_from<IDIR>(PR, gamma, auR, afR, acpR, acmR, aPR);
}

// ── HLLD (hlld.py:366-605, :1202-1543) at a solved p* ─────────────────────

// safe denominator of _sdiv / SharedDen: d itself unless |d| < tiny, where
// it is the constant +-tiny (zero derivative)
__device__ __forceinline__ bool live_den(double d) { return !(fabs(d) < K<double>::tiny); }
__device__ __forceinline__ double safe_den(double d) {
    if (fabs(d) < K<double>::tiny) {
        double s = tsign(d);
        if (s == 0.0) s = 1.0;
        return s * K<double>::tiny;
    }
    return d;
}

// C fields as an array, index names
enum {
    R_SiL, R_SiR, R_S1L, R_S1R, R_S2L, R_S2R, R_BiL, R_BiR, R_B1L, R_B1R, R_B2L, R_B2R,
    R_TL, R_TR, R_DL, R_DR, R_BnL, R_BnR, R_cm, R_cx, NRC
};

// all intermediates of hlld_vars<true> (hlld.py:431-583)
struct VarsFwd {
    double AL, AR, GL, GR, CL, CR, QL, QR, XL, XR, dXL, dXR;
    double nvaL, nvaR, n1L, n1R, n2L, n2R, vaL, vaR, vt1aL, vt1aR, vt2aL, vt2aR;
    double dAL, dAR, sAL, sAR, Bt1aL, Bt1aR, Bt2aL, Bt2aR, vRSL, vRSR, waL, waR, sqL, sqR;
    double dL, dR, sdL, sdR, KaL, KaR, Kt1aL, Kt1aR, Kt2aL, Kt2aR;
    double dll, sdll, nB1, nB2, Bt1c, Bt2c, KaL2, KaR2, KaLBc, KaRBc;
    double DaL, DaR, vBaL, vBaR, TauaL, TauaR, SaL, SaR, St1aL, St1aR, St2aL, St2aR;
};

__device__ __forceinline__ void vars_fwd(const double *c, double SL, double SR, double p,
                                         VarsFwd &v) {
    // The quantities the forward solver itself produces are taken from its
    // own hlld_vars, so that they are bit-identical to the values the forward
    // step saw (its fast forms multiply by a shared reciprocal where this
    // restatement divides, a one-rounding difference that would move the
    // tiny-denominator decisions: KaL == KaR exactly at a degenerate contact
    // in the forward but not here).  The intermediates between them, which
    // only the reverse needs, are recomputed.
    HlldR<double> C;
    C.RSiL = c[R_SiL]; C.RSiR = c[R_SiR]; C.RS1L = c[R_S1L]; C.RS1R = c[R_S1R];
    C.RS2L = c[R_S2L]; C.RS2R = c[R_S2R]; C.RBiL = c[R_BiL]; C.RBiR = c[R_BiR];
    C.RB1L = c[R_B1L]; C.RB1R = c[R_B1R]; C.RB2L = c[R_B2L]; C.RB2R = c[R_B2R];
    C.RTL = c[R_TL]; C.RTR = c[R_TR]; C.RDL = c[R_DL]; C.RDR = c[R_DR];
    C.S_L = SL; C.S_R = SR; C.BnL = c[R_BnL]; C.BnR = c[R_BnR]; C.cm = c[R_cm]; C.cx = c[R_cx];
    HlldV<double> h;
    hlld_vars<true>(C, p, h);
    const double cm = c[R_cm], cx = c[R_cx], ncm = -cm;
    const double BnL = c[R_BnL], BnR = c[R_BnR];
    v.AL = c[R_SiL] - ncm * c[R_TL] + p * (1.0 - cm * cm);
    v.AR = c[R_SiR] - cx * c[R_TR] + p * (1.0 - cx * cx);
    v.GL = c[R_B1L] * c[R_B1L] + c[R_B2L] * c[R_B2L];
    v.GR = c[R_B1R] * c[R_B1R] + c[R_B2R] * c[R_B2R];
    v.CL = c[R_S1L] * c[R_B1L] + c[R_S2L] * c[R_B2L];
    v.CR = c[R_S1R] * c[R_B1R] + c[R_S2R] * c[R_B2R];
    v.QL = -v.AL - v.GL + (BnL * BnL) * (1.0 - cm * cm);
    v.QR = -v.AR - v.GR + (BnR * BnR) * (1.0 - cx * cx);
    v.XL = BnL * (v.AL * ncm * BnL + v.CL) - (v.AL + v.GL) * (ncm * p + c[R_TL]);
    v.XR = BnR * (v.AR * cx * BnR + v.CR) - (v.AR + v.GR) * (cx * p + c[R_TR]);
    v.dXL = safe_den(v.XL);
    v.dXR = safe_den(v.XR);
    v.nvaL = BnL * (v.AL * BnL + ncm * v.CL) - (v.AL + v.GL) * (p + c[R_SiL]);
    v.nvaR = BnR * (v.AR * BnR + cx * v.CR) - (v.AR + v.GR) * (p + c[R_SiR]);
    v.vaL = h.vaL;
    v.vaR = h.vaR;
    v.n1L = v.CL + BnL * (ncm * c[R_SiL] - c[R_TL]);
    v.n1R = v.CR + BnR * (cx * c[R_SiR] - c[R_TR]);
    v.vt1aL = h.vt1aL;
    v.vt1aR = h.vt1aR;
    v.vt2aL = h.vt2aL;
    v.vt2aR = h.vt2aR;
    v.dAL = ncm - v.vaL;
    v.dAR = cx - v.vaR;
    v.sAL = safe_den(v.dAL);
    v.sAR = safe_den(v.dAR);
    v.Bt1aL = h.Bt1aL;
    v.Bt1aR = h.Bt1aR;
    v.Bt2aL = h.Bt2aL;
    v.Bt2aR = h.Bt2aR;
    v.vRSL = v.vaL * c[R_SiL] + v.vt1aL * c[R_S1L] + v.vt2aL * c[R_S2L];
    v.vRSR = v.vaR * c[R_SiR] + v.vt1aR * c[R_S1R] + v.vt2aR * c[R_S2R];
    v.waL = p + (c[R_TL] - v.vRSL) / v.sAL;
    v.waR = p + (c[R_TR] - v.vRSR) / v.sAR;
    v.sqL = h.sqL;
    v.sqR = h.sqR;
    v.dL = ncm * p + c[R_TL] - BnL * SL * v.sqL;
    v.dR = cx * p + c[R_TR] + BnR * SR * v.sqR;
    v.sdL = safe_den(v.dL);
    v.sdR = safe_den(v.dR);
    v.KaL = h.laL;
    v.KaR = h.laR;
    v.Kt1aL = h.Kt1aL;
    v.Kt1aR = h.Kt1aR;
    v.Kt2aL = h.Kt2aL;
    v.Kt2aR = h.Kt2aR;
    v.dll = v.KaR - v.KaL;
    v.sdll = safe_den(v.dll);
    v.nB1 = (v.Bt1aR * (v.KaR - v.vaR) + BnR * v.vt1aR) - (v.Bt1aL * (v.KaL - v.vaL) + BnL * v.vt1aL);
    v.nB2 = (v.Bt2aR * (v.KaR - v.vaR) + BnR * v.vt2aR) - (v.Bt2aL * (v.KaL - v.vaL) + BnL * v.vt2aL);
    v.Bt1c = h.Bt1c;
    v.Bt2c = h.Bt2c;
    v.KaL2 = h.KaL2;
    v.KaR2 = h.KaR2;
    v.KaLBc = h.KaLBc;
    v.KaRBc = h.KaRBc;
    v.DaL = h.DaL;
    v.DaR = h.DaR;
    v.vBaL = v.vaL * BnL + v.vt1aL * v.Bt1aL + v.vt2aL * v.Bt2aL;
    v.vBaR = v.vaR * BnR + v.vt1aR * v.Bt1aR + v.vt2aR * v.Bt2aR;
    v.TauaL = h.TauaL;
    v.TauaR = h.TauaR;
    v.SaL = h.SaL;
    v.SaR = h.SaR;
    v.St1aL = h.St1aL;
    v.St1aR = h.St1aR;
    v.St2aL = h.St2aL;
    v.St2aR = h.St2aR;
}

// adjoints of VarsFwd's outputs (only the fields the assembly and the
// residual read) -> adjoints of c[] and p
struct VarsAdj {
    double vaL, vaR, vt1aL, vt1aR, vt2aL, vt2aR, Bt1aL, Bt1aR, Bt2aL, Bt2aR, sqL, sqR;
    double KaL, KaR, Kt1aL, Kt1aR, Kt2aL, Kt2aR, Bt1c, Bt2c, KaL2, KaR2, KaLBc, KaRBc;
    double DaL, DaR, TauaL, TauaR, SaL, SaR, St1aL, St1aR, St2aL, St2aR;
};

// d(num / den) with den = safe_den(x), given inv = 1 / den: adds to a_num
// and a_x
__device__ __forceinline__ void div_rev(double g, double q, double inv, double x, double &a_num,
                                        double &a_x) {
    const double gi = g * inv;
    a_num += gi;
    if (live_den(x)) a_x -= gi * q;
}

__device__ __forceinline__ void vars_rev(const double *c, double SL, double SR, double p,
                                         const VarsFwd &v, VarsAdj a, double *ac, double &ap) {
    const double cm = c[R_cm], cx = c[R_cx], ncm = -cm;
    const double BnL = c[R_BnL], BnR = c[R_BnR];
    // one reciprocal per safe denominator (each is shared by several quotients)
    const double iXL = 1.0 / v.dXL, iXR = 1.0 / v.dXR, iAL = 1.0 / v.sAL, iAR = 1.0 / v.sAR;
    const double idL = 1.0 / v.sdL, idR = 1.0 / v.sdR, ill = 1.0 / v.sdll;
    // (FULL part, reversed first)
    const double eL = v.TauaL + v.DaL + p, eR = v.TauaR + v.DaR + p;
    double a_eL = 0, a_eR = 0, a_vBaL = 0, a_vBaR = 0;
    // St2a, St1a, Sa
    a_eL += a.St2aL * v.vt2aL; a.vt2aL += a.St2aL * eL; a_vBaL -= a.St2aL * v.Bt2aL; a.Bt2aL -= a.St2aL * v.vBaL;
    a_eR += a.St2aR * v.vt2aR; a.vt2aR += a.St2aR * eR; a_vBaR -= a.St2aR * v.Bt2aR; a.Bt2aR -= a.St2aR * v.vBaR;
    a_eL += a.St1aL * v.vt1aL; a.vt1aL += a.St1aL * eL; a_vBaL -= a.St1aL * v.Bt1aL; a.Bt1aL -= a.St1aL * v.vBaL;
    a_eR += a.St1aR * v.vt1aR; a.vt1aR += a.St1aR * eR; a_vBaR -= a.St1aR * v.Bt1aR; a.Bt1aR -= a.St1aR * v.vBaR;
    a_eL += a.SaL * v.vaL; a.vaL += a.SaL * eL; a_vBaL -= a.SaL * BnL; ac[R_BnL] -= a.SaL * v.vBaL;
    a_eR += a.SaR * v.vaR; a.vaR += a.SaR * eR; a_vBaR -= a.SaR * BnR; ac[R_BnR] -= a.SaR * v.vBaR;
    a.TauaL += a_eL; a.DaL += a_eL; ap += a_eL;
    a.TauaR += a_eR; a.DaR += a_eR; ap += a_eR;
    // Taua = (T + p va - vBa Bn) / sA - Da
    {
        double a_num = 0, a_x = 0;
        const double q = (c[R_TL] + p * v.vaL - v.vBaL * BnL) * iAL;
        div_rev(a.TauaL, q, iAL, v.dAL, a_num, a_x);
        a.DaL -= a.TauaL;
        ac[R_TL] += a_num; ap += a_num * v.vaL; a.vaL += a_num * p; a_vBaL -= a_num * BnL; ac[R_BnL] -= a_num * v.vBaL;
        double a_dAL = a_x;
        const double qr = (c[R_TR] + p * v.vaR - v.vBaR * BnR) * iAR;
        double b_num = 0, b_x = 0;
        div_rev(a.TauaR, qr, iAR, v.dAR, b_num, b_x);
        a.DaR -= a.TauaR;
        ac[R_TR] += b_num; ap += b_num * v.vaR; a.vaR += b_num * p; a_vBaR -= b_num * BnR; ac[R_BnR] -= b_num * v.vBaR;
        double a_dAR = b_x;
        // vBa = va Bn + vt1a Bt1a + vt2a Bt2a
        a.vaL += a_vBaL * BnL; ac[R_BnL] += a_vBaL * v.vaL; a.vt1aL += a_vBaL * v.Bt1aL; a.Bt1aL += a_vBaL * v.vt1aL;
        a.vt2aL += a_vBaL * v.Bt2aL; a.Bt2aL += a_vBaL * v.vt2aL;
        a.vaR += a_vBaR * BnR; ac[R_BnR] += a_vBaR * v.vaR; a.vt1aR += a_vBaR * v.Bt1aR; a.Bt1aR += a_vBaR * v.vt1aR;
        a.vt2aR += a_vBaR * v.Bt2aR; a.Bt2aR += a_vBaR * v.vt2aR;
        // Da = RD / sA
        double c_num = 0;
        div_rev(a.DaL, v.DaL, iAL, v.dAL, c_num, a_dAL);
        ac[R_DL] += c_num;
        double d_num = 0;
        div_rev(a.DaR, v.DaR, iAR, v.dAR, d_num, a_dAR);
        ac[R_DR] += d_num;
        // KaLBc / KaRBc / KaL2 / KaR2
        a.KaL += a.KaLBc * BnR; ac[R_BnR] += a.KaLBc * v.KaL; a.Kt1aL += a.KaLBc * v.Bt1c; a.Bt1c += a.KaLBc * v.Kt1aL;
        a.Kt2aL += a.KaLBc * v.Bt2c; a.Bt2c += a.KaLBc * v.Kt2aL;
        a.KaR += a.KaRBc * BnR; ac[R_BnR] += a.KaRBc * v.KaR; a.Kt1aR += a.KaRBc * v.Bt1c; a.Bt1c += a.KaRBc * v.Kt1aR;
        a.Kt2aR += a.KaRBc * v.Bt2c; a.Bt2c += a.KaRBc * v.Kt2aR;
        a.KaL += 2.0 * a.KaL2 * v.KaL; a.Kt1aL += 2.0 * a.KaL2 * v.Kt1aL; a.Kt2aL += 2.0 * a.KaL2 * v.Kt2aL;
        a.KaR += 2.0 * a.KaR2 * v.KaR; a.Kt1aR += 2.0 * a.KaR2 * v.Kt1aR; a.Kt2aR += 2.0 * a.KaR2 * v.Kt2aR;
        // Bt{1,2}c = nB / sdll, dll = KaR - KaL
        double a_nB1 = 0, a_nB2 = 0, a_dll = 0;
        div_rev(a.Bt1c, v.Bt1c, ill, v.dll, a_nB1, a_dll);
        div_rev(a.Bt2c, v.Bt2c, ill, v.dll, a_nB2, a_dll);
        a.KaR += a_dll;
        a.KaL -= a_dll;
        // nB = (Bt_aR (KaR - vaR) + BnR vt_aR) - (Bt_aL (KaL - vaL) + BnL vt_aL)
        a.Bt1aR += a_nB1 * (v.KaR - v.vaR); a.KaR += a_nB1 * v.Bt1aR; a.vaR -= a_nB1 * v.Bt1aR;
        ac[R_BnR] += a_nB1 * v.vt1aR; a.vt1aR += a_nB1 * BnR;
        a.Bt1aL -= a_nB1 * (v.KaL - v.vaL); a.KaL -= a_nB1 * v.Bt1aL; a.vaL += a_nB1 * v.Bt1aL;
        ac[R_BnL] -= a_nB1 * v.vt1aL; a.vt1aL -= a_nB1 * BnL;
        a.Bt2aR += a_nB2 * (v.KaR - v.vaR); a.KaR += a_nB2 * v.Bt2aR; a.vaR -= a_nB2 * v.Bt2aR;
        ac[R_BnR] += a_nB2 * v.vt2aR; a.vt2aR += a_nB2 * BnR;
        a.Bt2aL -= a_nB2 * (v.KaL - v.vaL); a.KaL -= a_nB2 * v.Bt2aL; a.vaL += a_nB2 * v.Bt2aL;
        ac[R_BnL] -= a_nB2 * v.vt2aL; a.vt2aL -= a_nB2 * BnL;
        // K vectors: (num) / sd
        double a_dL = 0, a_dR = 0, n;
        n = 0; div_rev(a.KaL, v.KaL, idL, v.dL, n, a_dL);
        ac[R_SiL] += n; ap += n; ac[R_BiL] -= n * SL * v.sqL; a.sqL -= n * c[R_BiL] * SL;
        n = 0; div_rev(a.KaR, v.KaR, idR, v.dR, n, a_dR);
        ac[R_SiR] += n; ap += n; ac[R_BiR] += n * SR * v.sqR; a.sqR += n * c[R_BiR] * SR;
        n = 0; div_rev(a.Kt1aL, v.Kt1aL, idL, v.dL, n, a_dL);
        ac[R_S1L] += n; ac[R_B1L] -= n * SL * v.sqL; a.sqL -= n * c[R_B1L] * SL;
        n = 0; div_rev(a.Kt1aR, v.Kt1aR, idR, v.dR, n, a_dR);
        ac[R_S1R] += n; ac[R_B1R] += n * SR * v.sqR; a.sqR += n * c[R_B1R] * SR;
        n = 0; div_rev(a.Kt2aL, v.Kt2aL, idL, v.dL, n, a_dL);
        ac[R_S2L] += n; ac[R_B2L] -= n * SL * v.sqL; a.sqL -= n * c[R_B2L] * SL;
        n = 0; div_rev(a.Kt2aR, v.Kt2aR, idR, v.dR, n, a_dR);
        ac[R_S2R] += n; ac[R_B2R] += n * SR * v.sqR; a.sqR += n * c[R_B2R] * SR;
        // dL = ncm p + TL - BnL SL sqL; dR = cx p + TR + BnR SR sqR
        ac[R_cm] -= a_dL * p; ap += a_dL * ncm; ac[R_TL] += a_dL; ac[R_BnL] -= a_dL * SL * v.sqL; a.sqL -= a_dL * BnL * SL;
        ac[R_cx] += a_dR * p; ap += a_dR * cx; ac[R_TR] += a_dR; ac[R_BnR] += a_dR * SR * v.sqR; a.sqR += a_dR * BnR * SR;
        // sq = sqrt(max(wa, 0))
        const double a_waL = (v.waL > 0.0 && v.sqL > 0.0) ? a.sqL * 0.5 / v.sqL : 0.0;
        const double a_waR = (v.waR > 0.0 && v.sqR > 0.0) ? a.sqR * 0.5 / v.sqR : 0.0;
        // wa = p + (T - vRS) / sA
        ap += a_waL + a_waR;
        double a_vRSL = 0, a_vRSR = 0;
        {
            double nn = 0;
            div_rev(a_waL, (c[R_TL] - v.vRSL) * iAL, iAL, v.dAL, nn, a_dAL);
            ac[R_TL] += nn; a_vRSL -= nn;
            nn = 0;
            div_rev(a_waR, (c[R_TR] - v.vRSR) * iAR, iAR, v.dAR, nn, a_dAR);
            ac[R_TR] += nn; a_vRSR -= nn;
        }
        // vRS = va Si + vt1a S1 + vt2a S2
        a.vaL += a_vRSL * c[R_SiL]; ac[R_SiL] += a_vRSL * v.vaL; a.vt1aL += a_vRSL * c[R_S1L]; ac[R_S1L] += a_vRSL * v.vt1aL;
        a.vt2aL += a_vRSL * c[R_S2L]; ac[R_S2L] += a_vRSL * v.vt2aL;
        a.vaR += a_vRSR * c[R_SiR]; ac[R_SiR] += a_vRSR * v.vaR; a.vt1aR += a_vRSR * c[R_S1R]; ac[R_S1R] += a_vRSR * v.vt1aR;
        a.vt2aR += a_vRSR * c[R_S2R]; ac[R_S2R] += a_vRSR * v.vt2aR;
        // Bt_a = (RB - Bn vt_a) / sA
        {
            double nn = 0;
            div_rev(a.Bt1aL, v.Bt1aL, iAL, v.dAL, nn, a_dAL);
            ac[R_B1L] += nn; ac[R_BnL] -= nn * v.vt1aL; a.vt1aL -= nn * BnL;
            nn = 0; div_rev(a.Bt2aL, v.Bt2aL, iAL, v.dAL, nn, a_dAL);
            ac[R_B2L] += nn; ac[R_BnL] -= nn * v.vt2aL; a.vt2aL -= nn * BnL;
            nn = 0; div_rev(a.Bt1aR, v.Bt1aR, iAR, v.dAR, nn, a_dAR);
            ac[R_B1R] += nn; ac[R_BnR] -= nn * v.vt1aR; a.vt1aR -= nn * BnR;
            nn = 0; div_rev(a.Bt2aR, v.Bt2aR, iAR, v.dAR, nn, a_dAR);
            ac[R_B2R] += nn; ac[R_BnR] -= nn * v.vt2aR; a.vt2aR -= nn * BnR;
        }
        // dA = ncm - va / cx - va
        ac[R_cm] -= a_dAL; a.vaL -= a_dAL;
        ac[R_cx] += a_dAR; a.vaR -= a_dAR;
        // va, vt1a, vt2a = (num) / dX
        double a_XL = 0, a_XR = 0, a_nvaL = 0, a_nvaR = 0, a_QL = 0, a_QR = 0, a_n1L = 0, a_n1R = 0;
        double nn1 = 0;
        div_rev(a.vaL, v.vaL, iXL, v.XL, a_nvaL, a_XL);
        div_rev(a.vaR, v.vaR, iXR, v.XR, a_nvaR, a_XR);
        nn1 = 0; div_rev(a.vt1aL, v.vt1aL, iXL, v.XL, nn1, a_XL);
        a_QL += nn1 * c[R_S1L]; ac[R_S1L] += nn1 * v.QL; ac[R_B1L] += nn1 * v.n1L; a_n1L += nn1 * c[R_B1L];
        nn1 = 0; div_rev(a.vt2aL, v.vt2aL, iXL, v.XL, nn1, a_XL);
        a_QL += nn1 * c[R_S2L]; ac[R_S2L] += nn1 * v.QL; ac[R_B2L] += nn1 * v.n1L; a_n1L += nn1 * c[R_B2L];
        nn1 = 0; div_rev(a.vt1aR, v.vt1aR, iXR, v.XR, nn1, a_XR);
        a_QR += nn1 * c[R_S1R]; ac[R_S1R] += nn1 * v.QR; ac[R_B1R] += nn1 * v.n1R; a_n1R += nn1 * c[R_B1R];
        nn1 = 0; div_rev(a.vt2aR, v.vt2aR, iXR, v.XR, nn1, a_XR);
        a_QR += nn1 * c[R_S2R]; ac[R_S2R] += nn1 * v.QR; ac[R_B2R] += nn1 * v.n1R; a_n1R += nn1 * c[R_B2R];
        // n1 = C + Bn (ncm Si - T) / C + Bn (cx Si - T)
        double a_CL = a_n1L, a_CR = a_n1R;
        ac[R_BnL] += a_n1L * (ncm * c[R_SiL] - c[R_TL]); ac[R_cm] -= a_n1L * BnL * c[R_SiL];
        ac[R_SiL] += a_n1L * BnL * ncm; ac[R_TL] -= a_n1L * BnL;
        ac[R_BnR] += a_n1R * (cx * c[R_SiR] - c[R_TR]); ac[R_cx] += a_n1R * BnR * c[R_SiR];
        ac[R_SiR] += a_n1R * BnR * cx; ac[R_TR] -= a_n1R * BnR;
        // nva = Bn (A Bn + ncm C) - (A + G)(p + Si)
        double a_AL = 0, a_AR = 0, a_GL = 0, a_GR = 0;
        ac[R_BnL] += a_nvaL * (v.AL * BnL + ncm * v.CL) + a_nvaL * BnL * v.AL;
        a_AL += a_nvaL * BnL * BnL - a_nvaL * (p + c[R_SiL]);
        ac[R_cm] -= a_nvaL * BnL * v.CL; a_CL += a_nvaL * BnL * ncm;
        a_GL -= a_nvaL * (p + c[R_SiL]); ap -= a_nvaL * (v.AL + v.GL); ac[R_SiL] -= a_nvaL * (v.AL + v.GL);
        ac[R_BnR] += a_nvaR * (v.AR * BnR + cx * v.CR) + a_nvaR * BnR * v.AR;
        a_AR += a_nvaR * BnR * BnR - a_nvaR * (p + c[R_SiR]);
        ac[R_cx] += a_nvaR * BnR * v.CR; a_CR += a_nvaR * BnR * cx;
        a_GR -= a_nvaR * (p + c[R_SiR]); ap -= a_nvaR * (v.AR + v.GR); ac[R_SiR] -= a_nvaR * (v.AR + v.GR);
        // X = Bn (A ncm Bn + C) - (A + G)(ncm p + T)
        ac[R_BnL] += a_XL * (v.AL * ncm * BnL + v.CL) + a_XL * BnL * v.AL * ncm;
        a_AL += a_XL * BnL * ncm * BnL - a_XL * (ncm * p + c[R_TL]);
        ac[R_cm] -= a_XL * BnL * v.AL * BnL;
        a_CL += a_XL * BnL;
        a_GL -= a_XL * (ncm * p + c[R_TL]);
        ac[R_cm] += a_XL * (v.AL + v.GL) * p;
        ap -= a_XL * (v.AL + v.GL) * ncm;
        ac[R_TL] -= a_XL * (v.AL + v.GL);
        ac[R_BnR] += a_XR * (v.AR * cx * BnR + v.CR) + a_XR * BnR * v.AR * cx;
        a_AR += a_XR * BnR * cx * BnR - a_XR * (cx * p + c[R_TR]);
        ac[R_cx] += a_XR * BnR * v.AR * BnR;
        a_CR += a_XR * BnR;
        a_GR -= a_XR * (cx * p + c[R_TR]);
        ac[R_cx] -= a_XR * (v.AR + v.GR) * p;
        ap -= a_XR * (v.AR + v.GR) * cx;
        ac[R_TR] -= a_XR * (v.AR + v.GR);
        // Q = -A - G + Bn^2 (1 - c^2)
        a_AL -= a_QL; a_GL -= a_QL; ac[R_BnL] += a_QL * 2.0 * BnL * (1.0 - cm * cm); ac[R_cm] -= a_QL * BnL * BnL * 2.0 * cm;
        a_AR -= a_QR; a_GR -= a_QR; ac[R_BnR] += a_QR * 2.0 * BnR * (1.0 - cx * cx); ac[R_cx] -= a_QR * BnR * BnR * 2.0 * cx;
        // C, G
        ac[R_S1L] += a_CL * c[R_B1L]; ac[R_B1L] += a_CL * c[R_S1L]; ac[R_S2L] += a_CL * c[R_B2L]; ac[R_B2L] += a_CL * c[R_S2L];
        ac[R_S1R] += a_CR * c[R_B1R]; ac[R_B1R] += a_CR * c[R_S1R]; ac[R_S2R] += a_CR * c[R_B2R]; ac[R_B2R] += a_CR * c[R_S2R];
        ac[R_B1L] += 2.0 * a_GL * c[R_B1L]; ac[R_B2L] += 2.0 * a_GL * c[R_B2L];
        ac[R_B1R] += 2.0 * a_GR * c[R_B1R]; ac[R_B2R] += 2.0 * a_GR * c[R_B2R];
        // A = Si - ncm T + p (1 - c^2)
        ac[R_SiL] += a_AL; ac[R_cm] += a_AL * c[R_TL]; ac[R_TL] -= a_AL * ncm; ap += a_AL * (1.0 - cm * cm);
        ac[R_cm] -= a_AL * p * 2.0 * cm;
        ac[R_SiR] += a_AR; ac[R_cx] -= a_AR * c[R_TR]; ac[R_TR] -= a_AR * cx; ap += a_AR * (1.0 - cx * cx);
        ac[R_cx] -= a_AR * p * 2.0 * cx;
    }
}

// residual (hlld.py:586-602): r = (laL - laR) + BnL (sdiv(1 - KaR2, denR) + sdiv(1 - KaL2, denL))
__device__ __forceinline__ double residual_val(const double *c, double SL, double SR,
                                               const VarsFwd &v) {
    const double denR = SR * v.sqR - v.KaRBc, denL = SL * v.sqL + v.KaLBc;
    return (v.KaL - v.KaR) + c[R_BnL] * ((1.0 - v.KaR2) / safe_den(denR) + (1.0 - v.KaL2) / safe_den(denL));
}

// adjoint of the residual with seed g -> VarsAdj fields and ac[R_BnL]
__device__ __forceinline__ void residual_rev(const double *c, double SL, double SR,
                                             const VarsFwd &v, double g, VarsAdj &a, double *ac) {
    const double denR = SR * v.sqR - v.KaRBc, denL = SL * v.sqL + v.KaLBc;
    const double sR = safe_den(denR), sL = safe_den(denL);
    const double tR = (1.0 - v.KaR2) / sR, tL = (1.0 - v.KaL2) / sL;
    a.KaL += g;
    a.KaR -= g;
    ac[R_BnL] += g * (tR + tL);
    const double gt = g * c[R_BnL];
    a.KaR2 -= gt / sR;
    a.KaL2 -= gt / sL;
    if (live_den(denR)) {
        const double ad = -gt * tR / sR;
        a.sqR += ad * SR;
        a.KaRBc -= ad;
    }
    if (live_den(denL)) {
        const double ad = -gt * tL / sL;
        a.sqL += ad * SL;
        a.KaLBc += ad;
    }
}

__device__ __forceinline__ void zero(VarsAdj &a) {
    double *p = reinterpret_cast<double *>(&a);
    for (unsigned k = 0; k < sizeof(VarsAdj) / sizeof(double); ++k) p[k] = 0.0;
}

// the HLLD face at a solved p* in reverse; failed: the HLL flux
template <int IDIR>
__device__ __forceinline__ void hlld_face_vjp(const double *PL, const double *PR, double gamma,
                                              double p_star, bool failed, const double *aF,
                                              double *aPL, double *aPR) {
    constexpr int i = IDIR, t1 = (IDIR + 1) % 3, t2 = (IDIR + 2) % 3;
    SideOut L, R;
    side_out<IDIR>(PL, gamma, L);
    side_out<IDIR>(PR, gamma, R);
    const Speeds sp = speeds(L, R);
    const double cm = sp.cmin, cx = sp.cmax;
    double auL[NCONS] = {}, afL[NCONS] = {}, auR[NCONS] = {}, afR[NCONS] = {};
    double acm = 0, acx = 0;
    double fH[NCONS], uH[NCONS];
    for (int k = 0; k < NCONS; ++k) {
        fH[k] = hf(L.f[k], R.f[k], L.u[k], R.u[k], cm, cx);
        uH[k] = hu(L.f[k], R.f[k], L.u[k], R.u[k], cm, cx);
    }
    if (failed) {
        for (int k = 0; k < NCONS; ++k)
            hf_rev(L.f[k], R.f[k], L.u[k], R.u[k], cm, cx, aF[k], afL[k], afR[k], auL[k], auR[k], acm, acx);
    } else {
        // R vectors on the energy form (uTau + uD)
        double c[NRC];
        auto UL = [&](int k) { return k == C_TAU ? L.u[C_TAU] + L.u[C_D] : L.u[k]; };
        auto UR = [&](int k) { return k == C_TAU ? R.u[C_TAU] + R.u[C_D] : R.u[k]; };
        auto FL = [&](int k) { return k == C_TAU ? L.f[C_TAU] + L.f[C_D] : L.f[k]; };
        auto FR = [&](int k) { return k == C_TAU ? R.f[C_TAU] + R.f[C_D] : R.f[k]; };
        const int kL[NRC] = {C_SX + i, -1, C_SX + t1, -1, C_SX + t2, -1, C_BX + i, -1, C_BX + t1, -1,
                             C_BX + t2, -1, C_TAU, -1, C_D, -1, -1, -1, -1, -1};
        const int kR[NRC] = {-1, C_SX + i, -1, C_SX + t1, -1, C_SX + t2, -1, C_BX + i, -1, C_BX + t1,
                             -1, C_BX + t2, -1, C_TAU, -1, C_D, -1, -1, -1, -1};
        for (int r = 0; r < R_BnL; ++r) {
            if (kL[r] >= 0) c[r] = -cm * UL(kL[r]) - FL(kL[r]);
            else c[r] = cx * UR(kR[r]) - FR(kR[r]);
        }
        c[R_BnL] = L.u[C_BX + i];
        c[R_BnR] = R.u[C_BX + i];
        c[R_cm] = cm;
        c[R_cx] = cx;
        const double SL = tsign(L.u[C_BX + i]), SR = tsign(R.u[C_BX + i]);
        const double p = p_star;
        VarsFwd V;
        vars_fwd(c, SL, SR, p, V);
        // star states (hlld.py:1359-1445) and region (:1447-1480)
        const double denf = -SL * V.sqL - V.KaLBc;
        const double sfac = safe_den(denf);
        const double fac = (1.0 - V.KaL2) / sfac;
        const double BnR = c[R_BnR], BnL = c[R_BnL];
        const double vc = V.KaL - BnR * fac;
        const double vt1 = V.Kt1aL - V.Bt1c * fac;
        const double vt2 = V.Kt2aL - V.Bt2c * fac;
        double vcomp[3], Bc[3];
        vcomp[i] = vc; vcomp[t1] = vt1; vcomp[t2] = vt2;
        Bc[i] = BnR; Bc[t1] = V.Bt1c; Bc[t2] = V.Bt2c;
        const double vBc = vc * Bc[i] + vt1 * V.Bt1c + vt2 * V.Bt2c;
        double uaL[NCONS], uaR[NCONS];
        uaL[C_BX + i] = BnL; uaL[C_BX + t1] = V.Bt1aL; uaL[C_BX + t2] = V.Bt2aL;
        uaL[C_D] = V.DaL; uaL[C_TAU] = V.TauaL; uaL[C_SX + i] = V.SaL; uaL[C_SX + t1] = V.St1aL; uaL[C_SX + t2] = V.St2aL;
        uaR[C_BX + i] = BnR; uaR[C_BX + t1] = V.Bt1aR; uaR[C_BX + t2] = V.Bt2aR;
        uaR[C_D] = V.DaR; uaR[C_TAU] = V.TauaR; uaR[C_SX + i] = V.SaR; uaR[C_SX + t1] = V.St1aR; uaR[C_SX + t2] = V.St2aR;
        const double laL = V.KaL, laR = V.KaR, vi = 0.0;
        const bool cL = vi <= -cm, caL = (-cm < vi) && (vi <= laL), ccL = (laL < vi) && (vi < vc);
        const bool ccR = (vc <= vi) && (vi < laR), caR = (laR <= vi) && (vi < cx), cR = vi >= cx;
        int reg = -1;
        if (cL) reg = 0;
        if (caL) reg = 1;
        if (ccL) reg = 2;
        if (ccR) reg = 3;
        if (caR) reg = 4;
        if (cR) reg = 5;
        VarsAdj a;
        zero(a);
        double ac[NRC] = {};
        double ap = 0.0;
        double a_uaL[NCONS] = {}, a_uaR[NCONS] = {};
        double a_vc = 0, a_vt1 = 0, a_vt2 = 0, a_vBc = 0, a_Bt1c = 0, a_Bt2c = 0, a_BnRc = 0;
        if (reg < 0) {
            for (int k = 0; k < NCONS; ++k)
                hf_rev(L.f[k], R.f[k], L.u[k], R.u[k], cm, cx, aF[k], afL[k], afR[k], auL[k], auR[k], acm, acx);
        } else if (reg == 0) {
            for (int k = 0; k < NCONS; ++k) afL[k] += aF[k];
        } else if (reg == 5) {
            for (int k = 0; k < NCONS; ++k) afR[k] += aF[k];
        } else if (reg == 1 || reg == 4) {
            // the side is a template argument, so that every selection below
            // is resolved at compile time (a runtime choice between the two
            // sides' arrays would put them in local memory)
            auto outer_star = [&](auto side) {
                // fa = f + (-cm)(ua - u) on the left, f + cx (ua - u) on the right
                constexpr bool left = decltype(side)::value;
                const SideOut &S = left ? L : R;
                const double sp_ = left ? -cm : cx;
                for (int k = 0; k < NCONS; ++k) {
                    const double g = aF[k];
                    if (left) { afL[k] += g; a_uaL[k] += g * sp_; auL[k] -= g * sp_; acm -= g * (uaL[k] - S.u[k]); }
                    else { afR[k] += g; a_uaR[k] += g * sp_; auR[k] -= g * sp_; acx += g * (uaR[k] - S.u[k]); }
                }
            };
            if (reg == 1) outer_star(SideTag<true>{});
            else outer_star(SideTag<false>{});
        } else {
            auto contact = [&](auto side) {
                // contact regions: f = fa + la (uc - ua)
                constexpr bool left = decltype(side)::value;
                const SideOut &S = left ? L : R;
                const double sp_ = left ? -cm : cx;
                const double la = left ? laL : laR;
                const double va = left ? V.vaL : V.vaR;
                const double *ua = left ? uaL : uaR;
                double *a_ua = left ? a_uaL : a_uaR;
                const double faT = S.f[C_TAU] + sp_ * (ua[C_TAU] - S.u[C_TAU]);
                const double dn = la - vc;
                const double sdn = safe_den(dn);
                const double rD = (la - va) / sdn;
                const double ucD = ua[C_D] * rD;
                const double nT = la * ua[C_TAU] - faT + p * vc - vBc * Bc[i];
                const double ucT = nT / sdn;
                double uc[NCONS];
                for (int k = 0; k < NCONS; ++k) {
                    if (k == C_D) uc[k] = ucD;
                    else if (k == C_TAU) uc[k] = ucT;
                    else if (k >= C_BX) uc[k] = Bc[k - C_BX];
                    else uc[k] = (ucT + p + ucD) * vcomp[k - C_SX] - vBc * Bc[k - C_SX];
                }
                double a_la = 0, a_ucD = 0, a_ucT = 0, a_uc[NCONS] = {}, a_sp = 0;
                double a_vcomp[3] = {0, 0, 0}, a_Bc[3] = {0, 0, 0};
                for (int k = 0; k < NCONS; ++k) {
                    const double g = aF[k];
                    const double fa = S.f[k] + sp_ * (ua[k] - S.u[k]);
                    (void)fa;
                    // f = fa + la (uc - ua), fa = fS + sp (ua - uS)
                    if (left) afL[k] += g; else afR[k] += g;
                    a_sp += g * (ua[k] - S.u[k]);
                    a_ua[k] += g * sp_ - g * la;
                    if (left) auL[k] -= g * sp_; else auR[k] -= g * sp_;
                    a_la += g * (uc[k] - ua[k]);
                    a_uc[k] += g * la;
                }
                // uc components
                for (int k = 0; k < NCONS; ++k) {
                    const double g = a_uc[k];
                    if (k == C_D) a_ucD += g;
                    else if (k == C_TAU) a_ucT += g;
                    else if (k >= C_BX) a_Bc[k - C_BX] += g;
                    else {
                        const int cc = k - C_SX;
                        a_ucT += g * vcomp[cc];
                        ap += g * vcomp[cc];
                        a_ucD += g * vcomp[cc];
                        a_vcomp[cc] += g * (ucT + p + ucD);
                        a_vBc -= g * Bc[cc];
                        a_Bc[cc] -= g * vBc;
                    }
                }
                // ucT = nT / sdn, nT = la uaT - faT + p vc - vBc Bc_i
                double a_nT = 0, a_dn = 0;
                const double isdn = 1.0 / sdn;
                div_rev(a_ucT, ucT, isdn, dn, a_nT, a_dn);
                a_la += a_nT * ua[C_TAU];
                a_ua[C_TAU] += a_nT * la;
                const double a_faT = -a_nT;
                ap += a_nT * vc;
                a_vc += a_nT * p;
                a_vBc -= a_nT * Bc[i];
                a_Bc[i] -= a_nT * vBc;
                // faT = fS_tau + sp (ua_tau - uS_tau)
                if (left) afL[C_TAU] += a_faT; else afR[C_TAU] += a_faT;
                a_sp += a_faT * (ua[C_TAU] - S.u[C_TAU]);
                a_ua[C_TAU] += a_faT * sp_;
                if (left) auL[C_TAU] -= a_faT * sp_; else auR[C_TAU] -= a_faT * sp_;
                // ucD = ua_D rD, rD = (la - va) / sdn
                a_ua[C_D] += a_ucD * rD;
                const double a_rD = a_ucD * ua[C_D];
                double a_nrD = 0;
                div_rev(a_rD, rD, isdn, dn, a_nrD, a_dn);
                a_la += a_nrD;
                if (left) a.vaL -= a_nrD; else a.vaR -= a_nrD;
                // dn = la - vc
                a_la += a_dn;
                a_vc -= a_dn;
                if (left) { a.KaL += a_la; acm -= a_sp; }
                else { a.KaR += a_la; acx += a_sp; }
                a_vc += a_vcomp[i];
                a_vt1 += a_vcomp[t1];
                a_vt2 += a_vcomp[t2];
                a_BnRc += a_Bc[i];
                a_Bt1c += a_Bc[t1];
                a_Bt2c += a_Bc[t2];
            };
            if (reg == 2) contact(SideTag<true>{});
            else contact(SideTag<false>{});
        }
        // ua arrays -> V fields and Bn
        ac[R_BnL] += a_uaL[C_BX + i];
        a.Bt1aL += a_uaL[C_BX + t1]; a.Bt2aL += a_uaL[C_BX + t2];
        a.DaL += a_uaL[C_D]; a.TauaL += a_uaL[C_TAU]; a.SaL += a_uaL[C_SX + i];
        a.St1aL += a_uaL[C_SX + t1]; a.St2aL += a_uaL[C_SX + t2];
        ac[R_BnR] += a_uaR[C_BX + i];
        a.Bt1aR += a_uaR[C_BX + t1]; a.Bt2aR += a_uaR[C_BX + t2];
        a.DaR += a_uaR[C_D]; a.TauaR += a_uaR[C_TAU]; a.SaR += a_uaR[C_SX + i];
        a.St1aR += a_uaR[C_SX + t1]; a.St2aR += a_uaR[C_SX + t2];
        // vBc = vc BnR + vt1 Bt1c + vt2 Bt2c
        a_vc += a_vBc * BnR; a_BnRc += a_vBc * vc; a_vt1 += a_vBc * V.Bt1c; a_Bt1c += a_vBc * vt1;
        a_vt2 += a_vBc * V.Bt2c; a_Bt2c += a_vBc * vt2;
        // vc = KaL - BnR fac; vt = Kt_aL - Bt_c fac
        double a_fac = -a_vc * BnR - a_vt1 * V.Bt1c - a_vt2 * V.Bt2c;
        a.KaL += a_vc; a_BnRc -= a_vc * fac;
        a.Kt1aL += a_vt1; a_Bt1c -= a_vt1 * fac;
        a.Kt2aL += a_vt2; a_Bt2c -= a_vt2 * fac;
        // fac = (1 - KaL2) / sdiv-den(-SL sqL - KaLBc)
        a.KaL2 -= a_fac / sfac;
        if (live_den(denf)) {
            const double ad = -a_fac * fac / sfac;
            a.sqL -= ad * SL;
            a.KaLBc -= ad;
        }
        a.Bt1c += a_Bt1c;
        a.Bt2c += a_Bt2c;
        ac[R_BnR] += a_BnRc;
        // V -> c, p (direct)
        vars_rev(c, SL, SR, p, V, a, ac, ap);
        // p* through the implicit-function theorem: reverse the residual
        // with seed -ap / r_p (r_p by a dual evaluation)
        {
            HlldR<Dual<1>> c1;
            c1.RSiL = c[R_SiL]; c1.RSiR = c[R_SiR]; c1.RS1L = c[R_S1L]; c1.RS1R = c[R_S1R];
            c1.RS2L = c[R_S2L]; c1.RS2R = c[R_S2R]; c1.RBiL = c[R_BiL]; c1.RBiR = c[R_BiR];
            c1.RB1L = c[R_B1L]; c1.RB1R = c[R_B1R]; c1.RB2L = c[R_B2L]; c1.RB2R = c[R_B2R];
            c1.RTL = c[R_TL]; c1.RTR = c[R_TR]; c1.RDL = c[R_DL]; c1.RDR = c[R_DR];
            c1.S_L = SL; c1.S_R = SR; c1.BnL = c[R_BnL]; c1.BnR = c[R_BnR]; c1.cm = cm; c1.cx = cx;
            const double rp = hlld_residual(c1, Dual<1>::var(p, 0)).d[0];
            const double g = -ap / rp;
            VarsAdj b;
            zero(b);
            double bp = 0.0;
            residual_rev(c, SL, SR, V, g, b, ac);
            vars_rev(c, SL, SR, p, V, b, ac, bp);  // bp: d r / d p * g, not used (IFT)
        }
        // c -> u, f, cm, cx
        for (int r = 0; r < R_BnL; ++r) {
            const double g = ac[r];
            if (g == 0.0) continue;
            if (kL[r] >= 0) {
                const int k = kL[r];
                acm -= g * UL(k);
                if (k == C_TAU) { auL[C_TAU] -= g * cm; auL[C_D] -= g * cm; afL[C_TAU] -= g; afL[C_D] -= g; }
                else { auL[k] -= g * cm; afL[k] -= g; }
            } else {
                const int k = kR[r];
                acx += g * UR(k);
                if (k == C_TAU) { auR[C_TAU] += g * cx; auR[C_D] += g * cx; afR[C_TAU] -= g; afR[C_D] -= g; }
                else { auR[k] += g * cx; afR[k] -= g; }
            }
        }
        auL[C_BX + i] += ac[R_BnL];
        auR[C_BX + i] += ac[R_BnR];
        acm += ac[R_cm];
        acx += ac[R_cx];
    }
    double acpL, acpR, acmL, acmR;
    speeds_rev(L, R, sp, acx, acm, acpL, acpR, acmL, acmR);
    side_rev_from<IDIR>(PL, gamma, auL, afL, acpL, acmL, aPL);
    side_rev_from<IDIR>(PR, gamma, auR, afR, acpR, acmR, aPR);
}

}  // namespace vjp
}  // namespace hlld
