// Reverse mode of the Kastaun conserved -> primitive map at a solved root
// (c2p.py:41-310, restated in srmhd_phys.cuh as Kastaun / kastaun_finish /
// cons_to_prim): lambda of the nine primitives -> lambda of the eight
// conserved variables, with the root's dependence by the implicit-function
// theorem on the master function (c2p.py:129-158).
//
// The map factors through five scalars of Kastaun::init, Z = (D, q, |r|^2,
// |B~|^2, B~.r), and the vectors r, B~: the master function and the
// recovered rho, eps depend on (mu, Z) only, the velocity on (mu, |B~|^2,
// B~.r, r, B~).  So one Dual<6> evaluation of the master function in
// (mu, Z) gives d(rho, eps, f)/d(mu, Z); the velocity and Kastaun::init are
// reversed by hand.  Every branch (tau floor, S rescale, the master
// function's clamps, velocity clamp, atmosphere) follows the value's.
#pragma once

#include "srmhd_phys.cuh"  // (includes dual.cuh)

namespace hlld {
namespace vjp {

__device__ __forceinline__ void c2p_vjp(const double *C, double gamma, double atmo_rho,
                                        double mu, const double *lP, double *lC) {
    constexpr double tiny = K<double>::tiny;
    // ── forward: Kastaun::init (c2p.py:48-106) ──
    const double Dv = C[C_D];
    const double tau0 = C[C_TAU];
    const double tau = clamp_lo(tau0, 0.0);
    double S[3] = {C[C_SX], C[C_SY], C[C_SZ]};
    const double B[3] = {C[C_BX], C[C_BY], C[C_BZ]};
    const double S2_0 = S[0] * S[0] + S[1] * S[1] + S[2] * S[2];
    const double Snorm = sqrt(S2_0);
    const double S_max = Dv + tau;
    const bool too_large = Snorm > S_max;
    const double fac = too_large ? 0.9999 * S_max / (Snorm + tiny) : 1.0;
    const double Sp[3] = {S[0] * fac, S[1] * fac, S[2] * fac};
    const double S2 = Sp[0] * Sp[0] + Sp[1] * Sp[1] + Sp[2] * Sp[2];
    const double B2 = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
    const double BdotS = B[0] * Sp[0] + B[1] * Sp[1] + B[2] * Sp[2];
    const double Dt = Dv + tiny;
    const double q = tau / Dt;
    const double r[3] = {Sp[0] / Dt, Sp[1] / Dt, Sp[2] / Dt};
    const double D2t = Dv * Dv + tiny;
    const double rNorm2 = S2 / D2t;
    const double sqrtD = sqrt(Dt);
    const double Bt[3] = {B[0] / sqrtD, B[1] / sqrtD, B[2] / sqrtD};
    const double BtNorm2 = B2 / Dt;
    const double den_Br = Dv * sqrtD + tiny;
    const double B_dot_r = BdotS / den_Br;

    // ── master function and rho, eps in dual arithmetic over (mu, Z) ──
    using D6 = Dual<6>;
    Kastaun<D6> k;
    k.D = D6::var(Dv, 1);
    k.q = D6::var(q, 2);
    k.rNorm2 = D6::var(rNorm2, 3);
    k.BtNorm2 = D6::var(BtNorm2, 4);
    k.B_dot_r = D6::var(B_dot_r, 5);
    k.B2_rPerp2 = k.rNorm2 * k.BtNorm2 - k.B_dot_r * k.B_dot_r;
    k.v02 = k.rNorm2 / (k.rNorm2 + D6(1.0));
    k.gamma = D6(gamma);
    D6 rho6, eps6;
    const D6 f6 = k.master(D6::var(mu, 0), &rho6, &eps6);

    // ── the finish (c2p.py:268-310) and the primitive assembly ──
    const double c = 1.0 / (1.0 + mu * BtNorm2);
    const double mc = mu * c, mB = mu * B_dot_r;
    double w[3], v[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        w[i] = r[i] + mB * Bt[i];
        v[i] = mc * w[i];
    }
    const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double lim = 1.0 - 1e-10;
    const bool vclamp = v2 > lim;
    const double norm = vclamp ? sqrt(clamp_hi(v2, lim) / (v2 + tiny)) : 1.0;
    const double rho = rho6.v, eps = eps6.v;
    const bool atmo = rho < atmo_rho;

    // ── reverse ──
    double l_rho = 0, l_eps = 0, l_ov[3] = {0, 0, 0};
    if (!atmo) {
        // p = max(eps, 0) rho (gamma - 1)
        l_rho = lP[P_RHO] + lP[P_P] * tmax(eps, 0.0) * (gamma - 1.0);
        l_eps = lP[P_EPS] + (eps < 0.0 ? 0.0 : lP[P_P] * rho * (gamma - 1.0));
        l_ov[0] = lP[P_VX];
        l_ov[1] = lP[P_VY];
        l_ov[2] = lP[P_VZ];
    }
    // adjoints of (mu, Z) and of r, B~
    double lz[6];
#pragma unroll
    for (int j = 0; j < 6; ++j) lz[j] = l_rho * rho6.d[j] + l_eps * eps6.d[j];
    double l_r[3] = {0, 0, 0}, l_Bt[3] = {0, 0, 0};
    {
        double l_v[3];
        if (vclamp) {
            // o.v = v norm, norm = sqrt(lim / (v2 + tiny))
            const double s = l_ov[0] * v[0] + l_ov[1] * v[1] + l_ov[2] * v[2];
            const double g = -s * norm / (v2 + tiny);  // d norm / d v_i = -norm v_i / (v2 + tiny)
#pragma unroll
            for (int i = 0; i < 3; ++i) l_v[i] = norm * l_ov[i] + g * v[i];
        } else {
#pragma unroll
            for (int i = 0; i < 3; ++i) l_v[i] = l_ov[i];
        }
        double l_mc = 0, l_mB = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            l_mc += l_v[i] * w[i];
            const double lw = mc * l_v[i];
            l_r[i] += lw;
            l_mB += lw * Bt[i];
            l_Bt[i] += mB * lw;
        }
        // mB = mu B~.r; mc = mu c; c = 1 / (1 + mu |B~|^2)
        lz[0] += l_mB * B_dot_r + l_mc * c;
        lz[5] += l_mB * mu;
        const double l_c = l_mc * mu;
        lz[0] -= l_c * c * c * BtNorm2;
        lz[4] -= l_c * c * c * mu;
    }
    // the root: d mu = -(d_Z f) / (d_mu f)
    {
        const double g = -lz[0] / f6.d[0];
#pragma unroll
        for (int j = 1; j < 6; ++j) lz[j] += g * f6.d[j];
    }
    // Kastaun::init in reverse
    double l_D = lz[1], l_tau = 0.0, l_Sp[3] = {0, 0, 0}, l_B[3] = {0, 0, 0};
    // q = tau / Dt
    l_tau += lz[2] / Dt;
    l_D -= lz[2] * q / Dt;
    // r_i = S'_i / Dt
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        l_Sp[i] += l_r[i] / Dt;
        l_D -= l_r[i] * r[i] / Dt;
    }
    // |r|^2 = S2 / (D^2 + tiny)
    const double l_S2 = lz[3] / D2t;
    l_D -= lz[3] * rNorm2 * 2.0 * Dv / D2t;
    // |B~|^2 = B2 / Dt
    const double l_B2 = lz[4] / Dt;
    l_D -= lz[4] * BtNorm2 / Dt;
    // B~.r = BdotS / (D sqrtD + tiny)
    const double l_BdotS = lz[5] / den_Br;
    const double l_den = -lz[5] * B_dot_r / den_Br;
    l_D += l_den * sqrtD;
    double l_sqrtD = l_den * Dv;
    // B~_i = B_i / sqrtD
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        l_B[i] += l_Bt[i] / sqrtD;
        l_sqrtD -= l_Bt[i] * Bt[i] / sqrtD;
    }
    l_D += l_sqrtD * 0.5 / sqrtD;
    // S2, B2, BdotS
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        l_Sp[i] += 2.0 * Sp[i] * l_S2 + B[i] * l_BdotS;
        l_B[i] += 2.0 * B[i] * l_B2 + Sp[i] * l_BdotS;
    }
    // S' = S fac
    double l_S[3], l_fac = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        l_S[i] = fac * l_Sp[i];
        l_fac += S[i] * l_Sp[i];
    }
    if (too_large) {
        // fac = 0.9999 S_max / (Snorm + tiny), S_max = D + tau
        const double l_Smax = l_fac * 0.9999 / (Snorm + tiny);
        const double l_Snorm = -l_fac * fac / (Snorm + tiny);
        l_D += l_Smax;
        l_tau += l_Smax;
#pragma unroll
        for (int i = 0; i < 3; ++i) l_S[i] += l_Snorm * S[i] / Snorm;
    }
    lC[C_D] = l_D;
    lC[C_SX] = l_S[0];
    lC[C_SY] = l_S[1];
    lC[C_SZ] = l_S[2];
    lC[C_TAU] = tau0 < 0.0 ? 0.0 : l_tau;
    lC[C_BX] = l_B[0] + lP[P_BX];
    lC[C_BY] = l_B[1] + lP[P_BY];
    lC[C_BZ] = l_B[2] + lP[P_BZ];
}

}  // namespace vjp
}  // namespace hlld
