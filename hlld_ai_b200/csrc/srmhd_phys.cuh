// Device-side SRMHD physics for sm_100a: ideal-gas EOS, primitive <->
// conserved maps, physical fluxes and wave speeds, HLLE, HLLD with its
// total-pressure root solve, and Kastaun C2P.
//
// Every function is a per-element restatement of kemi2805/HLLD-AI's
// element-wise PyTorch code (file:line cited at each function).  Operations
// are written in the reference's order so that a translation unit built
// with -fmad=false reproduces the reference arithmetic one rounding per
// operation; built with FMA contraction the same source is the fast form.
//
// The real type of the reconstruction / flux algebra is a template
// parameter (double, or float for the mixed-precision form); the Kastaun
// C2P and the HLLD p* iteration take their own real type.
#pragma once

// HLLD_EXACT_ARITH = 1 keeps every division of the reference (the exact,
// -fmad=false translation unit defines it)
#ifndef HLLD_EXACT_ARITH
#define HLLD_EXACT_ARITH 0
#endif

#include <cstdint>
#include <cuda_runtime.h>
#include <math.h>

// a function kept out of line (the host compile of these headers, used by
// the host-side checks, has no __noinline__)
#ifdef __CUDACC__
#define HLLD_NOINLINE __noinline__
#else
#define HLLD_NOINLINE __attribute__((noinline))
#endif

namespace hlld {

enum { P_RHO = 0, P_VX, P_VY, P_VZ, P_P, P_EPS, P_BX, P_BY, P_BZ, NPRIM };
enum { C_D = 0, C_SX, C_SY, C_SZ, C_TAU, C_BX, C_BY, C_BZ, NCONS };

// C2P status bits (c2p.py:290-294, :360-362)
constexpr uint8_t ST_BRACKET_OK = 1, ST_CONVERGED = 2, ST_V_CLAMPED = 4, ST_ATMO = 8,
                  ST_BISECTED = 16;
// Riemann flags (hlld.py:1487-1513)
constexpr uint8_t RF_WAVE_ORDER_BAD = 1, RF_BN_ZERO = 2, RF_FAILED = 4;

// Per-precision constants.  The FP64 values are the reference's own
// (hlld.py:29, :1080, c2p.py:29, :318-319); FP32 keeps each one representable.
template <typename T> struct K;
template <> struct K<double> {
    static constexpr double tiny = 1e-300;
    static constexpr double c2p_tol = 1e-15;
    static constexpr double pstar_tol = 1.0e-10;
    static constexpr double weno_eps = 1e-40;
    static constexpr double mp_eps = 1e-40;
    static constexpr double safe_df = 1e-30;
    static constexpr int mu_plus_iters = 50;
    static constexpr double warm_step = 1e-7;  // relative offset of a started C2P secant
};
template <> struct K<float> {
    static constexpr float tiny = 1e-30f;
    static constexpr float c2p_tol = 1e-6f;
    static constexpr float pstar_tol = 1e-5f;
    static constexpr float weno_eps = 1e-20f;  // tau5 / eps stays finite for tau5 < 3e18
    static constexpr float mp_eps = 1e-30f;
    static constexpr float safe_df = 1e-30f;
    static constexpr int mu_plus_iters = 24;
    static constexpr float warm_step = 1e-3f;  // well above FP32 round-off of the master function
};

}  // namespace hlld
#include "dual.cuh"
namespace hlld {
// tangent evaluations use the FP64 constants
template <int N> struct K<Dual<N>> : K<double> {};

// ── element-wise helpers with torch's semantics ─────────────────────────

// torch.maximum / torch.minimum: NaN-propagating, ties keep the first operand
template <typename T> __device__ __forceinline__ T tmax(T a, T b) {
    if (isnan(a)) return a;
    if (isnan(b)) return b;
    return (a < b) ? b : a;
}
template <typename T> __device__ __forceinline__ T tmin(T a, T b) {
    if (isnan(a)) return a;
    if (isnan(b)) return b;
    return (b < a) ? b : a;
}
template <typename T> __device__ __forceinline__ T clamp_lo(T x, T lo) { return (x < lo) ? lo : x; }
template <typename T> __device__ __forceinline__ T clamp_hi(T x, T hi) { return (x > hi) ? hi : x; }
// torch.sign: sign(NaN) = 0
template <typename T> __device__ __forceinline__ T tsign(T x) {
    return (x > T(0)) ? T(1) : ((x < T(0)) ? T(-1) : T(0));
}
// hlld.py:45-54 / c2p.py:32-36 _sdiv
template <typename T> __device__ __forceinline__ T sdiv(T num, T den) {
    if (fabs(den) < K<T>::tiny) {
        T s = tsign(den);
        if (s == T(0)) s = T(1);
        return num / (s * K<T>::tiny);
    }
    return num / den;
}

// Reciprocal by Newton's method on f(y) = 1/y - d, whose step
// y <- y + y (1 - d y) squares the relative error: the hardware's
// approximate reciprocal as the seed and HLLD_NR_STEPS steps.  Two steps
// leave at most 1 ulp against the correctly rounded 1.0 / d (measured on
// B200 over 2^20 doubles spread across the domain and its two ends; one step
// leaves thousands of ulp, and a third step made the mixed x sweep 3 %
// slower for nothing).  Used by the mixed form's FP64 p* solve and cell C2P
// (HLLD_NR_RCP), whose tolerances are far above it.
//
// Domain: finite d with 2^-1000 <= |d| < 2^1000.  The seed flushes to zero
// outside it, so d = +-inf gives NaN (1 / d would give 0), |d| >= 2^1022
// gives 0 (1 / d a subnormal) and |d| < 2^-1022 gives inf; a NaN gives NaN
// like the division.  The callers stay inside: SharedDen clamps |d| to at
// least 1e-300 (the reference's _sdiv rule), the p* residual's denominators
// are finite for finite face states, and the Kastaun master function takes
// reciprocals of 1 / W in [1e-5, 1], of 1 + W, of rho (1 + eps) in
// [1e-12, 1e20] and of 1 + mu |B~|^2 >= 1, which leaves the domain only for
// |B~|^2 = B^2 / D above 1e300, not a finite physical state.  (A check of the
// domain at every call made the mixed sweep 13 % slower, so there is none.)
#ifndef HLLD_NR_STEPS
#define HLLD_NR_STEPS 2
#endif
__device__ __forceinline__ double nr_rcp(double d) {
#if defined(__CUDA_ARCH__)
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
#pragma unroll
    for (int k = 0; k < HLLD_NR_STEPS; ++k) y = fma(y, fma(-d, y, 1.0), y);
    return y;
#else
    return 1.0 / d;
#endif
}

// Square root by Newton's method (HLLD_NR_SQRT): the hardware's approximate
// reciprocal square root y ~ 1/sqrt(x) as the seed, two steps of Newton on
// g(y) = 1/y^2 - x, y <- y + (y/2)(1 - x y^2), then s = x y and one Newton
// step on s^2 - x, s <- s + (y/2)(x - s^2).  For the mixed form's FP64 p*
// residual and Kastaun master function, whose tolerances are far above its
// error (checked against CUDA's correctly rounded sqrt on B200).  Domain: 0
// (exactly 0 returned) and finite x with 2^-1000 <= x < 2^1000 (the seed
// flushes outside it); a NaN gives a NaN.
__device__ __forceinline__ double nr_sqrt(double x) {
#if defined(__CUDA_ARCH__)
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double hy0 = 0.5 * y;
    y = fma(hy0, fma(-x * y, y, 1.0), y);
    const double hy1 = 0.5 * y;
    y = fma(hy1, fma(-x * y, y, 1.0), y);
    double sq = x * y;
    sq = fma(0.5 * y, fma(-sq, sq, x), sq);
    return x > 0.0 ? sq : x;
#else
    return sqrt(x);
#endif
}

// sqrt of the mixed form's FP64 p* residual and master function
template <typename T> __device__ __forceinline__ T sqrt_fast(T x) {
#if defined(HLLD_NR_SQRT)
    if constexpr (sizeof(T) == sizeof(double)) return nr_sqrt(x);
#endif
    return sqrt(x);
}

// 1 / x for the Kastaun master function: the Newton reciprocal in the mixed
// form's FP64 cell C2P, a division everywhere else (the FP64 forms keep the
// reference's quotients).
#if defined(HLLD_NR_RCP)
template <typename T> constexpr bool kNewtonRcp = sizeof(T) == sizeof(double);
#else
template <typename T> constexpr bool kNewtonRcp = false;
#endif
template <typename T> __device__ __forceinline__ T rcp_c2p(T x) {
    if constexpr (kNewtonRcp<T>) return nr_rcp(x);
    else return T(1) / x;
}

// Division by a denominator shared by several quotients.  The exact form
// (HLLD_EXACT_ARITH) divides each numerator as the reference does; the fast
// forms multiply by one reciprocal of the same safe denominator (the _sdiv
// tiny-denominator rule is kept), which differs from the quotient by at
// most one rounding.
template <typename T> struct SharedDen {
    T den;  // the safe denominator (exact form) or its reciprocal (fast forms)
    __device__ __forceinline__ explicit SharedDen(T d) {
        if (fabs(d) < K<T>::tiny) {
            T s = tsign(d);
            if (s == T(0)) s = T(1);
            d = s * K<T>::tiny;
        }
#if HLLD_EXACT_ARITH
        den = d;
#elif defined(HLLD_NR_RCP)
        if constexpr (sizeof(T) == sizeof(double)) den = nr_rcp(d);
        else den = T(1) / d;
#else
        den = T(1) / d;
#endif
    }
    __device__ __forceinline__ T operator()(T num) const {
#if HLLD_EXACT_ARITH
        return num / den;
#else
        return num * den;
#endif
    }
};

// ── EOS: hybrid_eos(K=0, gamma, gamma_th=gamma) (eos.py:32-76) ───────────

template <typename T> __device__ __forceinline__ T eos_press(T eps, T rho, T gamma) {
    T e = tmax(eps, T(0));
    return T(0) + (e - T(0)) * rho * (gamma - T(1));
}
template <typename T> __device__ __forceinline__ T eos_eps(T press, T rho, T gamma) {
    return T(0) + (press - T(0)) / (rho * (gamma - T(1)));
}
template <typename T>
__device__ __forceinline__ void eos_press_cs2(T eps, T rho, T gamma, T &p, T &cs2) {
    T press = eos_press(eps, rho, gamma);
    T h = T(1) + eps + press / rho;
    T press_th = press - T(0);
    p = press;
    cs2 = (gamma * T(0) + gamma * press_th) / (rho * h);
}

// ── primitive -> conserved (hlld.py:185-217) ─────────────────────────────
template <typename T> __device__ __forceinline__ void prim_to_cons(const T *P, T *C) {
    T rho = P[P_RHO], vx = P[P_VX], vy = P[P_VY], vz = P[P_VZ];
    T p = P[P_P], eps = P[P_EPS];
    T Bx = P[P_BX], By = P[P_BY], Bz = P[P_BZ];
    T v2 = vx * vx + vy * vy + vz * vz;
    T W = T(1) / sqrt(clamp_lo(T(1) - v2, T(1e-10)));
    T vB = vx * Bx + vy * By + vz * Bz;
    T B2 = Bx * Bx + By * By + Bz * Bz;
    T h = T(1) + eps + p / rho;
    T rHW2 = rho * h * (W * W);
    T D = rho * W;
    C[C_D] = D;
    C[C_SX] = (rHW2 + B2) * vx - vB * Bx;
    C[C_SY] = (rHW2 + B2) * vy - vB * By;
    C[C_SZ] = (rHW2 + B2) * vz - vB * Bz;
    C[C_TAU] = rHW2 - p - D + T(0.5) * (B2 + B2 * v2 - vB * vB);
    C[C_BX] = Bx;
    C[C_BY] = By;
    C[C_BZ] = Bz;
}

// ── Kastaun C2P (c2p.py:41-363) ──────────────────────────────────────────

template <typename T> struct Kastaun {
    T D, q, r[3], rNorm2, Bt[3], BtNorm2, B_dot_r, B2_rPerp2, v02, gamma;

    // c2p.py:48-106
    __device__ __forceinline__ void init(const T *C, T g) {
        T Dv = C[C_D];
        T Sx = C[C_SX], Sy = C[C_SY], Sz = C[C_SZ];
        T tau = C[C_TAU];
        T Bx = C[C_BX], By = C[C_BY], Bz = C[C_BZ];
        tau = clamp_lo(tau, T(0));
        T S2 = Sx * Sx + Sy * Sy + Sz * Sz;
        T Snorm = sqrt(S2);
        T S_max = Dv + tau;
        bool too_large = Snorm > S_max;
        T fac = too_large ? T(0.9999) * S_max / (Snorm + K<T>::tiny) : T(1);
        Sx = Sx * fac;
        Sy = Sy * fac;
        Sz = Sz * fac;
        S2 = Sx * Sx + Sy * Sy + Sz * Sz;
        T B2 = Bx * Bx + By * By + Bz * Bz;
        T BdotS = Bx * Sx + By * Sy + Bz * Sz;
        D = Dv;
        q = tau / (Dv + K<T>::tiny);
        r[0] = Sx / (Dv + K<T>::tiny);
        r[1] = Sy / (Dv + K<T>::tiny);
        r[2] = Sz / (Dv + K<T>::tiny);
        rNorm2 = S2 / (Dv * Dv + K<T>::tiny);
        T sqrtD = sqrt(Dv + K<T>::tiny);
        Bt[0] = Bx / sqrtD;
        Bt[1] = By / sqrtD;
        Bt[2] = Bz / sqrtD;
        BtNorm2 = B2 / (Dv + K<T>::tiny);
        B_dot_r = BdotS / (Dv * sqrtD + K<T>::tiny);
        B2_rPerp2 = rNorm2 * BtNorm2 - B_dot_r * B_dot_r;
        v02 = rNorm2 / (rNorm2 + T(1));
        gamma = g;
    }
    // c2p.py:110-127
    __device__ __forceinline__ T chi(T mu) const { return rcp_c2p(T(1) + mu * BtNorm2); }
    __device__ __forceinline__ T rbar2(T mu) const {
        T c = chi(mu);
        return rNorm2 * (c * c) + mu * c * (T(1) + c) * (B_dot_r * B_dot_r);
    }
    __device__ __forceinline__ T qbar(T mu) const {
        T c = chi(mu);
        T mc = mu * c;
        return q - T(0.5) * BtNorm2 - T(0.5) * (mc * mc) * B2_rPerp2;
    }
    __device__ __forceinline__ T fa(T mu) const { return mu * sqrt(T(1) + rbar2(mu)) - T(1); }

    // c2p.py:129-158 (f only, or the full set for _finish)
    __device__ __forceinline__ T master(T mu, T *rho_o = nullptr, T *eps_o = nullptr) const {
        T qb = qbar(mu);
        T rb2 = rbar2(mu);
        T vhat2 = tmin((mu * mu) * rb2, v02);
        const T sW = sqrt_fast(clamp_lo(T(1) - vhat2, T(1e-10)));  // 1 / What
        T What = rcp_c2p(sW);
        T rhohat0 = kNewtonRcp<T> ? D * sW : D / What;
        T rhohat = tmin(tmax(rhohat0, T(1e-12)), T(1e15));
        T epshat0 = What * (qb - mu * rb2) + (kNewtonRcp<T> ? vhat2 * (What * What) * rcp_c2p(T(1) + What)
                                                            : vhat2 * (What * What) / (T(1) + What));
        T epshat = tmin(tmax(epshat0, T(0)), T(1e5));
        T phat = eos_press(epshat, rhohat, gamma);
        T ahat = kNewtonRcp<T> ? phat * rcp_c2p(rhohat * (T(1) + epshat) + K<T>::tiny)
                               : phat / (rhohat * (T(1) + epshat) + K<T>::tiny);
        T h_eff = (T(1) + ahat) * (T(1) + epshat);
        T nu_A = kNewtonRcp<T> ? h_eff * sW : h_eff / What;
        T nu_B = (T(1) + ahat) * (T(1) + qb - mu * rb2);
        T nu = tmax(nu_A, nu_B);
        if (rho_o) *rho_o = rhohat;
        if (eps_o) *eps_o = epshat;
        return mu - sdiv(T(1), nu + mu * rb2);
    }

    // c2p.py:162-184: bisection of f_a on [0, 1] (its bracket width is
    // exactly 2^-k after k halvings, so the batch early stop never fires
    // early).  f_a(mu_lo) is a deterministic function of mu_lo, so the value
    // from the previous iteration is reused instead of re-evaluated.
    __device__ HLLD_NOINLINE T mu_plus_bisect() const {  // (a rare fallback: kept out of the hot code)
        T lo = T(0), hi = T(1) / (T(1) + K<T>::tiny);
        T f_lo = fa(lo);
#pragma unroll 1
        for (int it = 0; it < K<T>::mu_plus_iters; ++it) {
            T mid = T(0.5) * (lo + hi);
            T f_mid = fa(mid);
            bool lft = (f_lo * f_mid) <= T(0);
            if (lft) {
                hi = mid;
            } else {
                lo = mid;
                f_lo = f_mid;
            }
        }
        return hi;
    }

    // The same 50 halvings, evaluating f_a only where its sign is in doubt.
    //
    // f_a(mu) = mu sqrt(1 + rbar2(mu)) - 1 is strictly increasing: with
    // chi = 1/(1 + mu b), rbar2 = c/b + (r^2 - c/b) chi^2 (b = |B~|^2,
    // c = (B~.r)^2), so mu^2 (1 + rbar2) = mu^2 (1 + c/b) + (r^2 - c/b) (mu chi)^2
    // has derivative 2 mu [(1 + c/b) + (r^2 - c/b) chi^3] > 0 whenever the
    // rounding-level violation of r^2 >= c/b is below 1 + c/b (|r|^2 < 1e12
    // here).  Its evaluation is accurate to ~1e-15 absolute near the root
    // (all terms positive, the final x - 1 exact).  So once a root estimate r
    // is confirmed by f_a(r - d) < -8e-15 and f_a(r + d) > 8e-15, every
    // midpoint below r - d evaluates negative and every midpoint above
    // r + d non-negative, and the bisection's decision there is known
    // without evaluating.  With f_a(0) = -1 < 0 the reference's test
    // f_lo * f_mid <= 0 is f_mid >= 0 (|f_a| >= 2^-53 or 0 near the root, so
    // the product cannot underflow); a NaN f_mid freezes hi for good, as
    // in the reference.  Anything outside these conditions runs the plain
    // loop.  The result is the plain loop's bit for bit.
    __device__ __forceinline__ T mu_plus() const {
        if constexpr (sizeof(T) == 4) {
            // FP32 (the mixed form's HLL-state C2P, which only seeds the p*
            // bracket): the root by the same safeguarded Newton, stopped at a
            // relative step of 2e-7 (the 24 FP32 halvings resolve 6e-8),
            // moved just above the root and checked to bound it from above,
            // f_a(mu+) >= 0; the bisection's answer where the check fails.
            if (!(rNorm2 < T(1e12)) || !(BtNorm2 < T(1e30)) || !(fa(T(0)) < T(0)))
                return mu_plus_bisect();
            const T b = BtNorm2, c = B_dot_r * B_dot_r, rN = rNorm2;
            T m0 = T(0), m1 = T(1);
            T mu = T(1) / sqrt(T(1) + rN);
#pragma unroll 1
            for (int it = 0; it < 30; ++it) {
                T ch = T(1) / (T(1) + mu * b);
                T dch = -b * ch * ch;
                T rb = rN * ch * ch + mu * ch * (T(1) + ch) * c;
                T drb = rN * T(2) * ch * dch + c * ((ch + mu * dch) * (T(1) + ch) + mu * ch * dch);
                T g = mu * mu * (T(1) + rb) - T(1);
                T dg = T(2) * mu * (T(1) + rb) + mu * mu * drb;
                if (g < T(0)) m0 = mu;
                else m1 = mu;
                if (g == T(0)) break;
                T nm = mu - g / dg;
                if (!(nm > m0 && nm < m1)) nm = T(0.5) * (m0 + m1);
                T stp = fabs(nm - mu);
                mu = nm;
                if (stp <= T(2e-7) * mu) break;
            }
            const T hi = mu * (T(1) + T(1e-6));
            if (!(hi > T(0)) || !(fa(hi) >= T(0))) return mu_plus_bisect();
            return hi;
        }
        if constexpr (sizeof(T) == 8) {
            if (!(rNorm2 < T(1e12)) || !(BtNorm2 < (T(1) / K<T>::tiny)) || !(fa(T(0)) < T(0)))
                return mu_plus_bisect();
            // root of g(mu) = mu^2 (1 + rbar2(mu)) - 1 by safeguarded Newton
            const T b = BtNorm2, c = B_dot_r * B_dot_r, rN = rNorm2;
            T m0 = T(0), m1 = T(1);
            T mu = T(1) / sqrt(T(1) + rN);
#pragma unroll 1
            for (int it = 0; it < 60; ++it) {
                T ch = T(1) / (T(1) + mu * b);
                T dch = -b * ch * ch;
                T rb = rN * ch * ch + mu * ch * (T(1) + ch) * c;
                T drb = rN * T(2) * ch * dch + c * ((ch + mu * dch) * (T(1) + ch) + mu * ch * dch);
                T g = mu * mu * (T(1) + rb) - T(1);
                T dg = T(2) * mu * (T(1) + rb) + mu * mu * drb;
                if (g < T(0)) m0 = mu;
                else m1 = mu;
                if (g == T(0)) break;
                T nm = mu - g / dg;
                if (!(nm > m0 && nm < m1)) nm = T(0.5) * (m0 + m1);
                T stp = fabs(nm - mu);
                mu = nm;
                if (stp <= T(2e-16) * mu) break;
            }
            const T r = mu;
            T d = T(1e-13) * r;
            bool ok = false;
#pragma unroll 1
            for (int t = 0; t < 4 && !ok; ++t) {
                ok = (fa(r - d) < T(-8e-15)) && (fa(r + d) > T(8e-15));
                if (!ok) d *= T(32);
            }
            if (!ok) return mu_plus_bisect();
            T lo = T(0), hi = T(1) / (T(1) + K<T>::tiny);
#pragma unroll 1
            for (int it = 0; it < K<T>::mu_plus_iters; ++it) {
                T mid = T(0.5) * (lo + hi);
                if (mid < r - d) {
                    lo = mid;
                } else if (mid > r + d) {
                    hi = mid;
                } else {
                    T f_mid = fa(mid);
                    if (isnan(f_mid)) break;
                    if (f_mid >= T(0)) hi = mid;
                    else lo = mid;
                }
            }
            return hi;
        } else {
            return mu_plus_bisect();
        }
    }
};

template <typename T> struct C2POut {
    T rho, v[3], p, eps;
    T mu;  // the root the primitives were recovered from
    uint8_t status;
};

// c2p.py:268-310 _finish
template <typename T>
__device__ __forceinline__ void kastaun_finish(const Kastaun<T> &k, T mu, bool converged,
                                               bool good_bracket, C2POut<T> &o) {
    T rho, eps;
    k.master(mu, &rho, &eps);
    T c = k.chi(mu);
    T mc = mu * c;
    T mB = mu * k.B_dot_r;
    T v[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = mc * (k.r[i] + mB * k.Bt[i]);
    T v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    T lim = T(1) - T(1e-10);
    T v2c = clamp_hi(v2, lim);
    T norm = (v2 > lim) ? sqrt(v2c / (v2 + K<T>::tiny)) : T(1);
#pragma unroll
    for (int i = 0; i < 3; ++i) o.v[i] = v[i] * norm;
    o.mu = mu;
    o.rho = rho;
    o.eps = eps;
    o.p = eos_press(eps, rho, k.gamma);
    uint8_t st = 0;
    if (good_bracket) st |= ST_BRACKET_OK;
    if (converged) st |= ST_CONVERGED;
    if (v2 > lim) st |= ST_V_CLAMPED;
    o.status = st;
}

// c2p.py:188-236 invert, stopping per element
template <typename T>
__device__ __forceinline__ void kastaun_invert(const Kastaun<T> &k, T mu_plus, C2POut<T> &o) {
    const T tol = K<T>::c2p_tol;
    T mu_lo = T(0);
    T mu_hi = mu_plus * (T(1) - T(1e-10));
    T f_lo = k.master(mu_lo);
    T f_hi = k.master(mu_hi);
    bool good_bracket = (f_lo * f_hi) < T(0);
    T x0 = mu_lo, x1 = mu_hi, f0 = f_lo, f1 = f_hi;
#pragma unroll 1
    for (int it = 0; it < 60; ++it) {
        if (fabs(f1) < tol) break;
        T df = f1 - f0;
        bool safe = fabs(df) > T(1e-30);
        T x2s = safe ? x1 - f1 * (x1 - x0) / df : T(0.5) * (x0 + x1);
        bool inb = (x2s - x0) * (x2s - x1) < T(0);
        T x2 = inb ? x2s : T(0.5) * (x0 + x1);
        T f2 = k.master(x2);
        bool lft = (f0 * f2) <= T(0);
        if (!lft) {
            x0 = x1;
            f0 = f1;
        }
        x1 = x2;
        f1 = f2;
    }
    kastaun_finish(k, x1, fabs(f1) < tol, good_bracket, o);
}

// c2p.py:238-266 invert_bisection.  A bracket collapsed onto adjacent
// doubles maps onto itself, so stopping at the first unchanged iteration
// returns the 200-step answer.
template <typename T>
__device__ __forceinline__ void kastaun_bisect(const Kastaun<T> &k, T mu_plus, C2POut<T> &o) {
    const T tol = K<T>::c2p_tol;
    T x0 = T(0);
    T x1 = mu_plus * (T(1) - T(1e-10));
    T f0 = k.master(x0);
    T f1 = k.master(x1);
    bool good_bracket = (f0 * f1) < T(0);
#pragma unroll 1
    for (int it = 0; it < 200; ++it) {
        T xm = T(0.5) * (x0 + x1);
        T fm = k.master(xm);
        bool left = (f0 * fm) <= T(0);
        T nx0 = left ? x0 : xm, nf0 = left ? f0 : fm;
        T nx1 = left ? xm : x1, nf1 = left ? fm : f1;
        bool same = (nx0 == x0) && (nx1 == x1) && (nf0 == f0) && (nf1 == f1);
        x0 = nx0;
        f0 = nf0;
        x1 = nx1;
        f1 = nf1;
        if (same) break;
    }
    bool pick = fabs(f0) < fabs(f1);
    T mu = pick ? x0 : x1;
    T fmu = pick ? f0 : f1;
    kastaun_finish(k, mu, fabs(fmu) < tol, good_bracket, o);
}

// c2p.py:313-363 conservative_to_primitive for one element; P gets the nine
// primitives (B copied from C).
// Warm start (used by the mixed-precision form only): a secant on the
// master function from an estimate mu0 of the root -- the same cell's root
// at the previous RK stage, the root 1 / (h W) of its primitives at the
// start of the step, or for the HLL state of a face the mean of its two
// sides' roots.  It returns
// false -- and the caller runs the full bracketed solve -- unless it reaches
// |f| < tol within eight steps at a positive root.  The master function has
// a single root in the physical interval (0, mu+], and a start next to it
// converges to it.
template <typename T>
__device__ __forceinline__ bool kastaun_warm(const Kastaun<T> &k, T mu0, C2POut<T> &o) {
    const T tol = K<T>::c2p_tol;
    if (!(mu0 > T(0)) || !(mu0 < (T(1) / K<T>::tiny))) return false;
    T x0 = mu0 * (T(1) - K<T>::warm_step), x1 = mu0;
    T f0 = k.master(x0), f1 = k.master(x1);
#pragma unroll 1
    for (int it = 0; it < 8; ++it) {
        if (fabs(f1) < tol) {
            if (!(x1 > T(0))) return false;
            kastaun_finish(k, x1, true, true, o);
            return true;
        }
        const T df = f1 - f0;
        if (!(fabs(df) > K<T>::tiny)) return false;
        const T x2 = x1 - f1 * (x1 - x0) / df;
        if (!(x2 > T(0)) || !(x2 < (T(1) / K<T>::tiny))) return false;
        x0 = x1;
        f0 = f1;
        x1 = x2;
        f1 = k.master(x1);
    }
    return false;
}

template <typename T>
__device__ __forceinline__ uint8_t cons_to_prim(const T *C, T gamma, T atmo_rho, T atmo_eps,
                                                T *P, T *mu_out = nullptr, T mu_warm = T(0)) {
    Kastaun<T> k;
    k.init(C, gamma);
    C2POut<T> o;
    uint8_t extra = 0;
    if (!(mu_warm > T(0)) || !kastaun_warm(k, mu_warm, o)) {
        T mp = k.mu_plus();
        kastaun_invert(k, mp, o);
        if (!(o.status & ST_CONVERGED) && (o.status & ST_BRACKET_OK)) {
            kastaun_bisect(k, mp, o);
            o.status |= ST_BRACKET_OK;
            extra = ST_BISECTED;
        }
    }
    if (mu_out) *mu_out = o.mu;
    T rho = o.rho, eps = o.eps, vx = o.v[0], vy = o.v[1], vz = o.v[2];
    bool atmo = rho < atmo_rho;
    if (atmo) {
        rho = atmo_rho;
        eps = atmo_eps;
        vx = T(0);
        vy = T(0);
        vz = T(0);
    }
    P[P_RHO] = rho;
    P[P_VX] = vx;
    P[P_VY] = vy;
    P[P_VZ] = vz;
    P[P_P] = eos_press(eps, rho, gamma);
    P[P_EPS] = eps;
    P[P_BX] = C[C_BX];
    P[P_BY] = C[C_BY];
    P[P_BZ] = C[C_BZ];
    return (uint8_t)(o.status | extra | (atmo ? ST_ATMO : 0));
}

// Tangent of cons_to_prim at a solved element (the adjoint's C2P
// Jacobian): mu is the root the value computation found; its derivative
// follows from the implicit-function theorem on the master function,
// d mu = -(d_C f) / (d_mu f), realised as one Newton step from the root in
// dual arithmetic with the value kept at mu.  Branches (S rescale, velocity
// clamp, atmosphere) follow the value's.
template <typename D>
__device__ __forceinline__ void cons_to_prim_tangent(const D *C, double gamma, double atmo_rho,
                                                     double atmo_eps, double mu, D *P) {
    Kastaun<D> k;
    k.init(C, D(gamma));
    double dfdmu;
    {
        double Cr[NCONS];
#pragma unroll
        for (int i = 0; i < NCONS; ++i) Cr[i] = real_of(C[i]);
        Dual<1> C1[NCONS];
#pragma unroll
        for (int i = 0; i < NCONS; ++i) C1[i] = Dual<1>(Cr[i]);
        Kastaun<Dual<1>> k1;
        k1.init(C1, Dual<1>(gamma));
        dfdmu = k1.master(Dual<1>::var(mu, 0)).d[0];
    }
    D f = k.master(D(mu));
    D m = D(mu) - f / D(dfdmu);
    m.v = mu;
    C2POut<D> o;
    kastaun_finish(k, m, true, true, o);
    D rho = o.rho, eps = o.eps, vx = o.v[0], vy = o.v[1], vz = o.v[2];
    if (rho.v < atmo_rho) {
        rho = D(atmo_rho);
        eps = D(atmo_eps);
        vx = D(0.0);
        vy = D(0.0);
        vz = D(0.0);
    }
    P[P_RHO] = rho;
    P[P_VX] = vx;
    P[P_VY] = vy;
    P[P_VZ] = vz;
    P[P_P] = eos_press(eps, rho, D(gamma));
    P[P_EPS] = eps;
    P[P_BX] = C[C_BX];
    P[P_BY] = C[C_BY];
    P[P_BZ] = C[C_BZ];
}

// ── physical fluxes (hlld.py:57-113, :223-334) ───────────────────────────

template <typename T> struct Side {
    T u[NCONS], f[NCONS];
    T mu;  // Kastaun's C2P root of the side's state, 1 / (h W)
};

// hlld.py:100-113 compute_cp_cm (flat space)
template <typename T>
__device__ __forceinline__ void cp_cm(T v02, T u0, T vd, T &cp, T &cm) {
    T u0_sq = u0 * u0;
    T a = u0_sq * (T(1) - v02) + v02 * T(1);
    T b = T(2) * (T(0) * T(1) * v02 - u0_sq * vd * (T(1) - v02));
    T c = u0_sq * (vd * vd) * (T(1) - v02) - v02 * (T(1) - T(0) * T(0) * T(1));
    T det = sqrt(clamp_lo(b * b - T(4) * a * c, T(0)));
    T a_safe = clamp_lo(a, T(K<T>::tiny));
    T c1 = T(0.5) * (det - b) / a_safe;
    T c2 = T(-0.5) * (det + b) / a_safe;
    cp = tmax(c1, c2);
    cm = tmin(c1, c2);
}

// hlld.py:57-62
template <typename T> __device__ __forceinline__ T lorentz_W(const T *P) {
    T v2 = P[P_VX] * P[P_VX] + P[P_VY] * P[P_VY] + P[P_VZ] * P[P_VZ];
    T v2s = clamp_hi(v2, T(1) - T(1e-10));
    return T(1) / sqrt(T(1) - v2s);
}
// hlld.py:84-90
template <typename T> __device__ __forceinline__ T comp_b2(const T *P, T W) {
    T B2 = P[P_BX] * P[P_BX] + P[P_BY] * P[P_BY] + P[P_BZ] * P[P_BZ];
    T vdotB = P[P_VX] * P[P_BX] + P[P_VY] * P[P_BY] + P[P_VZ] * P[P_BZ];
    return B2 / (W * W) + vdotB * vdotB;
}

// one side of compute_srmhd_fluxes (hlld.py:234-332)
template <int IDIR, typename T>
__device__ __forceinline__ void phys_side(const T *P, T gamma, Side<T> &s, T &cp, T &cm) {
    T W = lorentz_W(P);
    T p, cs2;
    eos_press_cs2(P[P_EPS], P[P_RHO], gamma, p, cs2);
    T b2 = comp_b2(P, W);
    T v[3] = {P[P_VX], P[P_VY], P[P_VZ]};
    T B[3] = {P[P_BX], P[P_BY], P[P_BZ]};
    T vdotB = v[0] * B[0] + v[1] * B[1] + v[2] * B[2];
    T bt = W * vdotB;
    T bs[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) bs[i] = B[i] / W + vdotB * v[i] * W;
    T rho = P[P_RHO], eps = P[P_EPS];
    T h = T(1) + eps + p / rho;
    s.mu = T(1) / (h * W);
    T v02 = cs2 + (b2 / (rho * h + b2)) * (T(1) - cs2);
    cp_cm(v02, W, v[IDIR], cp, cm);
    T d = rho * W;
    T rhb2 = rho * h + b2;
    T Pb2 = p + T(0.5) * b2;
    T vd = v[IDIR];
    T bdir = bs[IDIR];
    s.u[C_D] = d;
    s.f[C_D] = d * vd;
    T Tt = rhb2 * (W * W) + Pb2 * T(-1) - bt * bt;
    s.u[C_TAU] = Tt - d;
    s.f[C_TAU] = (rhb2 * (W * W) * vd - bt * bdir) - d * vd;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        T delta = (i == IDIR) ? T(1) : T(0);
        T uDi = W * v[i];
        s.u[C_SX + i] = rhb2 * W * uDi - bt * bs[i];
        s.f[C_SX + i] = rhb2 * (W * vd) * uDi + Pb2 * delta - bdir * bs[i];
    }
    T Bdir = B[IDIR];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        s.u[C_BX + i] = B[i];
        s.f[C_BX + i] = vd * B[i] - v[i] * Bdir;
    }
}

template <typename T> struct Phys {
    Side<T> L, R;
    T cmax, cmin;
};

template <int IDIR, typename T>
__device__ __forceinline__ void srmhd_fluxes(const T *PL, const T *PR, T gamma, Phys<T> &ph) {
    T cp_l, cm_l, cp_r, cm_r;
    phys_side<IDIR>(PL, gamma, ph.L, cp_l, cm_l);
    phys_side<IDIR>(PR, gamma, ph.R, cp_r, cm_r);
    T cmax = clamp_lo(tmax(cp_l, cp_r), T(0));
    T cmin = clamp_lo(tmax(-cm_l, -cm_r), T(0));
    bool both_small = (cmax < T(1e-12)) && (cmin < T(1e-12));
    if (both_small) {
        cmax = T(1);
        cmin = T(1);
    }
    ph.cmax = cmax;
    ph.cmin = cmin;
}

// hlld.py:161-168.  In FP32 (the mixed form) the same average is written as
// the left value plus a correction built from the two sides' differences.
// The reference's weighted sum rounds an O(1) flux (the momentum flux
// carries the total pressure) to within a few ulp that depend on the bits
// of cx and cm, so neighbouring faces of a nearly uniform state get fluxes
// that differ by FP32 ulps, and their divergence seeds velocity noise of
// ~1e-8 everywhere the stencil has reached.  The difference form is exact
// when the two sides agree and errs no more than the differences
// themselves, so a state without signal stays without one, as in FP64.
template <typename T> __device__ __forceinline__ T hf(T fL, T fR, T uL, T uR, T cm, T cx) {
    if constexpr (sizeof(T) == sizeof(float))
        return fL + cm * ((fR - fL) - cx * (uR - uL)) / (cx + cm);
    return (cx * fL + cm * fR - cx * cm * (uR - uL)) / (cx + cm);
}
template <typename T> __device__ __forceinline__ T hu(T fL, T fR, T uL, T uR, T cm, T cx) {
    if constexpr (sizeof(T) == sizeof(float))
        return uL + (cx * (uR - uL) - (fR - fL)) / (cx + cm);
    return (cx * uR + cm * uL + fL - fR) / (cx + cm);
}

// Per-face solver output.  F has the eight conserved-variable fluxes; U the
// resolved state (only filled when want_u).
template <typename T> struct FaceOut {
    T F[NCONS];
    T U[NCONS];
    T pstar;
    int32_t err, iters;
    uint8_t flags;
};

// hlld.py:1036-1042
template <typename T>
__device__ __forceinline__ T hlle_p_estimate(const T *PL, const T *PR, T gamma) {
    T pl, pr, c;
    eos_press_cs2(PL[P_EPS], PL[P_RHO], gamma, pl, c);
    eos_press_cs2(PR[P_EPS], PR[P_RHO], gamma, pr, c);
    T wl = lorentz_W(PL), wr = lorentz_W(PR);
    T b2l = comp_b2(PL, wl), b2r = comp_b2(PR, wr);
    return clamp_lo(T(0.5) * (pl + T(0.5) * b2l + pr + T(0.5) * b2r), T(1e-30));
}

// hlld.py:1005-1044 hlle_flux
template <int IDIR, typename T>
__device__ __forceinline__ void hlle_face(const T *PL, const T *PR, T gamma, bool want_u,
                                          bool want_pstar, FaceOut<T> &o) {
    Phys<T> ph;
    srmhd_fluxes<IDIR>(PL, PR, gamma, ph);
    T cm = ph.cmin, cx = ph.cmax;
#pragma unroll
    for (int k = 0; k < NCONS; ++k) {
        T fL = ph.L.f[k], fR = ph.R.f[k], uL = ph.L.u[k], uR = ph.R.u[k];
        T fH = hf(fL, fR, uL, uR, cm, cx);
        o.F[k] = (cx <= T(0)) ? fR : ((cm <= T(0)) ? fL : fH);
        if (want_u) {
            T uH = hu(fL, fR, uL, uR, cm, cx);
            o.U[k] = (cm <= T(0)) ? uL : ((cx <= T(0)) ? uR : uH);
        }
    }
    o.pstar = want_pstar ? hlle_p_estimate(PL, PR, gamma) : T(0);
    o.err = 0;
    o.iters = 0;
    o.flags = 0;
}

// ── HLLC (hlld.py:1549-1765) ──────────────────────────────────────────────

// hllc_flux for one face: contact speed from the HLL state (minus root of the
// magnetised quadratic), star states on both sides, region at xi = 0, and the
// HLL flux where the contact is degenerate / superluminal or a result is not
// finite.  pstar gets the p_hll the reference returns in that slot.
template <int IDIR, typename T>
__device__ __forceinline__ void hllc_face(const T *PL, const T *PR, T gamma, bool want_u,
                                          FaceOut<T> &o) {
    constexpr int t1 = (IDIR + 1) % 3, t2 = (IDIR + 2) % 3;
    constexpr int Sn = C_SX + IDIR, S1 = C_SX + t1, S2 = C_SX + t2;
    constexpr int Bn = C_BX + IDIR, B1 = C_BX + t1, B2 = C_BX + t2;
    Phys<T> ph;
    srmhd_fluxes<IDIR>(PL, PR, gamma, ph);
    const T cmin = ph.cmin, cmax = ph.cmax;
    const T S_L = -cmin, S_R = cmax;
    T fH[NCONS], uH[NCONS];
#pragma unroll
    for (int k = 0; k < NCONS; ++k) {
        fH[k] = hf(ph.L.f[k], ph.R.f[k], ph.L.u[k], ph.R.u[k], cmin, cmax);
        uH[k] = hu(ph.L.f[k], ph.R.f[k], ph.L.u[k], ph.R.u[k], cmin, cmax);
    }
    const T BG = ph.L.u[Bn];
    const bool has_B = fabs(BG) > T(1e-15);
    const T cross = has_B ? uH[B1] * fH[B1] + uH[B2] * fH[B2] : T(0);
    const T bt2 = has_B ? uH[B1] * uH[B1] + uH[B2] * uH[B2] : T(0);
    const T fbt2 = has_B ? fH[B1] * fH[B1] + fH[B2] * fH[B2] : T(0);
    const T E_hll = uH[C_TAU] + uH[C_D];
    const T fE_hll = fH[C_TAU] + fH[C_D];
    const T qa = fE_hll - cross;
    const T qb = -fH[Sn] - E_hll + bt2 + fbt2;
    const T qc = uH[Sn] - cross;
    const T disc = sqrt(clamp_lo(qb * qb - T(4) * qa * qc, T(0)));
    const T vc_quad = sdiv(T(-0.5) * (qb + disc), qa);
    const T vc_lin = sdiv(-qc, qb);
    const T vc = fabs(qa) < T(1e-15) ? (fabs(qb) < T(1e-15) ? T(0) : vc_lin) : vc_quad;
    const T vt1 = has_B ? sdiv(uH[B1] * vc - fH[B1], BG) : T(0);
    const T vt2 = has_B ? sdiv(uH[B2] * vc - fH[B2], BG) : T(0);
    const T v2 = vc * vc + vt1 * vt1 + vt2 * vt2;
    const T v2s = clamp_hi(v2, T(1) - T(1e-10));
    const T gs = T(1) / sqrt(T(1) - v2s);
    const T vsBs = has_B ? vc * uH[Bn] + vt1 * uH[B1] + vt2 * uH[B2] : T(0);
    const T bgs = BG / gs;
    const T p_star = has_B ? fH[Sn] + bgs * bgs - vc * (fH[C_TAU] + fH[C_D] - BG * vsBs)
                           : fH[Sn] - vc * (fH[C_TAU] + fH[C_D]);
    const bool degen = (vc <= S_L) || (vc >= S_R) || (v2 >= T(1));
    // region at xi = 0, in the reference's order of overrides: L, *L, *R, R
    // (-1: none applies, the HLL state stays)
    int reg = -1;
    if (T(0) <= S_L) reg = 0;
    if (S_L < T(0) && T(0) < vc) reg = 1;
    if (vc <= T(0) && T(0) < S_R) reg = 2;
    if (T(0) >= S_R) reg = 3;
    T uc[NCONS];
    if (!degen && (reg == 1 || reg == 2)) {
        const Side<T> &sd = reg == 1 ? ph.L : ph.R;
        const T SK = reg == 1 ? S_L : S_R;
        const T vdK = (reg == 1 ? PL : PR)[P_VX + IDIR];
        const T denom = SK - vc;
        uc[Bn] = BG;
        uc[B1] = uH[B1];
        uc[B2] = uH[B2];
        uc[C_D] = sdiv(sd.u[C_D] * (SK - vdK), denom);
        uc[C_TAU] = sdiv(SK * sd.u[C_TAU] - sd.f[C_TAU] + p_star * vc - vsBs * BG, denom);
        uc[Sn] = (uc[C_TAU] + uc[C_D] + p_star) * vc - vsBs * BG;
        const T gs2 = gs * gs;
        uc[S1] = has_B ? sdiv(-BG * (uH[B1] / gs2 + vsBs * vt1) - sd.f[S1] + SK * sd.u[S1], denom)
                       : sdiv(sd.u[S1] * (SK - vdK), denom);
        uc[S2] = has_B ? sdiv(-BG * (uH[B2] / gs2 + vsBs * vt2) - sd.f[S2] + SK * sd.u[S2], denom)
                       : sdiv(sd.u[S2] * (SK - vdK), denom);
    }
#pragma unroll
    for (int k = 0; k < NCONS; ++k) {
        T f = fH[k], u = uH[k];
        if (!degen && reg >= 0) {
            if (reg == 0) {
                f = ph.L.f[k];
                u = ph.L.u[k];
            } else if (reg == 3) {
                f = ph.R.f[k];
                u = ph.R.u[k];
            } else {
                const Side<T> &sd = reg == 1 ? ph.L : ph.R;
                const T SK = reg == 1 ? S_L : S_R;
                f = sd.f[k] + SK * (uc[k] - sd.u[k]);
                u = uc[k];
            }
        }
        if (!isfinite(real_of(f)) || !isfinite(real_of(u))) {
            f = fH[k];
            u = uH[k];
        }
        o.F[k] = f;
        if (want_u) o.U[k] = u;
    }
    o.pstar = hlle_p_estimate(PL, PR, gamma);
    o.err = 0;
    o.iters = 0;
    o.flags = 0;
}

// ── HLLD (hlld.py:366-605, :669-746, :1202-1543) ─────────────────────────

// HLLDComputation R vectors (hlld.py:401-428), energy form
// words of hlld_face's shared-memory slot (PARK_STRIDE > 0)
constexpr int kParkWords = 5 * NCONS + 2;

template <typename T> struct HlldR {
    T RSiL, RSiR, RS1L, RS1R, RS2L, RS2R;
    T RBiL, RBiR, RB1L, RB1R, RB2L, RB2R;
    T RTL, RTR, RDL, RDR;
    T S_L, S_R, BnL, BnR, cm, cx;
};

template <typename T> struct HlldV {
    T vaL, vaR, vt1aL, vt2aL, vt1aR, vt2aR;
    T Bt1aL, Bt2aL, Bt1aR, Bt2aR;
    T sqL, sqR, DaL, DaR, TauaL, TauaR;
    T SaL, SaR, St1aL, St2aL, St1aR, St2aR;
    T laL, laR, Kt1aL, Kt2aL, Kt1aR, Kt2aR;
    T Bt1c, Bt2c, KaL2, KaR2, KaLBc, KaRBc;
};

// hlld.py:431-583 compute_all_variables.  FULL = false computes only what
// the residual needs.
template <bool FULL, typename T>
__device__ __forceinline__ void hlld_vars(const HlldR<T> &c, T p, HlldV<T> &o) {
    const T cm = c.cm, cx = c.cx, ncm = -c.cm;
    const T RSiL = c.RSiL, RSiR = c.RSiR, RS1L = c.RS1L, RS1R = c.RS1R;
    const T RS2L = c.RS2L, RS2R = c.RS2R;
    const T RB1L = c.RB1L, RB1R = c.RB1R, RB2L = c.RB2L, RB2R = c.RB2R;
    const T RTL = c.RTL, RTR = c.RTR, BnL = c.BnL, BnR = c.BnR;

    T AL = RSiL - ncm * RTL + p * (T(1) - cm * cm);
    T AR = RSiR - cx * RTR + p * (T(1) - cx * cx);
    T GL = RB1L * RB1L + RB2L * RB2L;
    T GR = RB1R * RB1R + RB2R * RB2R;
    T CL = RS1L * RB1L + RS2L * RB2L;
    T CR = RS1R * RB1R + RS2R * RB2R;
    T QL = -AL - GL + (BnL * BnL) * (T(1) - cm * cm);
    T QR = -AR - GR + (BnR * BnR) * (T(1) - cx * cx);
    T XL = BnL * (AL * ncm * BnL + CL) - (AL + GL) * (ncm * p + RTL);
    T XR = BnR * (AR * cx * BnR + CR) - (AR + GR) * (cx * p + RTR);

    const SharedDen<T> dXL(XL), dXR(XR);
    T vaL = dXL(BnL * (AL * BnL + ncm * CL) - (AL + GL) * (p + RSiL));
    T vaR = dXR(BnR * (AR * BnR + cx * CR) - (AR + GR) * (p + RSiR));
    T vt1aL = dXL(QL * RS1L + RB1L * (CL + BnL * (ncm * RSiL - RTL)));
    T vt1aR = dXR(QR * RS1R + RB1R * (CR + BnR * (cx * RSiR - RTR)));
    T vt2aL = dXL(QL * RS2L + RB2L * (CL + BnL * (ncm * RSiL - RTL)));
    T vt2aR = dXR(QR * RS2R + RB2R * (CR + BnR * (cx * RSiR - RTR)));

    const SharedDen<T> dAL(ncm - vaL), dAR(cx - vaR);
    T Bt1aL = dAL(RB1L - BnL * vt1aL);
    T Bt1aR = dAR(RB1R - BnR * vt1aR);
    T Bt2aL = dAL(RB2L - BnL * vt2aL);
    T Bt2aR = dAR(RB2R - BnR * vt2aR);

    T vRS_AL = vaL * RSiL + vt1aL * RS1L + vt2aL * RS2L;
    T vRS_AR = vaR * RSiR + vt1aR * RS1R + vt2aR * RS2R;

    T waL = p + dAL(RTL - vRS_AL);
    T waR = p + dAR(RTR - vRS_AR);

    T sqL = sqrt_fast(clamp_lo(waL, T(0)));
    T sqR = sqrt_fast(clamp_lo(waR, T(0)));

    const T S_L = c.S_L, S_R = c.S_R;
    T dL = ncm * p + RTL - BnL * S_L * sqL;
    T dR = cx * p + RTR + BnR * S_R * sqR;

    const SharedDen<T> ddL(dL), ddR(dR);
    T KaL = ddL(RSiL + p - c.RBiL * S_L * sqL);
    T KaR = ddR(RSiR + p + c.RBiR * S_R * sqR);
    T Kt1aL = ddL(RS1L - RB1L * S_L * sqL);
    T Kt1aR = ddR(RS1R + RB1R * S_R * sqR);
    T Kt2aL = ddL(RS2L - RB2L * S_L * sqL);
    T Kt2aR = ddR(RS2R + RB2R * S_R * sqR);

    T laL = KaL, laR = KaR;
    T denom_ll = laR - laL;
    T Bic = BnR;
    const SharedDen<T> dll(denom_ll);
    T Bt1c = dll((Bt1aR * (laR - vaR) + BnR * vt1aR) - (Bt1aL * (laL - vaL) + BnL * vt1aL));
    T Bt2c = dll((Bt2aR * (laR - vaR) + BnR * vt2aR) - (Bt2aL * (laL - vaL) + BnL * vt2aL));

    o.sqL = sqL;
    o.sqR = sqR;
    o.laL = laL;
    o.laR = laR;
    o.KaL2 = KaL * KaL + Kt1aL * Kt1aL + Kt2aL * Kt2aL;
    o.KaR2 = KaR * KaR + Kt1aR * Kt1aR + Kt2aR * Kt2aR;
    o.KaLBc = KaL * Bic + Kt1aL * Bt1c + Kt2aL * Bt2c;
    o.KaRBc = KaR * Bic + Kt1aR * Bt1c + Kt2aR * Bt2c;
    if (FULL) {
        T DaL = dAL(c.RDL);
        T DaR = dAR(c.RDR);
        T vBaL = vaL * BnL + vt1aL * Bt1aL + vt2aL * Bt2aL;
        T vBaR = vaR * BnR + vt1aR * Bt1aR + vt2aR * Bt2aR;
        T TauaL = dAL(RTL + p * vaL - vBaL * BnL) - DaL;
        T TauaR = dAR(RTR + p * vaR - vBaR * BnR) - DaR;
        o.SaL = (TauaL + DaL + p) * vaL - vBaL * BnL;
        o.SaR = (TauaR + DaR + p) * vaR - vBaR * BnR;
        o.St1aL = (TauaL + DaL + p) * vt1aL - vBaL * Bt1aL;
        o.St1aR = (TauaR + DaR + p) * vt1aR - vBaR * Bt1aR;
        o.St2aL = (TauaL + DaL + p) * vt2aL - vBaL * Bt2aL;
        o.St2aR = (TauaR + DaR + p) * vt2aR - vBaR * Bt2aR;
        o.DaL = DaL;
        o.DaR = DaR;
        o.TauaL = TauaL;
        o.TauaR = TauaR;
        o.vaL = vaL;
        o.vaR = vaR;
        o.vt1aL = vt1aL;
        o.vt2aL = vt2aL;
        o.vt1aR = vt1aR;
        o.vt2aR = vt2aR;
        o.Bt1aL = Bt1aL;
        o.Bt2aL = Bt2aL;
        o.Bt1aR = Bt1aR;
        o.Bt2aR = Bt2aR;
        o.Kt1aL = Kt1aL;
        o.Kt2aL = Kt2aL;
        o.Kt1aR = Kt1aR;
        o.Kt2aR = Kt2aR;
        o.Bt1c = Bt1c;
        o.Bt2c = Bt2c;
    }
}

// hlld.py:586-602 residual
template <typename T> __device__ __forceinline__ T hlld_residual_body(const HlldR<T> &c, T p) {
    HlldV<T> v;
    hlld_vars<false>(c, p, v);
    T denom_R = c.S_R * v.sqR - v.KaRBc;
    T denom_L = c.S_L * v.sqL + v.KaLBc;
    return (v.laL - v.laR) + c.BnL * (sdiv(T(1) - v.KaR2, denom_R) + sdiv(T(1) - v.KaL2, denom_L));
}
// For the real types the residual is kept out of line: the p* solve
// evaluates it at five call sites (bracket, widening, secant), and one
// shared body instead of five inlined copies keeps the persistent tube
// kernel's hot code within the instruction cache (measured on B200: tubes
// +15 %, the 2D step unchanged).  The dual-number uses (one per face, in the
// derivative code) stay inlined.
template <typename T> __device__ HLLD_NOINLINE T hlld_residual_ool(const HlldR<T> &c, T p) {
    return hlld_residual_body(c, p);
}
template <typename T> __device__ __forceinline__ T hlld_residual(const HlldR<T> &c, T p) {
    if constexpr (sizeof(T) <= sizeof(double)) return hlld_residual_ool(c, p);
    else return hlld_residual_body(c, p);
}
// The residual at a p* solve's call sites: inlined for the 2D sweeps
// (INLINE = true; measured on B200: the mixed x sweep 1.084 -> 1.000 ms,
// the FP64 one 2.62 -> 2.39 ms), out of line for the tube kernel, whose
// phases share the instruction cache.  (Inlining only the secant's call,
// with the bracket's and the widening's sharing one out-of-line body, was
// slower in the sweep: 0.976 against 0.902 ms with everything inlined.)
template <bool INLINE, typename T> __device__ __forceinline__ T hlld_residual_at(const HlldR<T> &c, T p) {
    if constexpr (INLINE) return hlld_residual_body(c, p);
    else return hlld_residual(c, p);
}

#define HLLD_R_FIELDS(X)                                                                        \
    X(RSiL) X(RSiR) X(RS1L) X(RS1R) X(RS2L) X(RS2R) X(RBiL) X(RBiR) X(RB1L) X(RB1R) X(RB2L)      \
    X(RB2R) X(RTL) X(RTR) X(RDL) X(RDR) X(S_L) X(S_R) X(BnL) X(BnR) X(cm) X(cx)

// p* as a dual number at a solved face: p*'s derivative from the
// implicit-function theorem on the residual, d p* = -(d_x r) / (d_p r), as
// one Newton step from the root with the value kept at p*.
template <typename TP> __device__ __forceinline__ TP hlld_ift_root(const HlldR<TP> &C, double ps) {
    HlldR<Dual<1>> c1;
#define HLLD_REAL_FIELD(f) c1.f = Dual<1>(real_of(C.f));
    HLLD_R_FIELDS(HLLD_REAL_FIELD)
#undef HLLD_REAL_FIELD
    const double drdp = hlld_residual(c1, Dual<1>::var(ps, 0)).d[0];
    TP r = hlld_residual(C, TP(ps));
    TP out = TP(ps) - r / TP(drdp);
    out.v = ps;
    return out;
}

// hlld.py:1202-1543 hlld_flux for one face.  T is the algebra's real type,
// TC the real type of the HLL-state C2P (legacy bracket) and TP that of the
// p* iteration; the fast and exact forms use double for all three.
// IFT = true is the tangent form (T = TP = Dual): given[0] is the face's
// solved p* and given[1] != 0 its fallback decision, both from the value
// computation; the bracket and the secant are skipped.  SKIP_BN0: no p*
// solve on faces without normal field (see below); with need_pstar false as
// well, not even the HLL-state C2P whose total pressure would only feed the
// p* output there (o.pstar is then 0).  INLINE_RES: the p* residual inlined
// at its call sites (hlld_residual_at).
template <int IDIR, typename T, typename TC = T, typename TP = T, bool IFT = false,
          bool SKIP_BN0 = (sizeof(TC) == sizeof(float)), bool INLINE_RES = false,
          int PARK_STRIDE = 0>
__device__ __forceinline__ void hlld_face(const T *PL, const T *PR, T gamma, bool want_u,
                                          FaceOut<T> &o, const double *given = nullptr,
                                          bool need_pstar = true, T *park = nullptr) {
    constexpr int i = IDIR, t1 = (IDIR + 1) % 3, t2 = (IDIR + 2) % 3;
    Phys<T> ph;
    srmhd_fluxes<IDIR>(PL, PR, gamma, ph);
    T cm = ph.cmin, cx = ph.cmax;
    T fH[NCONS], uH[NCONS];
#pragma unroll
    for (int k = 0; k < NCONS; ++k) {
        fH[k] = hf(ph.L.f[k], ph.R.f[k], ph.L.u[k], ph.R.u[k], cm, cx);
        uH[k] = hu(ph.L.f[k], ph.R.f[k], ph.L.u[k], ph.R.u[k], cm, cx);
    }

    constexpr int Sn = C_SX + i, Bn = C_BX + i;
    if constexpr (!IFT && SKIP_BN0) {
        // a face without normal field whose p* output nobody reads: the
        // HLLE fallback's flux and state, nothing else (hlld.py:1512-1531)
        if (!need_pstar && fabs(ph.L.u[Bn]) < T(1e-14) && fabs(ph.R.u[Bn]) < T(1e-14)) {
#pragma unroll
            for (int k = 0; k < NCONS; ++k) {
                o.F[k] = fH[k];
                if (want_u) o.U[k] = uH[k];
            }
            o.pstar = T(0);
            o.err = -1;
            o.iters = 0;
            o.flags = RF_BN_ZERO | RF_FAILED;
            return;
        }
    }

    // legacy bracket (hlld.py:1253-1263): total pressure of the HLL state
    TP p_hll = TP(0), p_lo = TP(0), p_hi = TP(0);
    if constexpr (!IFT) {
        TC Ch[NCONS], Ph[NPRIM];
#pragma unroll
        for (int k = 0; k < NCONS; ++k) Ch[k] = (TC)uH[k];
        // FP32 (the mixed form): the root search starts from the mean of the
        // two sides' roots, next to the HLL state's own, and takes the
        // bracketed solve only if that start does not converge; the FP64
        // forms solve from the bracket as the reference does
        TC mu_start = TC(0);
        if constexpr (sizeof(TC) == sizeof(float))
            mu_start = TC(0.5) * ((TC)ph.L.mu + (TC)ph.R.mu);
        cons_to_prim<TC>(Ch, (TC)gamma, TC(1e-10), TC(1e-10), Ph, nullptr, mu_start);
        TC pp, cs2;
        eos_press_cs2(Ph[P_EPS], Ph[P_RHO], (TC)gamma, pp, cs2);
        TC w = lorentz_W(Ph);
        TC b2 = comp_b2(Ph, w);
        p_hll = (TP)(pp + TC(0.5) * b2);

        // p0 from the Bn = 0 limit (hlld.py:1265-1287)
        TP a = (TP)fH[C_TAU] + (TP)fH[C_D];
        TP b = -(TP)fH[Sn] - (TP)uH[C_TAU] - (TP)uH[C_D];
        TP cq = (TP)uH[Sn];
        TP disc = b * b - TP(4) * a * cq;
        disc = clamp_lo(disc, TP(0));
        bool abig = fabs(a) > TP(1e-14);
        TP safe_a = abig ? a : TP(1);
        TP safe_b = abig ? b : TP(1);
        TP v_star = abig ? (-b - sqrt(disc)) / (TP(2) * safe_a) : -cq / safe_b;
        v_star = clamp_hi(clamp_lo(v_star, -(TP(1) - TP(1e-10))), TP(1) - TP(1e-10));
        TP p0 = (TP)fH[Sn] - ((TP)fH[C_TAU] + (TP)fH[C_D]) * v_star;
        p0 = clamp_lo(p0, TP(1e-30));

        const T BnL0 = ph.L.u[Bn], BnR0 = ph.R.u[Bn];
        TP Bn2 = TP(0.5) * ((TP)BnL0 * (TP)BnL0 + (TP)BnR0 * (TP)BnR0);
        bool use_p0 = (Bn2 / p_hll) < TP(0.1);
        p_lo = use_p0 ? p0 * TP(0.99) : p_hll * TP(0.99);
        p_hi = use_p0 ? p0 * TP(1.01) : p_hll * TP(1.01);
    }
    const T BnL = ph.L.u[Bn], BnR = ph.R.u[Bn];
    bool bn_zero = (fabs(BnL) < T(1e-14)) && (fabs(BnR) < T(1e-14));
    // A face without normal field always takes the HLLE fallback
    // (hlld.py:1512-1531): its flux, state and p* output do not depend on the
    // p* solve, which feeds only the solver counters.  With SKIP_BN0 (the 2D
    // sweeps and the tube kernel of every form but the exact one) the solve
    // is skipped there and the face is marked err = -1, so the counters
    // cover the faces that were solved; the exact form and the per-face
    // plugin solve every face as the reference does.
    if constexpr (!IFT && SKIP_BN0) {
        if (bn_zero) {
#pragma unroll
            for (int k = 0; k < NCONS; ++k) {
                o.F[k] = fH[k];
                if (want_u) o.U[k] = uH[k];
            }
            o.pstar = (T)(-fabs(p_hll) - TP(1e-10));
            o.err = -1;
            o.iters = 0;
            o.flags = RF_BN_ZERO | RF_FAILED;
            return;
        }
    }

    // R vectors on the energy-form state (hlld.py:337-360, :401-428)
    HlldR<TP> C;
    {
        const TP pcm = (TP)cm, pcx = (TP)cx;
        TP UiL[NCONS], UiR[NCONS], FiL[NCONS], FiR[NCONS];
#pragma unroll
        for (int k = 0; k < NCONS; ++k) {
            UiL[k] = (TP)ph.L.u[k];
            UiR[k] = (TP)ph.R.u[k];
            FiL[k] = (TP)ph.L.f[k];
            FiR[k] = (TP)ph.R.f[k];
        }
        UiL[C_TAU] = (TP)(ph.L.u[C_TAU] + ph.L.u[C_D]);
        UiR[C_TAU] = (TP)(ph.R.u[C_TAU] + ph.R.u[C_D]);
        FiL[C_TAU] = (TP)(ph.L.f[C_TAU] + ph.L.f[C_D]);
        FiR[C_TAU] = (TP)(ph.R.f[C_TAU] + ph.R.f[C_D]);
        C.cm = pcm;
        C.cx = pcx;
        C.RSiL = -pcm * UiL[C_SX + i] - FiL[C_SX + i];
        C.RSiR = pcx * UiR[C_SX + i] - FiR[C_SX + i];
        C.RS1L = -pcm * UiL[C_SX + t1] - FiL[C_SX + t1];
        C.RS1R = pcx * UiR[C_SX + t1] - FiR[C_SX + t1];
        C.RS2L = -pcm * UiL[C_SX + t2] - FiL[C_SX + t2];
        C.RS2R = pcx * UiR[C_SX + t2] - FiR[C_SX + t2];
        C.RBiL = -pcm * UiL[C_BX + i] - FiL[C_BX + i];
        C.RBiR = pcx * UiR[C_BX + i] - FiR[C_BX + i];
        C.RB1L = -pcm * UiL[C_BX + t1] - FiL[C_BX + t1];
        C.RB1R = pcx * UiR[C_BX + t1] - FiR[C_BX + t1];
        C.RB2L = -pcm * UiL[C_BX + t2] - FiL[C_BX + t2];
        C.RB2R = pcx * UiR[C_BX + t2] - FiR[C_BX + t2];
        C.RTL = -pcm * UiL[C_TAU] - FiL[C_TAU];
        C.RTR = pcx * UiR[C_TAU] - FiR[C_TAU];
        C.RDL = -pcm * UiL[C_D] - FiL[C_D];
        C.RDR = pcx * UiR[C_D] - FiR[C_D];
        C.S_L = tsign(UiL[C_BX + i]);
        C.S_R = tsign(UiR[C_BX + i]);
        C.BnL = UiL[C_BX + i];
        C.BnR = UiR[C_BX + i];
    }

    // PARK_STRIDE > 0: the two sides' states and fluxes, the HLL flux and the
    // wave speeds -- needed again only by the star states -- wait in the
    // caller's shared-memory slot (park[k * PARK_STRIDE], k < kParkWords)
    // during the p* solve instead of holding registers through it
    if constexpr (PARK_STRIDE > 0) {
#pragma unroll
        for (int k = 0; k < NCONS; ++k) {
            park[(0 * NCONS + k) * PARK_STRIDE] = ph.L.u[k];
            park[(1 * NCONS + k) * PARK_STRIDE] = ph.L.f[k];
            park[(2 * NCONS + k) * PARK_STRIDE] = ph.R.u[k];
            park[(3 * NCONS + k) * PARK_STRIDE] = ph.R.f[k];
            park[(4 * NCONS + k) * PARK_STRIDE] = fH[k];
        }
        park[(5 * NCONS + 0) * PARK_STRIDE] = cm;
        park[(5 * NCONS + 1) * PARK_STRIDE] = cx;
    }
    TP p_star;
    int32_t err = 30, iters_used = 30;
    if constexpr (IFT) {
        p_star = hlld_ift_root(C, given[0]);
        err = 0;
        iters_used = 0;
    } else {
        TP f_lo = hlld_residual_at<INLINE_RES>(C, p_lo);
        TP f_hi = hlld_residual_at<INLINE_RES>(C, p_hi);
        // bracket widening (hlld.py:1314-1321)
#pragma unroll 1
        for (int w = 0; w < 5; ++w) {
            if (!((f_lo * f_hi) > TP(0))) break;
            p_lo = p_lo / TP(2);
            p_hi = p_hi * TP(2);
            f_lo = hlld_residual_at<INLINE_RES>(C, p_lo);
            f_hi = hlld_residual_at<INLINE_RES>(C, p_hi);
        }

        // clamped secant (hlld.py:669-746, _PSTAR_TOL hlld.py:1080, 30 iterations)
        const TP tol = K<TP>::pstar_tol;
        TP x0 = p_lo, x1 = p_hi, f0 = f_lo, f1 = f_hi;
        bool done = false;
#pragma unroll 1
        for (int it = 1; it <= 30; ++it) {
            if (fabs(f1) < tol) {
                err = 0;
                iters_used = it - 1;
                done = true;
                break;
            }
            TP df = f1 - f0;
            bool safe = fabs(df) > TP(1e-30) * fabs(f1);
            TP dx = safe ? f1 * (x1 - x0) / df : TP(0);
            TP x2 = x1 - dx;
            x2 = clamp_lo(x2, TP(1e-30));
            TP f2 = hlld_residual_at<INLINE_RES>(C, x2);
            x0 = x1;
            f0 = f1;
            x1 = x2;
            f1 = f2;
        }
        if (!done && fabs(f1) < tol) {
            err = 0;
            iters_used = 30;
        }
        p_star = x1;
    }

    if constexpr (PARK_STRIDE > 0) {
        // (volatile: read back from the slot, not kept in registers)
        const volatile T *pk = park;
#pragma unroll
        for (int k = 0; k < NCONS; ++k) {
            ph.L.u[k] = pk[(0 * NCONS + k) * PARK_STRIDE];
            ph.L.f[k] = pk[(1 * NCONS + k) * PARK_STRIDE];
            ph.R.u[k] = pk[(2 * NCONS + k) * PARK_STRIDE];
            ph.R.f[k] = pk[(3 * NCONS + k) * PARK_STRIDE];
            fH[k] = pk[(4 * NCONS + k) * PARK_STRIDE];
        }
        cm = pk[(5 * NCONS + 0) * PARK_STRIDE];
        cx = pk[(5 * NCONS + 1) * PARK_STRIDE];
    }
    HlldV<TP> V;
    hlld_vars<true>(C, p_star, V);

    // star states (hlld.py:1359-1445), in the algebra's real type
    const TP pcm = (TP)cm, pcx = (TP)cx;
    const TP laL = V.laL, laR = V.laR;
    TP fac = sdiv(TP(1) - V.KaL2, -C.S_L * V.sqL - V.KaLBc);
    TP vc = laL - (TP)BnR * fac;
    TP vt1 = V.Kt1aL - V.Bt1c * fac;
    TP vt2 = V.Kt2aL - V.Bt2c * fac;
    TP vcomp[3], Bc[3];
    vcomp[i] = vc;
    vcomp[t1] = vt1;
    vcomp[t2] = vt2;
    Bc[i] = (TP)BnR;
    Bc[t1] = V.Bt1c;
    Bc[t2] = V.Bt2c;
    TP vBc = vc * Bc[i] + vt1 * V.Bt1c + vt2 * V.Bt2c;

    bool wave_order_bad = (V.vaR > pcx) || (V.vaL < -pcm) || (vc < laL) || (vc > laR);
    bool failed = (err > 0) || wave_order_bad || bn_zero;
    if constexpr (IFT) failed = given[1] != 0.0;

    if (failed) {
#pragma unroll
        for (int k = 0; k < NCONS; ++k) {
            o.F[k] = fH[k];
            if (want_u) o.U[k] = uH[k];
        }
        o.pstar = (T)(-fabs(p_hll) - TP(1e-10));
    } else {
        TP uaL[NCONS], uaR[NCONS];
        uaL[C_BX + i] = (TP)BnL;
        uaL[C_BX + t1] = V.Bt1aL;
        uaL[C_BX + t2] = V.Bt2aL;
        uaL[C_D] = V.DaL;
        uaL[C_TAU] = V.TauaL;
        uaL[C_SX + i] = V.SaL;
        uaL[C_SX + t1] = V.St1aL;
        uaL[C_SX + t2] = V.St2aL;
        uaR[C_BX + i] = (TP)BnR;
        uaR[C_BX + t1] = V.Bt1aR;
        uaR[C_BX + t2] = V.Bt2aR;
        uaR[C_D] = V.DaR;
        uaR[C_TAU] = V.TauaR;
        uaR[C_SX + i] = V.SaR;
        uaR[C_SX + t1] = V.St1aR;
        uaR[C_SX + t2] = V.St2aR;
        // region selection at xi = 0 (hlld.py:1447-1480)
        const TP vi = TP(0);
        const TP lC = vc;
        const bool cL_mask = vi <= -pcm;
        const bool caL_mask = (-pcm < vi) && (vi <= laL);
        const bool ccL_mask = (laL < vi) && (vi < lC);
        const bool ccR_mask = (lC <= vi) && (vi < laR);
        const bool caR_mask = (laR <= vi) && (vi < pcx);
        const bool cR_mask = vi >= pcx;
        // the contact states are needed only in the contact regions
        const bool need_c = ccL_mask || ccR_mask;
        TP ucD_L = TP(0), ucD_R = TP(0), ucT_L = TP(0), ucT_R = TP(0);
        TP faTL = TP(0), faTR = TP(0);
        if (need_c) {
            faTL = (TP)ph.L.f[C_TAU] + (-pcm) * (uaL[C_TAU] - (TP)ph.L.u[C_TAU]);
            faTR = (TP)ph.R.f[C_TAU] + (pcx) * (uaR[C_TAU] - (TP)ph.R.u[C_TAU]);
            ucD_L = uaL[C_D] * sdiv(laL - V.vaL, laL - vc);
            ucD_R = uaR[C_D] * sdiv(laR - V.vaR, laR - vc);
            ucT_L = sdiv(laL * uaL[C_TAU] - faTL + p_star * vc - vBc * Bc[i], laL - vc);
            ucT_R = sdiv(laR * uaR[C_TAU] - faTR + p_star * vc - vBc * Bc[i], laR - vc);
        }
#pragma unroll
        for (int k = 0; k < NCONS; ++k) {
            const TP fLk = (TP)ph.L.f[k], fRk = (TP)ph.R.f[k];
            const TP uLk = (TP)ph.L.u[k], uRk = (TP)ph.R.u[k];
            const TP faLk = fLk + (-pcm) * (uaL[k] - uLk);
            const TP faRk = fRk + (pcx) * (uaR[k] - uRk);
            TP ucLk = TP(0), ucRk = TP(0);
            if (need_c) {
                if (k == C_D) {
                    ucLk = ucD_L;
                    ucRk = ucD_R;
                } else if (k == C_TAU) {
                    ucLk = ucT_L;
                    ucRk = ucT_R;
                } else if (k >= C_BX) {
                    ucLk = Bc[k - C_BX];
                    ucRk = Bc[k - C_BX];
                } else {
                    const int cc = k - C_SX;
                    ucLk = (ucT_L + p_star + ucD_L) * vcomp[cc] - vBc * Bc[cc];
                    ucRk = (ucT_R + p_star + ucD_R) * vcomp[cc] - vBc * Bc[cc];
                }
            }
            TP f = (TP)fH[k];
            if (cL_mask) f = fLk;
            if (caL_mask) f = faLk;
            if (ccL_mask) f = faLk + laL * (ucLk - uaL[k]);
            if (ccR_mask) f = faRk + laR * (ucRk - uaR[k]);
            if (caR_mask) f = faRk;
            if (cR_mask) f = fRk;
            o.F[k] = (T)f;
            if (want_u) {
                TP u = (TP)uH[k];
                if (cL_mask) u = uLk;
                if (caL_mask) u = uaL[k];
                if (ccL_mask) u = ucLk;
                if (ccR_mask) u = ucRk;
                if (caR_mask) u = uaR[k];
                if (cR_mask) u = uRk;
                o.U[k] = (T)u;
            }
        }
        o.pstar = (T)p_star;
    }
    o.err = err;
    o.iters = iters_used;
    o.flags = (uint8_t)((wave_order_bad ? RF_WAVE_ORDER_BAD : 0) | (bn_zero ? RF_BN_ZERO : 0) |
                        (failed ? RF_FAILED : 0));
}

}  // namespace hlld
