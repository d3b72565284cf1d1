// Forward-mode dual numbers for the tangent (Jacobian) evaluations of the
// adjoint: Dual<N> carries a value and N directional derivatives.  The
// device physics templates instantiate with it unchanged; comparisons and
// branches act on the value, so a tangent evaluation follows the same
// branches as the value computation (limiter cases, region selection and
// clamps are frozen at their forward outcome).
//
// The math functions are hidden friends (found by argument-dependent lookup
// only), so they never hide the double overloads inside namespace hlld.
#pragma once

#include <math.h>

namespace hlld {

template <int N> struct Dual {
    double v;
    double d[N];

    __host__ __device__ constexpr Dual() : v(0.0), d{} {}
    __host__ __device__ constexpr Dual(double x) : v(x), d{} {}

    // x with unit derivative in direction k
    __device__ static Dual var(double x, int k) {
        Dual r(x);
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = (i == k) ? 1.0 : 0.0;
        return r;
    }

    __device__ friend Dual operator+(const Dual &a, const Dual &b) {
        Dual r(a.v + b.v);
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
        return r;
    }
    __device__ friend Dual operator-(const Dual &a, const Dual &b) {
        Dual r(a.v - b.v);
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
        return r;
    }
    __device__ friend Dual operator-(const Dual &a) {
        Dual r(-a.v);
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
        return r;
    }
    __device__ friend Dual operator*(const Dual &a, const Dual &b) {
        Dual r(a.v * b.v);
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
        return r;
    }
    __device__ friend Dual operator/(const Dual &a, const Dual &b) {
        const double q = a.v / b.v;
        const double ib = 1.0 / b.v;
        Dual r(q);
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - q * b.d[i]) * ib;
        return r;
    }
    __device__ Dual &operator+=(const Dual &b) { return *this = *this + b; }
    __device__ Dual &operator-=(const Dual &b) { return *this = *this - b; }
    __device__ Dual &operator*=(const Dual &b) { return *this = *this * b; }

    __device__ friend bool operator<(const Dual &a, const Dual &b) { return a.v < b.v; }
    __device__ friend bool operator>(const Dual &a, const Dual &b) { return a.v > b.v; }
    __device__ friend bool operator<=(const Dual &a, const Dual &b) { return a.v <= b.v; }
    __device__ friend bool operator>=(const Dual &a, const Dual &b) { return a.v >= b.v; }
    __device__ friend bool operator==(const Dual &a, const Dual &b) { return a.v == b.v; }
    __device__ friend bool operator!=(const Dual &a, const Dual &b) { return a.v != b.v; }

    // d sqrt(x) = dx / (2 sqrt(x)); at x = 0 (a clamped argument) the
    // derivative is taken as 0
    __device__ friend Dual sqrt(const Dual &a) {
        const double s = ::sqrt(a.v);
        Dual r(s);
        const double g = s > 0.0 ? 0.5 / s : 0.0;
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = g * a.d[i];
        return r;
    }
    __device__ friend Dual fabs(const Dual &a) {
        const double s = a.v > 0.0 ? 1.0 : (a.v < 0.0 ? -1.0 : 0.0);
        Dual r(::fabs(a.v));
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
        return r;
    }
    __device__ friend bool isnan(const Dual &a) { return ::isnan(a.v); }
};

template <typename T> struct RealOf { static __device__ double get(const T &x) { return (double)x; } };
template <int N> struct RealOf<Dual<N>> {
    static __device__ double get(const Dual<N> &x) { return x.v; }
};
template <typename T> __device__ __forceinline__ double real_of(const T &x) { return RealOf<T>::get(x); }

}  // namespace hlld
