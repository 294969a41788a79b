// bh_dual.cuh - Forward-mode dual numbers with N tangent slots.
//
// Used where a short closed-form expression has to be differentiated with
// respect to a handful of inputs at once: the disc temperature, four-velocity
// and redshift of a disc hit, the escape direction and sky radiance of an
// escaped ray, and the camera tetrad of a frame.  Every operation carries the
// exact derivative of the binary64 primal (chain rule, no finite differences).
#pragma once

#include <cmath>

namespace bhg {
// The functions live beside the type so that argument-dependent lookup finds
// them for Dual arguments while calls on double still reach the C library's.
namespace dual {

template <int N>
struct Dual {
    double v;
    double d[N];

    __host__ __device__ Dual() : v(0.0) {
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
    __host__ __device__ Dual(double x) : v(x) {  // NOLINT: a constant
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
    // The k-th input variable with value x.
    __host__ __device__ static Dual var(double x, int k) {
        Dual r(x);
        r.d[k] = 1.0;
        return r;
    }
    // A constant carrying a given tangent vector.
    __host__ __device__ static Dual with(double x, const double* t) {
        Dual r(x);
        for (int i = 0; i < N; ++i) r.d[i] = t[i];
        return r;
    }
};

template <int N>
__host__ __device__ inline Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v + b.v);
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v - b.v);
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r(-a.v);
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v * b.v);
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    const double q = a.v / b.v;
    Dual<N> r(q);
    const double ib = 1.0 / b.v;
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - q * b.d[i]) * ib;
    return r;
}
template <int N> __host__ __device__ inline Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N> __host__ __device__ inline Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N> __host__ __device__ inline Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N> __host__ __device__ inline Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N>
__host__ __device__ inline Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> r(a.v * b);
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
    return r;
}
template <int N> __host__ __device__ inline Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N> __host__ __device__ inline Dual<N> operator/(const Dual<N>& a, double b) { return a / Dual<N>(b); }
template <int N> __host__ __device__ inline Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }

// f(a) with f'(a) = fp: the chain rule for every unary function below.
template <int N>
__host__ __device__ inline Dual<N> chain(const Dual<N>& a, double f, double fp) {
    Dual<N> r(f);
    for (int i = 0; i < N; ++i) r.d[i] = fp * a.d[i];
    return r;
}
template <int N>
__host__ __device__ inline Dual<N> sqrt(const Dual<N>& a) {
    const double s = ::sqrt(a.v);
    return chain(a, s, (s > 0.0) ? 0.5 / s : 0.0);
}
template <int N>
__host__ __device__ inline Dual<N> log(const Dual<N>& a) { return chain(a, ::log(a.v), 1.0 / a.v); }
template <int N>
__host__ __device__ inline Dual<N> log10(const Dual<N>& a) {
    return chain(a, ::log10(a.v), 1.0 / (a.v * 2.302585092994045684));
}
template <int N>
__host__ __device__ inline Dual<N> exp(const Dual<N>& a) {
    const double e = ::exp(a.v);
    return chain(a, e, e);
}
template <int N>
__host__ __device__ inline Dual<N> sin(const Dual<N>& a) { return chain(a, ::sin(a.v), ::cos(a.v)); }
template <int N>
__host__ __device__ inline Dual<N> cos(const Dual<N>& a) { return chain(a, ::cos(a.v), -::sin(a.v)); }
template <int N>
__host__ __device__ inline Dual<N> acos(const Dual<N>& a) {
    const double s = 1.0 - a.v * a.v;
    return chain(a, ::acos(a.v), (s > 0.0) ? -1.0 / ::sqrt(s) : 0.0);
}
template <int N>
__host__ __device__ inline Dual<N> atan2(const Dual<N>& y, const Dual<N>& x) {
    const double r2 = x.v * x.v + y.v * y.v;
    Dual<N> r(::atan2(y.v, x.v));
    if (r2 > 0.0)
        for (int i = 0; i < N; ++i) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) / r2;
    return r;
}
// a^p for a constant exponent p.
template <int N>
__host__ __device__ inline Dual<N> pow(const Dual<N>& a, double p) {
    const double f = ::pow(a.v, p);
    return chain(a, f, (a.v != 0.0) ? p * f / a.v : 0.0);
}
template <int N>
__host__ __device__ inline Dual<N> cbrt(const Dual<N>& a) {
    const double c = ::cbrt(a.v);
    return chain(a, c, (c != 0.0) ? 1.0 / (3.0 * c * c) : 0.0);
}
template <int N>
__host__ __device__ inline Dual<N> fabs(const Dual<N>& a) { return (a.v < 0.0) ? -a : a; }

}  // namespace dual

using dual::Dual;

}  // namespace bhg
