// bh_dp5.cuh - The Dormand-Prince 5(4) tableau, its PI-controller constants
// and the dense-output polynomial (geodesic.h:77-121, 176-185), shared by the
// trace kernels and the adjoint kernel.
#pragma once

#include <cmath>

namespace bhg {

// ---- Dormand-Prince 5(4) (Hairer, Norsett & Wanner, Solving ODEs I, II.4) ----
constexpr double A21 = 1.0 / 5.0;
constexpr double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
constexpr double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
constexpr double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0, A53 = 64448.0 / 6561.0,
                 A54 = -212.0 / 729.0;
constexpr double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0, A63 = 46732.0 / 5247.0,
                 A64 = 49.0 / 176.0, A65 = -5103.0 / 18656.0;
constexpr double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0,
                 B5 = -2187.0 / 6784.0, B6 = 11.0 / 84.0;
constexpr double E1 = 35.0 / 384.0 - 5179.0 / 57600.0;
constexpr double E3 = 500.0 / 1113.0 - 7571.0 / 16695.0;
constexpr double E4 = 125.0 / 192.0 - 393.0 / 640.0;
constexpr double E5 = -2187.0 / 6784.0 - (-92097.0 / 339200.0);
constexpr double E6 = 11.0 / 84.0 - 187.0 / 2100.0;
constexpr double E7 = 0.0 - 1.0 / 40.0;
constexpr double D1 = -12715105075.0 / 11282082432.0, D3 = 87487479700.0 / 32700410799.0,
                 D4 = -10690763975.0 / 1880347072.0, D5 = 701980252875.0 / 199316789632.0,
                 D6 = -1453857185.0 / 822651844.0, D7 = 69997945.0 / 29380423.0;
// PI controller (Gustafsson): alpha = 0.7/5, beta = 0.4/5, safety 0.9, [0.2, 5].
constexpr double kAlpha = 0.7 / 5.0, kBeta = 0.4 / 5.0;
constexpr double kLnErrFloor = -9.210340371976184;   // ln 1e-4, the floor of err_prev

// Dense-output polynomial of one component (geodesic.h:109-121, 176-185).
struct DenseC { double r1, r2, r3, r4, r5; };

__host__ __device__ __forceinline__ DenseC dense_coef(double h, double y, double yn, double k1, double k3,
                                                      double k4, double k5, double k6, double k7) {
    DenseC c;
    c.r1 = y;
    c.r2 = yn - y;
    c.r3 = h * k1 - c.r2;
    c.r4 = c.r2 - h * k7 - c.r3;
    c.r5 = h * (D1 * k1 + D3 * k3 + D4 * k4 + D5 * k5 + D6 * k6 + D7 * k7);
    return c;
}
__host__ __device__ __forceinline__ double dense_eval(const DenseC& c, double s) {
    const double s1 = 1.0 - s;
    return c.r1 + s * (c.r2 + s1 * (c.r3 + s * (c.r4 + s1 * c.r5)));
}
__host__ __device__ __forceinline__ double dense_deriv(const DenseC& c, double s) {
    const double u = 1.0 - s;
    return c.r2 + (u - s) * c.r3 + (2.0 * s * u - s * s) * c.r4 + (2.0 * s * u * u - 2.0 * s * s * u) * c.r5;
}

// Crossing of `target` by the dense polynomial on [0, 1]: safeguarded Newton
// inside a shrinking bracket.  It converges to the same point (to rounding) as
// the reference's 60-step bisection on the same polynomial (render.cpp:158-166,
// 181-189), in a handful of binary64 evaluations.  f(0) <= 0 -> s = 0.
__host__ __device__ inline double dense_crossing(const DenseC& c, double target) {
    double lo = 0.0, hi = 1.0;
    const double f0 = c.r1 - target;
    const double f1 = (c.r1 + c.r2) - target;
    if (f0 == 0.0) return 0.0;
    if (f1 == 0.0 || !((f0 < 0.0) != (f1 < 0.0))) {
        // no bracket (the crossing and back inside one step): plain bisection
        // on the sign at s = 0, as the reference does
        for (int it = 0; it < 60; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (((dense_eval(c, mid) - target) < 0.0) != (f0 < 0.0)) hi = mid; else lo = mid;
        }
        return 0.5 * (lo + hi);
    }
    const bool neg0 = f0 < 0.0;
    double s = f0 / (f0 - f1);
    for (int it = 0; it < 50; ++it) {
        const double f = dense_eval(c, s) - target;
        if (f == 0.0) return s;
        if ((f < 0.0) == neg0) lo = s; else hi = s;
        const double d = dense_deriv(c, s);
        double sn = s - f / d;
        if (!(sn > lo && sn < hi)) sn = 0.5 * (lo + hi);
        if (std::fabs(sn - s) <= 4e-16 || hi - lo <= 4e-16) return sn;
        s = sn;
    }
    return s;
}

}  // namespace bhg
