// bh_jet.cuh - The jet's volumetric emission on the device (binary64).
//
// jet.h:96-315 and render.cpp:44-62, 107-122: the prescribed parabolic jet
// (radius and Lorentz factor ~ z^k, limb-brightened Gaussian sheath,
// emissivity ~ Gamma^-(2+alpha) R^-(3+alpha) (z/z_base)^zeta with soft ends),
// its plasma four-velocity built in the ZAMO frame, and the optically thin
// transfer integral  j_nu0 Integral shape g^(2+alpha) dlambda  accumulated
// with four-point Gauss-Legendre quadrature on each accepted step's dense
// output, truncated at an occluding event.
#pragma once

#include <cuda_runtime.h>

#include "bh_common.cuh"
#include "bh_dp5.cuh"
#include "bh_frame.h"

namespace bhg {

// Four-point Gauss-Legendre nodes and weights on [0, 1] (render.cpp:46-50).
__device__ __forceinline__ double gl_x(int q) {
    return q == 0 ? 0.06943184420297371 : q == 1 ? 0.33000947820757187 : q == 2 ? 0.66999052179242813
                                                                                 : 0.93056815579702629;
}
__device__ __forceinline__ double gl_w(int q) {
    return (q == 0 || q == 3) ? 0.17392742256872693 : 0.32607257743127307;
}

__device__ __forceinline__ double jet_smoothstep(double t) {
    t = dclamp(t, 0.0, 1.0);
    return t * t * (3.0 - 2.0 * t);
}
__device__ __forceinline__ double jet_radius(const FrameParams& F, double z_abs) {
    return F.jet_R_base * pow(dmaxr(z_abs, 1e-6) / F.jet_z_base, F.jet_k);
}
__device__ __forceinline__ double jet_gamma_at(const FrameParams& F, double z_abs) {
    const double t = dminr(1.0, pow(dmaxr(z_abs, 1e-6) / F.jet_z_sat, F.jet_k));
    return 1.0 + (F.jet_gamma_max - 1.0) * t;
}

// Comoving emissivity profile at cylindrical (z, rho) (jet.h:194-207).
__device__ __forceinline__ double jet_shape(const FrameParams& F, double z, double rho) {
    const double az = fabs(z);
    if (az <= F.jet_z_base || az >= F.jet_z_top) return 0.0;
    const double R = jet_radius(F, az);
    const double u = rho / R;
    const double s = (u - F.jet_u_peak) / F.jet_u_wid;
    const double t = u / F.jet_spine_wid;
    const double f = exp(-s * s) + F.jet_spine * exp(-t * t);
    if (f < 1e-9) return 0.0;
    const double g = pow(jet_gamma_at(F, az) / jet_gamma_at(F, F.jet_z_base), -(2.0 + F.jet_alpha)) *
                     pow(R / F.jet_R_base, -(3.0 + F.jet_alpha)) * pow(az / F.jet_z_base, F.jet_zeta);
    const double ramp = jet_smoothstep((az - F.jet_z_base) / (0.5 * F.jet_z_base)) *
                        jet_smoothstep((F.jet_z_top - az) / (0.15 * F.jet_z_top));
    return f * g * ramp;
}

// g = 1 / (p . u) for the jet plasma at (r, th) (jet.h:215-240,
// render.cpp:31-34); p = (p_t, p_r, p_th, p_phi).
__device__ __forceinline__ double jet_redshift(const FrameParams& F, double r, double th, const double p[4]) {
    const double a = F.a, a2 = F.a2;
    double sn, cs;
    sincos(th, &sn, &cs);
    if (fabs(sn) < 1e-9) sn = (sn < 0.0) ? -1e-9 : 1e-9;
    const double sn2 = sn * sn, cs2 = cs * cs;
    const double Sigma = r * r + a2 * cs2;
    const double Delta = r * r - 2.0 * r + a2;
    const double A = (r * r + a2) * (r * r + a2) - a2 * Delta * sn2;
    const double lapse = sqrt(Sigma * Delta / A);
    const double omega = 2.0 * a * r / A;
    const double sqrt_gpp = sn * sqrt(A / Sigma);
    const double z = r * cs;
    const double G_at = jet_gamma_at(F, fabs(z));
    const double v = sqrt(dmaxr(0.0, 1.0 - 1.0 / (G_at * G_at)));
    double v_phi = (F.jet_Omega_F - omega) * sqrt_gpp / dmaxr(lapse, 1e-12);
    v_phi = dclamp(v_phi, -0.5 * v, 0.5 * v);
    const double v_pol = sqrt(dmaxr(0.0, v * v - v_phi * v_phi));
    const double sgn = (cs >= 0.0) ? 1.0 : -1.0;
    const double d_r = sgn * cs;
    const double d_th = -sgn * sn;
    const double G = 1.0 / sqrt(dmaxr(1e-12, 1.0 - v * v));
    // ZAMO legs (kerr.h:283-292): e0 = (1/lapse, 0, 0, omega/lapse),
    // e1 = sqrt(Delta/Sigma) d_r, e2 = d_th / sqrt(Sigma), e3 = sqrt(Sigma/A)/sin d_phi.
    const double u0 = G * (1.0 / lapse);
    const double u1 = G * (v_pol * (d_r * sqrt(Delta / Sigma)));
    const double u2 = G * (v_pol * (d_th * (1.0 / sqrt(Sigma))));
    const double u3 = G * (omega / lapse + v_phi * (sqrt(Sigma / A) / sn));
    const double ku = p[0] * u0 + p[1] * u1 + p[2] * u2 + p[3] * u3;
    return (ku > 1e-12) ? 1.0 / ku : 0.0;
}

// Shortest distance from the origin to the segment p0 -> p1 (render.cpp:55-62).
__device__ __forceinline__ double segment_distance_to_origin(const double p0[3], const double p1[3]) {
    const double d0 = p1[0] - p0[0], d1 = p1[1] - p0[1], d2 = p1[2] - p0[2];
    const double dd = d0 * d0 + d1 * d1 + d2 * d2;
    double t = 0.0;
    if (dd > 0.0) t = dclamp(-(p0[0] * d0 + p0[1] * d1 + p0[2] * d2) / dd, 0.0, 1.0);
    const double q0 = p0[0] + t * d0, q1 = p0[1] + t * d1, q2 = p0[2] + t * d2;
    return sqrt(q0 * q0 + q1 * q1 + q2 * q2);
}

// Pseudo-Cartesian position (geodesic.h:256-262).
__device__ __forceinline__ void bl_cartesian(double a, double r, double th, double ph, double q[3]) {
    const double rr = sqrt(r * r + a * a);
    double sn, cs, sp, cp;
    sincos(th, &sn, &cs);
    sincos(ph, &sp, &cp);
    q[0] = rr * sn * cp;
    q[1] = rr * sn * sp;
    q[2] = r * cs;
}

// The transfer integral over [0, s_end] of one step of size h from the dense
// polynomials of r, th, p_r, p_th (render.cpp:107-122); p_t = -E, p_phi = L_z.
__device__ __noinline__ double jet_step_integral(const FrameParams& F, const DenseC& cr, const DenseC& cth,
                                                 const DenseC& cpr, const DenseC& cpth, double E, double Lz,
                                                 double h, double s_end) {
    if (!(s_end > 0.0)) return 0.0;
    double sum = 0.0;
    #pragma unroll 1
    for (int q = 0; q < 4; ++q) {
        const double s = gl_x(q) * s_end;
        const double r = dense_eval(cr, s), th = dense_eval(cth, s);
        double sn, cs;
        sincos(th, &sn, &cs);
        const double z = r * cs;
        const double rho = sqrt(r * r + F.a2) * sn;
        const double sh = jet_shape(F, z, rho);
        if (sh <= 0.0) continue;
        const double p[4] = {-E, dense_eval(cpr, s), dense_eval(cpth, s), Lz};
        const double gf = jet_redshift(F, r, th, p);
        if (gf <= 0.0) continue;
        sum += gl_w(q) * sh * pow(gf, 2.0 + F.jet_alpha);
    }
    return F.jet_j_nu0 * sum * h * s_end;
}

}  // namespace bhg
