// bh_adjoint.cuh - The per-ray discrete adjoint of the binary64 render path.
//
// For one camera ray this computes the ray's luminance Y (the CIE Y of its
// shaded colour) and, for a loss weight w = dLoss/dY, the ray's contribution
// to dLoss/d(spin, inclination, Eddington ratio, r_out):
//
//   1. forward: the ray is integrated with the render path's DP5(4) scheme,
//      PI controller, step limiter and events (render.cpp:69-260,
//      geodesic.h:123-204); the state (y, h, controller memory) after every
//      `interval` accepted steps is stored in the ray's checkpoint slots.
//      When the slots are full every second checkpoint is dropped and the
//      interval doubles, so memory stays bounded for any step count;
//   2. seed: the shading of the hit (disc: Novikov-Thorne temperature,
//      Keplerian redshift, blackbody table, disc.h:94-126, render.cpp:31-34,
//      spectrum.cpp:123-134; sky: the escape direction and the star field,
//      render.cpp:15-26, scene.h:111-158) is differentiated in forward mode
//      (dual numbers) with respect to the hit state and the parameters;
//   3. reverse: segment by segment from the last, the accepted steps are
//      replayed from their checkpoint and the adjoint state is carried back
//      through each DP5 step in reverse (the vector-Jacobian products of its
//      six stages), with the accepted step sizes held fixed: the discrete
//      adjoint of the step sequence the forward pass took.  The disc-crossing
//      root s* (theta(s*) = pi/2 on the dense-output polynomial) is
//      differentiated by the implicit-function theorem;
//   4. the adjoint of the initial photon is contracted with the derivatives of
//      the initial state (camera tetrad and metric at the camera).
//
// The disc's edges are steps in the image: a ray's luminance does not depend
// on r_out except when its crossing radius passes r_out, so the derivative of
// a point-sampled frame with respect to r_out is zero, and the edges move
// with the spin and the inclination too.  The edge term (edge_sample below)
// is the derivative of the frame averaged over each sample's cell: for a
// crossing near an edge, the luminance jump times the edge's length in the
// cell times its speed, the image-plane gradient of the crossing radius and
// its parameter derivatives coming from a reverse sweep seeded with that
// radius.
//
// All arithmetic is binary64.  The functions compile for the host as well, so
// the same code can be checked against finite differences on a CPU.
#pragma once

#include <cmath>
#include <cstdint>

#include "../../include/bh_gpu.h"
#include "bh_adjoint.h"
#include "bh_common.cuh"
#include "bh_dp5.cuh"
#include "bh_dual.cuh"
#include "bh_frame.h"

#if defined(__CUDA_ARCH__)
#define BHA_NOINLINE __noinline__
#else
#define BHA_NOINLINE
#endif

namespace bhg {
namespace adj {

// Exact (non-contracted) binary64 products and sums for the ray set-up, so the
// initial photon is the render path's to the last bit.
__host__ __device__ __forceinline__ double xm(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ __forceinline__ double xa(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
__host__ __device__ __forceinline__ double xs(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
__host__ __device__ __forceinline__ double xd(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}
__host__ __device__ __forceinline__ double xsqrt(double a) {
#if defined(__CUDA_ARCH__)
    return __dsqrt_rn(a);
#else
    return std::sqrt(a);
#endif
}
__host__ __device__ __forceinline__ bool is_finite(double x) {
#if defined(__CUDA_ARCH__)
    return isfinite(x);
#else
    return std::isfinite(x);
#endif
}
__host__ __device__ __forceinline__ void sc(double x, double* s, double* c) {
#if defined(__CUDA_ARCH__)
    sincos(x, s, c);
#else
    *s = std::sin(x);
    *c = std::cos(x);
#endif
}

// Constants of a ray's right-hand side.
struct RayC {
    double a, a2, E, Lz, rp, rm;
    int factored;
};

// Hamilton's equations in Carter's separated form (the render path's
// right-hand side, geodesic.h:50-71):
//   2 Sigma H = Delta p_r^2 + p_th^2 + (L_z - a E sin^2)^2 / sin^2
//               - ((r^2 + a^2) E - a L_z)^2 / Delta,
// at sin(th) = sn, cos(th) = cs, with one reciprocal (of Sigma Delta sin^2)
// for the three quotients.  d = (dt, dr, dth, dphi, dp_r, dp_th) / dlambda.
__host__ __device__ BHA_NOINLINE void rhs6(const RayC& c, double r, double sn, double cs, double pr, double pth,
                                           double d[6]) {
    if (fabs(sn) < 1e-9) sn = (sn < 0.0) ? -1e-9 : 1e-9;   // kerr.h:51
    const double sn2 = sn * sn, cs2 = cs * cs, r2 = r * r;
    const double S = r2 + c.a2 * cs2;
    const double D = c.factored ? (r - c.rp) * (r - c.rm) : (r2 - 2.0 * r + c.a2);
    const double inv = rcp_nr(S * D * sn2);
    const double iS = inv * D * sn2, iD = inv * S * sn2, isn2 = inv * S * D;
    const double r2a2 = r2 + c.a2;
    const double K = r2a2 * c.E - c.a * c.Lz;
    const double Lp = c.Lz - c.a * c.E * sn2;
    const double KiD = K * iD;
    const double B = D * pr * pr + pth * pth + Lp * Lp * isn2 - K * KiD;
    const double Dr = 2.0 * r - 2.0;
    d[0] = iS * (c.a * Lp + r2a2 * KiD);
    d[1] = D * pr * iS;
    d[2] = pth * iS;
    d[3] = iS * (Lp * isn2 + c.a * KiD);
    d[4] = -0.5 * iS * (Dr * pr * pr - 4.0 * r * c.E * KiD + Dr * KiD * KiD - 2.0 * r * B * iS);
    d[5] = -sn * cs * iS * (c.a2 * c.E * c.E - c.Lz * c.Lz * isn2 * isn2 + c.a2 * B * iS);
}

// The right-hand side at angle th; *sn_out, *cs_out receive sin(th), cos(th).
__host__ __device__ __forceinline__ void rhs6_th(const RayC& c, double r, double th, double pr, double pth,
                                                 double d[6], double* sn_out, double* cs_out) {
    double sn, cs;
    sc(th, &sn, &cs);
    rhs6(c, r, sn, cs, pr, pth, d);
    *sn_out = sn;
    *cs_out = cs;
}

// Vector-Jacobian product of rhs6 at (r, th, p_r, p_th) given sin(th) = sn
// and cos(th) = cs: for db = dLoss/d(d), adds dLoss/d(r, th, p_r, p_th) into
// g[0..3] and dLoss/d(E, L_z, a) into *Eb, *Lzb, *ab.  Reverse-mode
// differentiation of the expressions of rhs6, written out.
__host__ __device__ BHA_NOINLINE void rhs6_vjp(const RayC& c, double r, double sn, double cs, double pr, double pth,
                                               const double db[6], double g[4], double* Eb, double* Lzb,
                                               double* ab) {
    const double sn_true = sn;
    const bool clamped = fabs(sn) < 1e-9;
    if (clamped) sn = (sn < 0.0) ? -1e-9 : 1e-9;
    const double a = c.a, a2 = c.a2, E = c.E, Lz = c.Lz;
    const double sn2 = sn * sn, cs2 = cs * cs, r2 = r * r;
    const double S = r2 + a2 * cs2;
    const double D = c.factored ? (r - c.rp) * (r - c.rm) : (r2 - 2.0 * r + a2);
    const double inv = rcp_nr(S * D * sn2);
    const double iS = inv * D * sn2, iD = inv * S * sn2, isn2 = inv * S * D;
    const double r2a2 = r2 + a2;
    const double K = r2a2 * E - a * Lz;
    const double Lp = Lz - a * E * sn2;
    const double KiD = K * iD;
    const double B = D * pr * pr + pth * pth + Lp * Lp * isn2 - K * KiD;
    const double Dr = 2.0 * r - 2.0;
    const double X0 = a * Lp + r2a2 * KiD;
    const double X3 = Lp * isn2 + a * KiD;
    const double X4 = Dr * pr * pr - 4.0 * r * E * KiD + Dr * KiD * KiD - 2.0 * r * B * iS;
    const double X5 = a2 * E * E - Lz * Lz * isn2 * isn2 + a2 * B * iS;
    const double P5 = -sn * cs;

    // outputs
    double b_iS = db[0] * X0 + db[1] * D * pr + db[2] * pth + db[3] * X3 - 0.5 * db[4] * X4 + db[5] * P5 * X5;
    const double bX0 = db[0] * iS;
    double bD = db[1] * pr * iS;
    double bpr = db[1] * D * iS;
    double bpth = db[2] * iS;
    const double bX3 = db[3] * iS;
    const double bX4 = -0.5 * db[4] * iS;
    const double bP5 = db[5] * iS * X5;
    const double bX5 = db[5] * P5 * iS;
    // X0 = a Lp + r2a2 KiD
    double ba = bX0 * Lp;
    double bLp = bX0 * a;
    double br2a2 = bX0 * KiD;
    double bKiD = bX0 * r2a2;
    // X3 = Lp isn2 + a KiD
    bLp += bX3 * isn2;
    double bisn2 = bX3 * Lp;
    ba += bX3 * KiD;
    bKiD += bX3 * a;
    // X4 = Dr pr^2 - 4 r E KiD + Dr KiD^2 - 2 r B iS
    const double bDr = bX4 * (pr * pr + KiD * KiD);
    bpr += bX4 * 2.0 * Dr * pr;
    double br = bX4 * (-4.0 * E * KiD - 2.0 * B * iS);
    double bE = bX4 * (-4.0 * r * KiD);
    bKiD += bX4 * (-4.0 * r * E + 2.0 * Dr * KiD);
    double bB = bX4 * (-2.0 * r * iS);
    b_iS += bX4 * (-2.0 * r * B);
    // X5 = a2 E^2 - Lz^2 isn2^2 + a2 B iS
    double ba2 = bX5 * (E * E + B * iS);
    bE += bX5 * 2.0 * a2 * E;
    double bLz = bX5 * (-2.0 * Lz * isn2 * isn2);
    bisn2 += bX5 * (-2.0 * Lz * Lz * isn2);
    bB += bX5 * a2 * iS;
    b_iS += bX5 * a2 * B;
    // P5 = -sn cs
    double bsn = -bP5 * cs;
    double bcs = -bP5 * sn;
    // Dr = 2 r - 2
    br += 2.0 * bDr;
    // B = D pr^2 + pth^2 + Lp^2 isn2 - K KiD
    bD += bB * pr * pr;
    bpr += bB * 2.0 * D * pr;
    bpth += bB * 2.0 * pth;
    bLp += bB * 2.0 * Lp * isn2;
    bisn2 += bB * Lp * Lp;
    double bK = -bB * KiD;
    bKiD += -bB * K;
    // KiD = K iD
    bK += bKiD * iD;
    const double biD = bKiD * K;
    // Lp = Lz - a E sn2
    bLz += bLp;
    ba += -bLp * E * sn2;
    bE += -bLp * a * sn2;
    double bsn2 = -bLp * a * E;
    // K = r2a2 E - a Lz
    br2a2 += bK * E;
    bE += bK * r2a2;
    ba += -bK * Lz;
    bLz += -bK * a;
    // r2a2 = r2 + a2
    double br2 = br2a2;
    ba2 += br2a2;
    // the reciprocals
    const double bS = -b_iS * iS * iS;
    bD += -biD * iD * iD;
    bsn2 += -bisn2 * isn2 * isn2;
    // Delta = r^2 - 2 r + a^2 (the factored form has the same value)
    br += bD * (2.0 * r - 2.0);
    ba2 += bD;
    // Sigma = r2 + a2 cs2
    br2 += bS;
    ba2 += bS * cs2;
    const double bcs2 = bS * a2;
    br += 2.0 * r * br2;
    bsn += 2.0 * sn * bsn2;
    bcs += 2.0 * cs * bcs2;
    ba += 2.0 * a * ba2;
    const double bth = (clamped ? 0.0 : cs * bsn) - sn_true * bcs;
    g[0] += br;
    g[1] += bth;
    g[2] += bpr;
    g[3] += bpth;
    *Eb += bE;
    *Lzb += bLz;
    *ab += ba;
}

// Integrator state of one ray.
struct Integ {
    double y[6];        // t, r, th, phi, p_r, p_th
    double k1[6];       // FSAL stage at y
    double h;
    double errp_mem;    // beta ln err_prev, err_prev the last accepted error norm (>= 1e-4)
    double c0;          // cos(th) at y
    int have_k1;
    int tries;
    int steps;
};

// One accepted step of an attempt loop.
struct StepRec {
    double y[6];        // state at the start of the step
    double yn[6];
    double kr[7], kth[7];   // r and th components of k1..k7 (dense output)
    double h;
    double c0, c7;      // cos(th) at y and at yn
};

// Attempt steps from `s` until one is accepted (render.cpp:127-137 with
// geodesic.h:123-204), then advance `s`.  Returns false when no acceptable
// step was found (more than 40 rejections or |h| < 1e-14).
__host__ __device__ BHA_NOINLINE bool advance(const FrameParams& F, const RayC& c, Integ& s, StepRec* rec) {
    constexpr double A[6][5] = {{0, 0, 0, 0, 0},
                                {A21, 0, 0, 0, 0},
                                {A31, A32, 0, 0, 0},
                                {A41, A42, A43, 0, 0},
                                {A51, A52, A53, A54, 0},
                                {A61, A62, A63, A64, A65}};
    if (!s.have_k1) {
        double sn0;
        rhs6_th(c, s.y[1], s.y[2], s.y[4], s.y[5], s.k1, &sn0, &s.c0);
        s.have_k1 = 1;
    }
    for (;;) {
        if (s.tries == 0) {
            const double hmax = 0.05 * dmaxr(1.0, s.y[1] - F.r_h) + 0.01;
            if (s.h > hmax) s.h = hmax;
        }
        const double h = s.h;
        double k[7][6], t[6], yn[6], c7, sn, cs;
        for (int i = 0; i < 6; ++i) k[0][i] = s.k1[i];
        #pragma unroll
        for (int j = 1; j < 6; ++j) {
            #pragma unroll
            for (int i = 0; i < 6; ++i) {
                double acc = 0.0;
                #pragma unroll
                for (int l = 0; l < j; ++l) acc += A[j][l] * k[l][i];
                t[i] = s.y[i] + h * acc;
            }
            rhs6_th(c, t[1], t[2], t[4], t[5], k[j], &sn, &cs);
        }
        for (int i = 0; i < 6; ++i)
            yn[i] = s.y[i] + h * (B1 * k[0][i] + B3 * k[2][i] + B4 * k[3][i] + B5 * k[4][i] + B6 * k[5][i]);
        rhs6_th(c, yn[1], yn[2], yn[4], yn[5], k[6], &sn, &c7);
        double err2 = 0.0;
        for (int i = 0; i < 6; ++i) {
            const double e = h * (E1 * k[0][i] + E3 * k[2][i] + E4 * k[3][i] + E5 * k[4][i] + E6 * k[5][i] +
                                  E7 * k[6][i]);
            const double scl = F.atol + F.rtol * dmaxr(fabs(s.y[i]), fabs(yn[i]));
            const double q = e * rcp_nr(scl);
            err2 += q * q;
        }
        // err: the square of the RMS norm; the PI factor 0.9 err^-alpha
        // err_prev^beta (geodesic.h:171-173) as one exp of logarithms, the
        // forward pass and every replay alike
        double err = err2 * 0.125;
        if (!is_finite(err)) err = 1e10;
        const double lq = log(dmaxr(err, 1e-32));
        double fac = 0.9 * exp(fma(-0.5 * kAlpha, lq, s.errp_mem));
        fac = dclamp(fac, 0.2, 5.0);
        if (!(err <= 1.0)) {
            s.h *= dminr(fac, 1.0);
            if (++s.tries > 40 || fabs(s.h) < 1e-14) return false;
            continue;
        }
        s.tries = 0;
        ++s.steps;
        if (rec) {
            for (int i = 0; i < 6; ++i) {
                rec->y[i] = s.y[i];
                rec->yn[i] = yn[i];
            }
            for (int j = 0; j < 7; ++j) {
                rec->kr[j] = k[j][1];
                rec->kth[j] = k[j][2];
            }
            rec->h = h;
            rec->c0 = s.c0;
            rec->c7 = c7;
        }
        for (int i = 0; i < 6; ++i) {
            s.y[i] = yn[i];
            s.k1[i] = k[6][i];
        }
        s.c0 = c7;
        s.errp_mem = kBeta * dmaxr(0.5 * lq, kLnErrFloor);
        s.h = h * fac;
        return true;
    }
}

// Equatorial target angle pi/2 + m pi between th0 and th1 (render.cpp:180-189).
__host__ __device__ __forceinline__ double crossing_target(double th0, double th1) {
    const double m = (th1 > th0) ? ceil((th0 - 0.5 * kPi) / kPi) : floor((th0 - 0.5 * kPi) / kPi);
    return 0.5 * kPi + m * kPi;
}

// Reverse of one component's dense output at s with weight v (adds into the
// adjoints of y, yn and the stages k1, k3..k7 held as kb[0], kb[2..6]).
__host__ __device__ __forceinline__ void dense_vjp(double h, double s, double v, int i, double* yb, double* ynb,
                                                   double kb[7][6]) {
    const double s1 = 1.0 - s;
    const double r1b = v;
    double r2b = s * v;
    double r3b = s * s1 * v;
    const double r4b = s * s * s1 * v;
    const double r5b = s * s * s1 * s1 * v;
    kb[0][i] += h * D1 * r5b;
    kb[2][i] += h * D3 * r5b;
    kb[3][i] += h * D4 * r5b;
    kb[4][i] += h * D5 * r5b;
    kb[5][i] += h * D6 * r5b;
    kb[6][i] += h * D7 * r5b;
    r2b += r4b;
    kb[6][i] += -h * r4b;
    r3b += -r4b;
    kb[0][i] += h * r3b;
    r2b += -r3b;
    ynb[i] += r2b;
    yb[i] += -r2b;
    yb[i] += r1b;
}

// Carries the adjoint yb of the state after one accepted step (from ys with
// step h) back to the state before it, accumulating the E, L_z and spin
// adjoints.  rstar_b != 0 marks the step that ends on the disc: the hit
// radius r* = P_r(s*) at the crossing theta(s*) = target of the dense
// polynomials then receives the weight rstar_b (and yb, the adjoint of the
// step's end state, is zero).
__host__ __device__ BHA_NOINLINE void step_vjp(const RayC& c, const double ys[6], double h, double yb[6],
                                               double* Eb, double* Lzb, double* ab, double rstar_b) {
    constexpr double A[6][5] = {{0, 0, 0, 0, 0},
                                {A21, 0, 0, 0, 0},
                                {A31, A32, 0, 0, 0},
                                {A41, A42, A43, 0, 0},
                                {A51, A52, A53, A54, 0},
                                {A61, A62, A63, A64, A65}};
    // Stage inputs (r, th, p_r, p_th) and the sine and cosine of their th,
    // kept for the stages' vector-Jacobian products.
    double k[7][6], Y[6][4], Ysn[6], Ycs[6], t[6], yn[6];
    Y[0][0] = ys[1]; Y[0][1] = ys[2]; Y[0][2] = ys[4]; Y[0][3] = ys[5];
    rhs6_th(c, ys[1], ys[2], ys[4], ys[5], k[0], &Ysn[0], &Ycs[0]);
    #pragma unroll
    for (int j = 1; j < 6; ++j) {
        #pragma unroll
        for (int i = 0; i < 6; ++i) {
            double acc = 0.0;
            #pragma unroll
            for (int l = 0; l < j; ++l) acc += A[j][l] * k[l][i];
            t[i] = ys[i] + h * acc;
        }
        Y[j][0] = t[1]; Y[j][1] = t[2]; Y[j][2] = t[4]; Y[j][3] = t[5];
        rhs6_th(c, t[1], t[2], t[4], t[5], k[j], &Ysn[j], &Ycs[j]);
    }
    for (int i = 0; i < 6; ++i)
        yn[i] = ys[i] + h * (B1 * k[0][i] + B3 * k[2][i] + B4 * k[3][i] + B5 * k[4][i] + B6 * k[5][i]);

    double kb[7][6], ynb[6], ybar[6];
    for (int j = 0; j < 7; ++j)
        for (int i = 0; i < 6; ++i) kb[j][i] = 0.0;
    for (int i = 0; i < 6; ++i) {
        ynb[i] = yb[i];
        ybar[i] = 0.0;
    }
    if (rstar_b != 0.0) {
        double sn7, cs7;
        rhs6_th(c, yn[1], yn[2], yn[4], yn[5], k[6], &sn7, &cs7);
        const DenseC cth = dense_coef(h, ys[2], yn[2], k[0][2], k[2][2], k[3][2], k[4][2], k[5][2], k[6][2]);
        const DenseC crr = dense_coef(h, ys[1], yn[1], k[0][1], k[2][1], k[3][1], k[4][1], k[5][1], k[6][1]);
        const double target = crossing_target(cth.r1, cth.r1 + cth.r2);
        const double s = dense_crossing(cth, target);
        const double dth = dense_deriv(cth, s), dr = dense_deriv(crr, s);
        dense_vjp(h, s, rstar_b, 1, ybar, ynb, kb);
        if (dth != 0.0) dense_vjp(h, s, -rstar_b * dr / dth, 2, ybar, ynb, kb);
        double g4[4] = {0.0, 0.0, 0.0, 0.0};
        rhs6_vjp(c, yn[1], sn7, cs7, yn[4], yn[5], kb[6], g4, Eb, Lzb, ab);
        ynb[1] += g4[0]; ynb[2] += g4[1]; ynb[4] += g4[2]; ynb[5] += g4[3];
    }
    for (int i = 0; i < 6; ++i) {
        ybar[i] += ynb[i];
        kb[0][i] += h * B1 * ynb[i];
        kb[2][i] += h * B3 * ynb[i];
        kb[3][i] += h * B4 * ynb[i];
        kb[4][i] += h * B5 * ynb[i];
        kb[5][i] += h * B6 * ynb[i];
    }
    #pragma unroll
    for (int j = 5; j >= 0; --j) {
        double g4[4] = {0.0, 0.0, 0.0, 0.0};
        rhs6_vjp(c, Y[j][0], Ysn[j], Ycs[j], Y[j][2], Y[j][3], kb[j], g4, Eb, Lzb, ab);
        const double Yb[6] = {0.0, g4[0], g4[1], 0.0, g4[2], g4[3]};
        #pragma unroll
        for (int i = 0; i < 6; ++i) {
            ybar[i] += Yb[i];
            #pragma unroll
            for (int l = 0; l < j; ++l) kb[l][i] += h * A[j][l] * Yb[i];
        }
    }
    for (int i = 0; i < 6; ++i) yb[i] = ybar[i];
}

// ---- shading in forward mode ---------------------------------------------------

using D5 = Dual<5>;   // slots: r, E, L_z, spin, Eddington ratio
using D8 = Dual<8>;   // slots: r, th, phi, p_r, p_th, E, L_z, spin
enum { kS5R = 0, kS5E = 1, kS5L = 2, kS5A = 3, kS5M = 4 };

template <class T>
__host__ __device__ T circ_energy_t(const T& a, const T& r, int sg) {
    const T sr = sqrt(r);
    const T num = r * r - 2.0 * r + (double)sg * a * sr;
    const T den = r * sqrt(r * r - 3.0 * r + 2.0 * (double)sg * a * sr);
    return num / den;
}
template <class T>
__host__ __device__ T circ_angmom_t(const T& a, const T& r, int sg) {
    const T sr = sqrt(r);
    const T num = (double)sg * sr * (r * r - 2.0 * (double)sg * a * sr + a * a);
    const T den = r * sqrt(r * r - 3.0 * r + 2.0 * (double)sg * a * sr);
    return num / den;
}

// CIE Y of the blackbody table at temperature T (spectrum.cpp:123-134).
template <class T>
__host__ __device__ T blackbody_Y(const double* tab, const T& Tk) {
    const double kLogTMin = 1.6989700043360187, kLogTMax = 9.4771212547196626;
    T Tc = Tk;
    if (Tk.v < 50.0) Tc = T(50.0);
    if (Tk.v > 3.0e9) Tc = T(3.0e9);
    const T f = (log10(Tc) - kLogTMin) / (kLogTMax - kLogTMin) * (double)(kTableN - 1);
    int i = (int)f.v;
    i = (i < 0) ? 0 : (i > kTableN - 2 ? kTableN - 2 : i);
    const T u = f - (double)i;
    return exp(tab[kTableN + i] * (1.0 - u) + tab[kTableN + i + 1] * u);
}

// Luminance of a disc hit at radius r (disc.h:94-121, kerr.h:260-266,
// render.cpp:31-34, 277-297) as a dual over (r, E, L_z, spin, Eddington).
__host__ __device__ inline D5 disc_luminance(const FrameParams& F, const AdjointFrame& X, const double* tab,
                                             double r_hit, double E_, double Lz_) {
    if (r_hit <= F.r_in || r_hit > F.r_out) return D5(0.0);
    const D5 r = D5::var(r_hit, kS5R);
    const D5 E = D5::var(E_, kS5E);
    const D5 Lz = D5::var(Lz_, kS5L);
    auto par = [](double v, double da) {
        D5 q(v);
        q.d[kS5A] = da;
        return q;
    };
    const int sg = F.disc_sigma;
    const D5 a = par(F.disc_a, X.d_disc_a);
    const D5 x0 = par(F.x0, X.d_x0);
    const D5 x = sqrt(r);
    D5 W = x - x0 - 1.5 * a * log(x / x0);
    for (int i = 0; i < 3; ++i)
        if (F.pt_c[i] != 0.0) {
            const D5 ci = par(F.pt_c[i], X.d_pt_c[i]);
            const D5 xi = par(F.pt_x[i], X.d_pt_x[i]);
            const D5 di = par(F.pt_den[i], X.d_pt_den[i]);
            W = W - ci * log((x - xi) / di);
        }
    const D5 r32 = r * sqrt(r);
    const D5 dd = r32 + (double)sg * a;
    const D5 Om = (double)sg / dd;
    const D5 dOm = -(double)sg * 1.5 * sqrt(r) / (dd * dd);
    const D5 Ec = circ_energy_t(a, r, sg);
    const D5 Lc = circ_angmom_t(a, r, sg);
    const D5 den = Ec - Om * Lc;
    if (!(den.v > 0.0)) return D5(0.0);
    const D5 Fd = (-dOm) / (4.0 * kPi * r * den * den) * W;
    if (!(Fd.v > 0.0 && is_finite(Fd.v))) return D5(0.0);
    D5 mdot(F.disc_mdot);
    mdot.d[kS5A] = X.d_mdot_da;
    mdot.d[kS5M] = X.d_mdot_dedd;
    const D5 Fl = Fd * mdot * (2.99792458e8 * 2.99792458e8) / F.disc_rg2;
    if (!(Fl.v > 0.0)) return D5(0.0);
    const D5 T = pow(Fl / 5.670374419e-8, 0.25);
    // Keplerian four-velocity and g = 1 / (p . u), p_t = -E, p_phi = L_z.
    const D5 dsc = r * r * r - 3.0 * r * r + 2.0 * (double)sg * a * r32;
    const D5 ut = dd / sqrt(dsc.v > 1e-300 ? dsc : D5(1e-300));
    const D5 ku = (-E) * ut + Lz * (Om * ut);
    if (!(ku.v > 1e-12)) return D5(0.0);
    const D5 g = 1.0 / ku;
    return blackbody_Y(tab, g * T);
}

// Escape direction (render.cpp:15-26, normalised as render.cpp:364-366) as a
// dual over (r, th, phi, p_r, p_th, E, L_z, spin).  False if degenerate.
__host__ __device__ inline bool escape_direction(const double y[6], double E_, double Lz_, double a_, D8 v[3]) {
    const D8 r = D8::var(y[1], 0), th = D8::var(y[2], 1), ph = D8::var(y[3], 2);
    const D8 pr = D8::var(y[4], 3), pth = D8::var(y[5], 4);
    const D8 E = D8::var(E_, 5), Lz = D8::var(Lz_, 6), a = D8::var(a_, 7);
    const D8 a2 = a * a;
    const D8 sn_raw = sin(th), cs = cos(th);
    D8 sn = sn_raw;
    if (fabs(sn.v) < 1e-9) sn = D8((sn.v < 0.0) ? -1e-9 : 1e-9);
    const D8 sn2 = sn * sn, cs2 = cs * cs;
    const D8 Sig = r * r + a2 * cs2;
    const D8 Del = r * r - 2.0 * r + a2;
    const D8 SD = Sig * Del;
    const D8 gtp = -2.0 * a * r / SD;
    const D8 gpp = (Del - a2 * sn2) / (SD * sn2);
    const D8 dr = (Del / Sig) * pr;
    const D8 dth = pth / Sig;
    const D8 dph = gtp * (-E) + gpp * Lz;
    const D8 R = sqrt(r * r + a * a);
    const D8 sp = sin(ph), cp = cos(ph);
    const D8 dR = (R.v > 0.0) ? r / R * dr : dr;
    v[0] = dR * sn_raw * cp + R * cs * dth * cp - R * sn_raw * sp * dph;
    v[1] = dR * sn_raw * sp + R * cs * dth * sp + R * sn_raw * cp * dph;
    v[2] = dr * cs - r * sn_raw * dth;
    const D8 vn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (!(vn.v > 0.0)) return false;
    v[0] = v[0] / vn;
    v[1] = v[1] / vn;
    v[2] = v[2] / vn;
    return true;
}

// CIE Y of the sky along unit direction d and its gradient with respect to d
// (scene.h:111-158, 202-223; the star field's Gaussian point-spread function
// and the diffuse background).
__host__ __device__ inline double sky_luminance(const SkyData& sky, const FrameParams& F, const double d[3],
                                                double gY[3]) {
    using D3 = Dual<3>;
    gY[0] = gY[1] = gY[2] = 0.0;
    double Y = 0.0;
    if (sky.n_stars > 0 && F.stars_enabled) {
        const double cutoff = F.cutoff, inv2s2 = F.inv2s2, norm = F.psf_norm;
        const double theta = acos(dclamp(d[2], -1.0, 1.0));
        const double phi = atan2(d[1], d[0]);
        const int it = (int)(theta / kPi * kLat);
        const double sn = dmaxr(sin(theta), 1e-6);
        const double dlon = 2.0 * kPi / kLon;
        int span_p = (int)ceil(cutoff / (sn * dlon));
        if (span_p < 1) span_p = 1;
        const int sp = (span_p * 2 + 1 >= kLon) ? kLon / 2 : span_p;
        const int pbase = (int)((phi + kPi) / (2.0 * kPi) * kLon);
        for (int a = -F.span_t; a <= F.span_t; ++a) {
            const int ti = it + a;
            if (ti < 0 || ti >= kLat) continue;
            for (int b = -sp; b <= sp; ++b) {
                int pi = pbase + b;
                pi = ((pi % kLon) + kLon) % kLon;
                const int bin = ti * kLon + pi;
                const int k0 = sky.bin_start[bin], k1 = sky.bin_start[bin + 1];
                for (int k = k0; k < k1; ++k) {
                    const double4 s = sky.star_pos[k];
                    const double dot_raw = d[0] * s.x + d[1] * s.y + d[2] * s.z;
                    const double dot = dclamp(dot_raw, -1.0, 1.0);
                    if (dot < F.cut_dot) continue;   // outside the cutoff, without the acos
                    double ang, dang2;   // angle and d(angle^2)/d(dot)
                    if (dot > 0.9999995) {
                        ang = sqrt(dmaxr(0.0, 2.0 * (1.0 - dot)));
                        dang2 = -2.0;
                    } else {
                        ang = acos(dot);
                        const double q = 1.0 - dot * dot;
                        dang2 = (q > 0.0) ? -2.0 * ang / sqrt(q) : 0.0;
                    }
                    if (ang > cutoff) continue;
                    const double w = norm * exp(-ang * ang * inv2s2) * s.w;
                    Y += w;
                    if (dot_raw > -1.0 && dot_raw < 1.0) {
                        const double dw = -w * inv2s2 * dang2;   // dw / d(dot)
                        gY[0] += dw * s.x;
                        gY[1] += dw * s.y;
                        gY[2] += dw * s.z;
                    }
                }
            }
        }
    }
    if (F.milky_way) {
        if (F.sky_mode == BH_SKY_UNIFORM) {
            Y += sky.diffuse_L;
        } else {
            const D3 d0 = D3::var(d[0], 0), d1 = D3::var(d[1], 1), d2 = D3::var(d[2], 2);
            const double ca = 0.8660254037844387, sa = 0.5;
            const D3 g1 = ca * d1 + sa * d2;
            D3 g2 = -sa * d1 + ca * d2;
            if (g2.v < -1.0) g2 = D3(-1.0);
            if (g2.v > 1.0) g2 = D3(1.0);
            const D3 band = exp(-fabs(g2) / 0.055);
            const D3 l = atan2(g1, d0);
            const D3 bulge = 0.55 + 0.45 * exp(-(l * l) / (2.0 * 0.45 * 0.45));
            const D3 lane = 0.65 + 0.35 * sin(l * 7.3 + g2 * 41.0) * sin(l * 3.1 - g2 * 17.0);
            if (lane.v > 0.0) {
                const D3 amp = sky.diffuse_L * band * bulge * lane;
                Y += amp.v;
                for (int i = 0; i < 3; ++i) gY[i] += amp.d[i];
            }
        }
    }
    return Y;
}

// ---- the ray ----------------------------------------------------------------------

struct RayResult {
    double Y;               // luminance of the ray
    double grad[4];         // w * dY/d(spin, inclination, Eddington ratio, r_out)
    int what;               // BH_HIT_*
    int steps;              // accepted steps of the forward pass
    long long replay;       // accepted steps replayed by the reverse pass
    int interval;           // final checkpoint interval
};

// Initial photon of frame-local ray `local_id` (render.cpp:440-451,
// scene.h:356-384, geodesic.h:215-231) and its derivatives with respect to
// the spin and the inclination.
// The image-plane position of sample k of pixel (px, py) (scene.h:356-384
// with the render path's jitter): su, sv in [-1, 1]; *x_pix, *y_pix in pixels.
__host__ __device__ inline void sample_position_at(const FrameParams& F, int px, int py, int k, double* su,
                                                   double* sv, double* x_pix, double* y_pix) {
    const int S = F.S;
    const int sy = k / S, sx = k - (k / S) * S;
    const uint64_t s0 = F.seed ^ ((uint64_t)py << 32) ^ ((uint64_t)px * 0x9E3779B97F4A7C15ull);
    const uint64_t g = 0x9E3779B97F4A7C15ull;
    const double u1 = u53(mix64(s0 + (uint64_t)(2 * k + 1) * g));
    const double u2 = u53(mix64(s0 + (uint64_t)(2 * k + 2) * g));
    const double jx = xm(xa((double)sx, u1), F.inv_S);
    const double jy = xm(xa((double)sy, u2), F.inv_S);
    *x_pix = xa((double)px, jx);
    *y_pix = xa((double)py, jy);
    *su = xs(xd(xm(2.0, *x_pix), (double)F.width), 1.0);
    *sv = xs(1.0, xd(xm(2.0, *y_pix), (double)F.height));
}

// The same for frame-local sample `local_id` (work order).
__host__ __device__ inline void sample_position(const FrameParams& F, long long local_id, double* su, double* sv,
                                                double* x_pix, double* y_pix) {
    const int S = F.S;
    const long long pixel = local_id / (S * S);
    const int k = (int)(local_id - pixel * (S * S));
    int px, py;
    pixel_xy(F.width, F.height, pixel, &px, &py);
    sample_position_at(F, px, py, k, su, sv, x_pix, y_pix);
}

// The initial photon at image-plane position (su, sv) and its derivatives
// with respect to the spin and the inclination.
__host__ __device__ inline void ray_start_at(const FrameParams& F, const AdjointFrame& X, double su, double sv,
                                             double y[6], double* E, double* Lz, double dy[2][6], double dE[2],
                                             double dLz[2]) {
    double x = xm(su, F.tanf);
    double yy = xd(xm(sv, F.tanf), F.aspect);
    const double z = 1.0;
    if (F.has_roll) {
        const double xr = xs(xm(F.cr, x), xm(F.sr, yy));
        const double yr = xa(xm(F.sr, x), xm(F.cr, yy));
        x = xr; yy = yr;
    }
    const double y2 = xs(xm(F.cp, yy), xm(F.sp, z));
    const double z2 = xa(xm(F.sp, yy), xm(F.cp, z));
    const double x2 = xa(xm(F.cy, x), xm(F.sy, z2));
    const double z3 = xa(xm(-F.sy, x), xm(F.cy, z2));
    const double v0 = -z3, v1 = -y2, v2 = x2;
    const double n = xsqrt(xa(xa(xm(v0, v0), xm(v1, v1)), xm(v2, v2)));
    const double d0 = xd(v0, n), d1 = xd(v1, n), d2 = xd(v2, n);
    // p^mu = -(e_0 - d^i e_i), lowered: the same expressions as the render path
    const double zero = 0.0;
    const double p0 = -xa(F.tet00, xm(-1.0, xa(xa(xm(d0, zero), xm(d1, zero)), xm(d2, zero))));
    const double p1 = -xa(zero, xm(-1.0, xa(xa(xm(d0, F.tet11), xm(d1, zero)), xm(d2, zero))));
    const double p2 = -xa(zero, xm(-1.0, xa(xa(xm(d0, zero), xm(d1, F.tet22)), xm(d2, zero))));
    const double p3 = -xa(F.tet03, xm(-1.0, xa(xa(xm(d0, zero), xm(d1, zero)), xm(d2, F.tet33))));
    const double pt = xa(xm(F.ml_tt, p0), xm(F.ml_tp, p3));
    const double pph = xa(xm(F.ml_tp, p0), xm(F.ml_pp, p3));
    y[0] = 0.0;
    y[1] = F.cam_r;
    y[2] = F.cam_th;
    y[3] = F.cam_ph;
    y[4] = xm(F.ml_rr, p1);
    y[5] = xm(F.ml_thth, p2);
    *E = -pt;
    *Lz = pph;
    for (int q = 0; q < 2; ++q) {
        const double p0q = -X.d_tet[0][q];
        const double p1q = d0 * X.d_tet[2][q];
        const double p2q = d1 * X.d_tet[3][q];
        const double p3q = -X.d_tet[1][q] + d2 * X.d_tet[4][q];
        const double ptq = X.d_ml[0][q] * p0 + F.ml_tt * p0q + X.d_ml[1][q] * p3 + F.ml_tp * p3q;
        const double pphq = X.d_ml[1][q] * p0 + F.ml_tp * p0q + X.d_ml[4][q] * p3 + F.ml_pp * p3q;
        dy[q][0] = 0.0;
        dy[q][1] = 0.0;
        dy[q][2] = (q == kParIncl) ? 1.0 : 0.0;
        dy[q][3] = 0.0;
        dy[q][4] = X.d_ml[2][q] * p1 + F.ml_rr * p1q;
        dy[q][5] = X.d_ml[3][q] * p2 + F.ml_thth * p2q;
        dE[q] = -ptq;
        dLz[q] = pphq;
    }
}

// The initial photon of frame-local sample `local_id`.
__host__ __device__ inline void ray_start(const FrameParams& F, const AdjointFrame& X, long long local_id,
                                          double y[6], double* E, double* Lz, double dy[2][6], double dE[2],
                                          double dLz[2]) {
    double su, sv, xp, yp;
    sample_position(F, local_id, &su, &sv, &xp, &yp);
    ray_start_at(F, X, su, sv, y, E, Lz, dy, dE, dLz);
}

// Accepted steps of the replay buffer: the reverse pass recomputes a segment
// in pieces of at most this many steps.
constexpr int kReplay = 16;

// Checkpoint store of one ray: `slots` states of 8 doubles (y, h, beta ln err_prev)
// after every `interval` accepted steps; full slots drop every second state
// and double the interval.
struct Checkpoints {
    double* ck;
    int slots;
    int interval;
    int n;
    __host__ __device__ void push(const Integ& st) {
        double* p = ck + 8 * n;
        for (int i = 0; i < 6; ++i) p[i] = st.y[i];
        p[6] = st.h;
        p[7] = st.errp_mem;
        ++n;
    }
    __host__ __device__ void after_step(const Integ& st) {
        if (st.steps % interval != 0) return;
        if (n == slots) {
            for (int j = 0; j < slots / 2; ++j)
                for (int i = 0; i < 8; ++i) ck[8 * j + i] = ck[8 * (2 * j) + i];
            n = slots / 2;
            interval *= 2;
        }
        if (st.steps % interval == 0) push(st);
    }
};

// The first two equatorial crossings of a ray: their radii and the accepted
// steps they lie in (0: none); `count` counts all of them.
struct Crossings {
    double r[2];
    int step[2];
    int n;
    int count;
};

// Integrates from `s` with the render path's events (render.cpp:158-257)
// until the ray ends, returning its class, or until its equatorial crossing
// number `stop_crossing` (counted from `s`; 0: none), returning -1 after that
// crossing's step with its radius in *r_hit and without looking at whether
// it hits the disc.  The crossing radius of a disc hit goes to *r_hit.
// Checkpoints (cp) and the first two equatorial crossings (xr) are recorded
// when given.
__host__ __device__ inline int forward_run(const FrameParams& F, const RayC& c, Integ& s, Checkpoints* cp,
                                           Crossings* xr, int stop_crossing, double* r_hit) {
    if (F.max_steps <= 0) return BH_HIT_EXHAUSTED;
    StepRec rec;
    int crossings = 0;
    for (;;) {
        if (!advance(F, c, s, &rec)) return BH_HIT_HORIZON;   // no acceptable step (render.cpp:133-136)
        const double rn = rec.yn[1];
        if (rn <= F.r_stop) return BH_HIT_HORIZON;
        if (F.disc_enabled && rec.c0 * rec.c7 < 0.0) {
            const DenseC cth = dense_coef(rec.h, rec.y[2], rec.yn[2], rec.kth[0], rec.kth[2], rec.kth[3],
                                          rec.kth[4], rec.kth[5], rec.kth[6]);
            const double s_end = dense_crossing(cth, crossing_target(cth.r1, cth.r1 + cth.r2));
            const DenseC crr = dense_coef(rec.h, rec.y[1], rec.yn[1], rec.kr[0], rec.kr[2], rec.kr[3],
                                          rec.kr[4], rec.kr[5], rec.kr[6]);
            const double rc = dense_eval(crr, s_end);
            if (xr) {
                if (xr->n < 2) {
                    xr->r[xr->n] = rc;
                    xr->step[xr->n++] = s.steps;
                }
                ++xr->count;
            }
            if (++crossings == stop_crossing) {
                *r_hit = rc;
                return -1;
            }
            if (rc >= F.r_in && rc <= F.r_out) {
                *r_hit = rc;
                return BH_HIT_DISC;
            }
        }
        if (rn > F.r_escape) return BH_HIT_SKY;
        if (s.steps >= F.max_steps) return BH_HIT_EXHAUSTED;
        if (cp) cp->after_step(s);
    }
}

// The reverse pass: carries the adjoint yb of the state after accepted step N
// (and, when rstar_b != 0, the weight of the disc-crossing radius of step N)
// back to the initial photon, segment by segment from the checkpoints, with
// the E, L_z and spin adjoints accumulated.  Returns the steps replayed.
__host__ __device__ inline long long reverse_sweep(const FrameParams& F, const RayC& c, const Checkpoints& cp,
                                                   int N, double rstar_b, double yb[6], double* Eb, double* Lzb,
                                                   double* ab) {
    long long replay = 0;
    const int interval = cp.interval;
    double ys_buf[kReplay][6], hs_buf[kReplay];
    for (int seg = (N - 1) / interval; seg >= 0; --seg) {
        const int first = seg * interval + 1;               // first step of the segment
        const int last = (first + interval - 1 < N) ? first + interval - 1 : N;
        const int len = last - first + 1;
        const int npiece = (len + kReplay - 1) / kReplay;
        for (int piece = npiece - 1; piece >= 0; --piece) {
            Integ r;
            const double* p = cp.ck + 8 * seg;
            for (int i = 0; i < 6; ++i) r.y[i] = p[i];
            r.h = p[6];
            r.errp_mem = p[7];
            r.have_k1 = 0;
            r.tries = 0;
            r.steps = 0;
            for (int j = 0; j < piece * kReplay; ++j) advance(F, c, r, nullptr);
            const int m = (len - piece * kReplay < kReplay) ? len - piece * kReplay : kReplay;
            for (int j = 0; j < m; ++j) {
                StepRec q;
                advance(F, c, r, &q);
                for (int i = 0; i < 6; ++i) ys_buf[j][i] = q.y[i];
                hs_buf[j] = q.h;
            }
            replay += piece * kReplay + m;
            for (int j = m - 1; j >= 0; --j) {
                const bool final_step = first + piece * kReplay + j == N;
                step_vjp(c, ys_buf[j], hs_buf[j], yb, Eb, Lzb, ab, final_step ? rstar_b : 0.0);
            }
        }
    }
    return replay;
}

__host__ __device__ inline RayC ray_consts(const FrameParams& F, double E, double Lz) {
    RayC c;
    c.a = F.a;
    c.a2 = F.a2;
    c.E = E;
    c.Lz = Lz;
    c.rp = F.r_plus;
    c.rm = F.r_minus;
    c.factored = F.factored_delta;
    return c;
}

__host__ __device__ inline void integ_start(const FrameParams& F, const double y0[6], Integ& s) {
    for (int i = 0; i < 6; ++i) s.y[i] = y0[i];
    s.h = F.h0;
    s.errp_mem = kBeta * kLnErrFloor;
    s.have_k1 = 0;
    s.tries = 0;
    s.steps = 0;
}

// The forward pass, the seed and the reverse pass of one ray.  `ck` holds
// `slots` checkpoints of 8 doubles.  With w == 0 (or forward_only) only the
// luminance is computed.  xr (may be null) receives the ray's first two
// equatorial crossings.
__host__ __device__ inline void adjoint_ray(const FrameParams& F, const AdjointFrame& X, const SkyData& sky,
                                            long long local_id, double w, double* ck, int slots,
                                            bool forward_only, RayResult* out, Crossings* xr = nullptr) {
    double y0[6], E, Lz, dy0[2][6], dE[2], dLz[2];
    ray_start(F, X, local_id, y0, &E, &Lz, dy0, dE, dLz);
    const RayC c = ray_consts(F, E, Lz);
    out->Y = 0.0;
    for (int q = 0; q < 4; ++q) out->grad[q] = 0.0;
    out->replay = 0;

    Integ s;
    integ_start(F, y0, s);
    Checkpoints cp{ck, slots, X.checkpoint_interval, 0};
    cp.push(s);
    double r_hit = 0.0;
    const int what = forward_run(F, c, s, &cp, xr, 0, &r_hit);
    out->what = what;
    out->steps = s.steps;
    out->interval = cp.interval;

    // ---- seed --------------------------------------------------------------------
    double yb[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double Eb = 0.0, Lzb = 0.0, ab = 0.0, rstar_b = 0.0;
    if (what == BH_HIT_DISC) {
        const D5 Y = disc_luminance(F, X, sky.table, r_hit, E, Lz);
        out->Y = Y.v;
        rstar_b = w * Y.d[kS5R];
        Eb = w * Y.d[kS5E];
        Lzb = w * Y.d[kS5L];
        ab = w * Y.d[kS5A];
        out->grad[2] = w * Y.d[kS5M];
    } else if (what == BH_HIT_SKY) {
        D8 v[3];
        if (escape_direction(s.y, E, Lz, F.a, v)) {
            const double d[3] = {v[0].v, v[1].v, v[2].v};
            double gY[3];
            out->Y = sky_luminance(sky, F, d, gY);
            double gs[8];
            for (int k = 0; k < 8; ++k)
                gs[k] = w * (gY[0] * v[0].d[k] + gY[1] * v[1].d[k] + gY[2] * v[2].d[k]);
            yb[1] = gs[0]; yb[2] = gs[1]; yb[3] = gs[2]; yb[4] = gs[3]; yb[5] = gs[4];
            Eb = gs[5];
            Lzb = gs[6];
            ab = gs[7];
        }
    }
    if (forward_only || w == 0.0 || (what != BH_HIT_DISC && what != BH_HIT_SKY)) return;
    if (rstar_b == 0.0 && Eb == 0.0 && Lzb == 0.0 && ab == 0.0 && yb[1] == 0.0 && yb[2] == 0.0 &&
        yb[3] == 0.0 && yb[4] == 0.0 && yb[5] == 0.0)
        return;

    // ---- reverse and the initial photon ------------------------------------------------
    out->replay = reverse_sweep(F, c, cp, s.steps, what == BH_HIT_DISC ? rstar_b : 0.0, yb, &Eb, &Lzb, &ab);
    for (int q = 0; q < 2; ++q) {
        double gq = Eb * dE[q] + Lzb * dLz[q];
        for (int i = 0; i < 6; ++i) gq += yb[i] * dy0[q][i];
        out->grad[q] += gq;
    }
    out->grad[kParSpin] += ab;
}

// ---- the edge term ---------------------------------------------------------------------
//
// A point-sampled frame changes with r_out only where a sample's equatorial
// crossing radius r_c passes the edge, so the discrete adjoint above has no
// r_out term.  The derivative of the frame averaged over each sample's cell
// of the pixel has one: with r_c linear in the image plane across the cell,
//   d(pixel)/d(r_out)  =  (Y_in - Y_out) L / |grad r_c|,
// L the length of the line r_c = r_out inside the cell (pixel units), Y_in
// the disc's luminance at r_out along the ray (the same E, L_z), Y_out what
// the ray sees when this crossing misses the disc (its continuation traced
// on).  The same edge moves with any parameter q that moves r_c, which adds
//   -(Y_in - Y_out) (d r_c/d q) L / |grad r_c|
// to d(pixel)/dq.  grad r_c and d r_c/dq come from a reverse sweep seeded
// with the crossing radius alone.

// d(initial p_r, p_th, E, L_z)/d(su, sv): the image-plane coordinates of
// scene.h:356-384 (su = 2 (x + jx)/W - 1, sv = 1 - 2 (y + jy)/H).
__host__ __device__ inline void ray_start_pixel_tangents(const FrameParams& F, double su0, double sv0,
                                                         double dpr[2], double dpth[2], double dE[2],
                                                         double dLz[2]) {
    using D2 = Dual<2>;
    const D2 su = D2::var(su0, 0), sv = D2::var(sv0, 1);
    D2 x = su * F.tanf;
    D2 yy = sv * F.tanf / F.aspect;
    if (F.has_roll) {
        const D2 xr = F.cr * x - F.sr * yy;
        const D2 yr = F.sr * x + F.cr * yy;
        x = xr;
        yy = yr;
    }
    const D2 y2 = F.cp * yy - F.sp;
    const D2 z2 = F.sp * yy + F.cp;
    const D2 x2 = F.cy * x + F.sy * z2;
    const D2 z3 = -F.sy * x + F.cy * z2;
    const D2 v0 = -z3, v1 = -y2, v2 = x2;
    const D2 n = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    const D2 d0 = v0 / n, d1 = v1 / n, d2 = v2 / n;
    for (int k = 0; k < 2; ++k) {
        const double p1 = d0.d[k] * F.tet11, p2 = d1.d[k] * F.tet22, p3 = d2.d[k] * F.tet33;
        dpr[k] = F.ml_rr * p1;
        dpth[k] = F.ml_thth * p2;
        dE[k] = -(F.ml_tp * p3);
        dLz[k] = F.ml_pp * p3;
    }
}

// Length of the line g . (x - c) = rhs inside the rectangle [x0, x1] x [y0, y1].
__host__ __device__ inline double line_in_cell(double gx, double gy, double cx, double cy, double rhs, double x0,
                                               double x1, double y0, double y1) {
    double px[4], py[4];
    int n = 0;
    if (gy != 0.0) {
        for (int e = 0; e < 2; ++e) {
            const double x = e ? x1 : x0;
            const double y = cy + (rhs - gx * (x - cx)) / gy;
            if (y >= y0 && y <= y1) { px[n] = x; py[n] = y; ++n; }
        }
    }
    if (gx != 0.0) {
        for (int e = 0; e < 2; ++e) {
            const double y = e ? y1 : y0;
            const double x = cx + (rhs - gy * (y - cy)) / gx;
            if (x >= x0 && x <= x1) { px[n] = x; py[n] = y; ++n; }
        }
    }
    double best = 0.0;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
            const double dx = px[i] - px[j], dy = py[i] - py[j];
            const double l = sqrt(dx * dx + dy * dy);
            if (l > best) best = l;
        }
    return best;
}

// Edges of the disc an equatorial crossing can be near.
enum { kEdgeOuter = 1, kEdgeInner = 2 };

// The edge term of equatorial crossing number `crossing` (1 or 2) of sample k
// of pixel (px, py), for the disc edges in `edges` (kEdgeOuter: r_out;
// kEdgeInner: r_in, the ISCO) and pixel weight w = dLoss/d(pixel).  With
// phi = r_out - r_c (outer) or r_c - r_in (inner), positive on the disc side,
//   d(pixel)/dq = (Y_disc - Y_beyond) (d phi/d q) L / |grad r_c|.
// out[0..2] receive the contributions to dLoss/d(r_out), d(spin),
// d(inclination); *cells the number of edges that cross the sample's cell.
// diag (may be null) receives r_c, |grad r_c| (per pixel), d r_c/d(spin,
// inclination), d r_c/d(su, sv), and per edge (outer, inner) L and
// Y_disc - Y_beyond.  Returns the accepted steps integrated (forward,
// continuation and replay).
__host__ __device__ BHA_NOINLINE long long edge_sample(const FrameParams& F, const AdjointFrame& X, const SkyData& sky,
                                                 int px, int py, int k, int crossing, int edges, double w,
                                                 double* ck, int slots, double out[3], int* cells,
                                                 double* diag = nullptr) {
    out[0] = out[1] = out[2] = 0.0;
    *cells = 0;
    double su, sv, xp, yp;
    sample_position_at(F, px, py, k, &su, &sv, &xp, &yp);
    double y0[6], E, Lz, dy0[2][6], dE[2], dLz[2];
    ray_start_at(F, X, su, sv, y0, &E, &Lz, dy0, dE, dLz);
    const RayC c = ray_consts(F, E, Lz);
    Integ s;
    integ_start(F, y0, s);
    Checkpoints cp{ck, slots, X.checkpoint_interval, 0};
    cp.push(s);
    double rc = 0.0;
    if (forward_run(F, c, s, &cp, nullptr, crossing, &rc) != -1) return s.steps;
    const int step = s.steps;

    // What the ray meets when this crossing misses the disc: its
    // continuation traced on from there.
    Integ t = s;
    double r_hit = 0.0;
    const int what = forward_run(F, c, t, nullptr, nullptr, 0, &r_hit);
    long long work = t.steps;
    double Y_beyond = 0.0;
    if (what == BH_HIT_DISC) {
        Y_beyond = disc_luminance(F, X, sky.table, r_hit, E, Lz).v;
    } else if (what == BH_HIT_SKY) {
        D8 v[3];
        if (escape_direction(t.y, E, Lz, F.a, v)) {
            const double d[3] = {v[0].v, v[1].v, v[2].v};
            double gY[3];
            Y_beyond = sky_luminance(sky, F, d, gY);
        }
    }
    // the disc's side of each edge: its luminance at r_out along this ray; the
    // Novikov-Thorne flux vanishes at r_in
    const double dY[2] = {(edges & kEdgeOuter) ? disc_luminance(F, X, sky.table, F.r_out, E, Lz).v - Y_beyond : 0.0,
                          (edges & kEdgeInner) ? -Y_beyond : 0.0};
    if (dY[0] == 0.0 && dY[1] == 0.0 && !diag) return work;

    // d r_c / d(initial state, E, L_z, spin) by a reverse sweep seeded with r_c
    double yb[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double Eb = 0.0, Lzb = 0.0, ab = 0.0;
    work += reverse_sweep(F, c, cp, step, 1.0, yb, &Eb, &Lzb, &ab);

    double dpr[2], dpth[2], dEp[2], dLzp[2];
    ray_start_pixel_tangents(F, su, sv, dpr, dpth, dEp, dLzp);
    double drc[2];
    for (int j = 0; j < 2; ++j) drc[j] = yb[4] * dpr[j] + yb[5] * dpth[j] + Eb * dEp[j] + Lzb * dLzp[j];
    // grad r_c in pixel units: su = 2 x / W - 1, sv = 1 - 2 y / H
    const double gx = drc[0] * (2.0 / F.width), gy = drc[1] * (-2.0 / F.height);
    const double gn = sqrt(gx * gx + gy * gy);
    double drq[2];
    for (int q = 0; q < 2; ++q) {
        drq[q] = Eb * dE[q] + Lzb * dLz[q];
        for (int i = 0; i < 6; ++i) drq[q] += yb[i] * dy0[q][i];
    }
    drq[kParSpin] += ab;
    // the sample's cell in pixel units
    const int S = F.S;
    const int sy = k / S, sx = k - (k / S) * S;
    const double x0 = px + sx * F.inv_S, x1 = px + (sx + 1) * F.inv_S;
    const double y0c = py + sy * F.inv_S, y1 = py + (sy + 1) * F.inv_S;
    double L[2] = {0.0, 0.0};
    for (int e = 0; e < 2; ++e) {
        if (!(edges & (e == 0 ? kEdgeOuter : kEdgeInner)) || !(gn > 0.0)) continue;
        const double r_edge = (e == 0) ? F.r_out : F.r_in;
        L[e] = line_in_cell(gx, gy, xp, yp, r_edge - rc, x0, x1, y0c, y1);
        if (!(L[e] > 0.0) || dY[e] == 0.0) continue;
        ++*cells;
        const double swept = w * dY[e] * L[e] / gn;
        if (e == 0) {
            out[0] += swept;
            out[1] -= swept * drq[kParSpin];
            out[2] -= swept * drq[kParIncl];
        } else {
            out[1] += swept * (drq[kParSpin] - 2.0 * F.x0 * X.d_x0);
            out[2] += swept * drq[kParIncl];
        }
    }
    if (diag) {
        diag[0] = rc;
        diag[1] = gn;
        diag[2] = drq[0];
        diag[3] = drq[1];
        diag[4] = drc[0];
        diag[5] = drc[1];
        diag[6] = L[0];
        diag[7] = dY[0];
        diag[8] = L[1];
        diag[9] = dY[1];
    }
    return work;
}

// Whether the crossing at radius rc (sample grid neighbours' same crossing
// differing by at most dmax; 0 when none has one) is examined for the disc's
// edges: within twice that spread of an edge, or within a tenth of the edge
// radius when no neighbour has the crossing.  Returns kEdge* bits.
__host__ __device__ inline int edge_mask(const FrameParams& F, double rc, double dmax) {
    int m = 0;
    auto near = [&](double re) { return dmax > 0.0 ? fabs(rc - re) <= 2.0 * dmax : fabs(rc - re) <= 0.1 * re; };
    if (rc >= F.r_in && near(F.r_out)) m |= kEdgeOuter;
    if (rc <= F.r_out && near(F.r_in)) m |= kEdgeInner;
    return m;
}

}  // namespace adj
}  // namespace bhg
