/*
 * bh_oracle.c - CPU oracle of the per-pixel geodesic render path (FP64).
 *
 * TEST INFRASTRUCTURE ONLY (see bh_oracle.h).  A plain-C restatement of the
 * reference renderer's algorithm.  Every expression keeps the reference's
 * operand order, so that with the same compiler flags (-O3, no FMA
 * contraction, glibc libm) it reproduces the reference bit for bit; the
 * tests compare it against oracle/_ref/libbh_ref.so, which is compiled from
 * the reference sources.  Citations are file:line in the reference project.
 *
 * Two settings exist only here and in the GPU library, not in the reference:
 * sky_mode BH_SKY_UNIFORM (an isotropic m <= 6.5 catalogue with a uniform
 * 21.5 mag/arcsec^2 background) and stop_mode BH_STOP_RELATIVE
 * (r_stop = r_+ (1 + stop_epsilon)).
 */
#include "bh_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846

/* ---- constants.h:20-60 -------------------------------------------------- */
#define PH_G        6.67430e-11
#define PH_C        2.99792458e8
#define PH_H        6.62607015e-34
#define PH_KB       1.380649e-23
#define PH_SIGMA_SB 5.670374419e-8
#define PH_SIGMA_T  6.6524587321e-29
#define PH_M_P      1.67262192369e-27
#define PH_M_SUN    1.98847e30
#define PH_R_SUN    6.957e8

static double dmax(double a, double b) { return (a < b) ? b : a; }   /* std::max */
static double dmin(double a, double b) { return (b < a) ? b : a; }   /* std::min */
static double dclamp(double v, double lo, double hi) {               /* std::clamp */
    return (v < lo) ? lo : (hi < v) ? hi : v;
}
static int iclamp(int v, int lo, int hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

/* ======================================================================== */
/* Kerr geometry                                                            */
/* ======================================================================== */

typedef struct { double r, th, sn, cs, sn2, cs2, Sigma, Delta, A, a, a2; } geom_t;
typedef struct { double tt, tp, rr, thth, pp; } metric_t;

/* kerr.h:44-59 */
static geom_t geom_at(double a, double r, double th) {
    geom_t g;
    g.a = a;
    g.a2 = a * a;
    g.r = r;
    g.th = th;
    g.sn = sin(th);
    if (fabs(g.sn) < 1e-9) g.sn = (g.sn < 0.0 ? -1e-9 : 1e-9);
    g.cs = cos(th);
    g.sn2 = g.sn * g.sn;
    g.cs2 = g.cs * g.cs;
    g.Sigma = r * r + g.a2 * g.cs2;
    g.Delta = r * r - 2.0 * r + g.a2;
    g.A = (r * r + g.a2) * (r * r + g.a2) - g.a2 * g.Delta * g.sn2;
    return g;
}

/* kerr.h:69-77 */
static metric_t metric_lower(const geom_t* g) {
    metric_t m;
    m.tt = -(1.0 - 2.0 * g->r / g->Sigma);
    m.tp = -2.0 * g->a * g->r * g->sn2 / g->Sigma;
    m.rr = g->Sigma / g->Delta;
    m.thth = g->Sigma;
    m.pp = g->A * g->sn2 / g->Sigma;
    return m;
}

/* kerr.h:107-116 */
static metric_t metric_upper(const geom_t* g) {
    metric_t m;
    const double SD = g->Sigma * g->Delta;
    m.tt = -g->A / SD;
    m.tp = -2.0 * g->a * g->r / SD;
    m.rr = g->Delta / g->Sigma;
    m.thth = 1.0 / g->Sigma;
    m.pp = (g->Delta - g->a2 * g->sn2) / (SD * g->sn2);
    return m;
}

typedef struct { metric_t g, dr, dth; } metric_deriv_t;

/* kerr.h:129-176: quotient-rule derivatives of g^{mu nu} in r and theta. */
static metric_deriv_t metric_upper_deriv(const geom_t* gm) {
    metric_deriv_t o;
    o.g = metric_upper(gm);
    const double r = gm->r, a2 = gm->a2, a = gm->a;
    const double sn = gm->sn, cs = gm->cs, sn2 = gm->sn2;
    const double S = gm->Sigma, D = gm->Delta, A = gm->A;
    const double S_r = 2.0 * r, S_th = -2.0 * a2 * sn * cs;
    const double D_r = 2.0 * r - 2.0, D_th = 0.0;
    const double A_r = 4.0 * r * (r * r + a2) - a2 * D_r * sn2;
    const double A_th = -2.0 * a2 * D * sn * cs;
    const double Q = S * D;
    const double Q_r = S_r * D + S * D_r;
    const double Q_th = S_th * D + S * D_th;
    const double Q2 = Q * Q;
    o.dr.tt = -(A_r * Q - A * Q_r) / Q2;
    o.dth.tt = -(A_th * Q - A * Q_th) / Q2;
    const double N = -2.0 * a * r, N_r = -2.0 * a, N_th = 0.0;
    o.dr.tp = (N_r * Q - N * Q_r) / Q2;
    o.dth.tp = (N_th * Q - N * Q_th) / Q2;
    o.dr.rr = (D_r * S - D * S_r) / (S * S);
    o.dth.rr = (D_th * S - D * S_th) / (S * S);
    o.dr.thth = -S_r / (S * S);
    o.dth.thth = -S_th / (S * S);
    const double P = D - a2 * sn2;
    const double P_r = D_r;
    const double P_th = -2.0 * a2 * sn * cs;
    const double R = Q * sn2;
    const double R_r = Q_r * sn2;
    const double R_th = Q_th * sn2 + Q * 2.0 * sn * cs;
    o.dr.pp = (P_r * R - P * R_r) / (R * R);
    o.dth.pp = (P_th * R - P * R_th) / (R * R);
    return o;
}

/* kerr.h:187-194 */
static double horizon_outer(double a) { const double d = 1.0 - a * a; return 1.0 + sqrt(dmax(0.0, d)); }
static double horizon_inner(double a) { const double d = 1.0 - a * a; return 1.0 - sqrt(dmax(0.0, d)); }

/* kerr.h:217-220 */
static double photon_circular_orbit(double a, int sigma) {
    const double x = dclamp(-(double)sigma * a, -1.0, 1.0);
    return 2.0 * (1.0 + cos((2.0 / 3.0) * acos(x)));
}

/* kerr.h:223-229 (Bardeen, Press & Teukolsky 1972) */
static double isco_radius(double a, int sigma) {
    const double a2 = a * a;
    const double Z1 = 1.0 + cbrt(1.0 - a2) * (cbrt(1.0 + a) + cbrt(1.0 - a));
    const double Z2 = sqrt(3.0 * a2 + Z1 * Z1);
    const double s = sqrt(dmax(0.0, (3.0 - Z1) * (3.0 + Z1 + 2.0 * Z2)));
    return 3.0 + Z2 - (double)sigma * s;
}

/* kerr.h:232-245 */
static double circular_energy(double a, double r, int sigma) {
    const double sr = sqrt(r);
    const double num = r * r - 2.0 * r + sigma * a * sr;
    const double den = r * sqrt(r * r - 3.0 * r + 2.0 * sigma * a * sr);
    return num / den;
}
static double circular_angmom(double a, double r, int sigma) {
    const double sr = sqrt(r);
    const double num = sigma * sr * (r * r - 2.0 * sigma * a * sr + a * a);
    const double den = r * sqrt(r * r - 3.0 * r + 2.0 * sigma * a * sr);
    return num / den;
}

/* kerr.h:250-252 */
static double disc_efficiency(double a, int sigma) {
    return 1.0 - circular_energy(a, isco_radius(a, sigma), sigma);
}

/* kerr.h:260-266 */
static void keplerian_four_velocity(double a, double r, int sigma, double u[4]) {
    const double r32 = r * sqrt(r);
    const double Omega = sigma / (r32 + sigma * a);
    const double disc = r * r * r - 3.0 * r * r + 2.0 * sigma * a * r32;
    const double ut = (r32 + sigma * a) / sqrt(dmax(1e-300, disc));
    u[0] = ut; u[1] = 0.0; u[2] = 0.0; u[3] = Omega * ut;
}

/* kerr.h:270-293 */
typedef struct { double e[4][4]; } tetrad_t;
static tetrad_t zamo_tetrad(const geom_t* g) {
    tetrad_t T;
    memset(&T, 0, sizeof T);
    const double alpha = sqrt(g->Sigma * g->Delta / g->A);
    const double omega = 2.0 * g->a * g->r / g->A;
    T.e[0][0] = 1.0 / alpha;
    T.e[0][3] = omega / alpha;
    T.e[1][1] = sqrt(g->Delta / g->Sigma);
    T.e[2][2] = 1.0 / sqrt(g->Sigma);
    T.e[3][3] = sqrt(g->Sigma / g->A) / g->sn;
    return T;
}

/* kerr.h:301-321 */
static double hamiltonian(const metric_t* m, const double p[4]) {
    return m->tt * p[0] * p[0] + 2.0 * m->tp * p[0] * p[3] + m->rr * p[1] * p[1] +
           m->thth * p[2] * p[2] + m->pp * p[3] * p[3];
}
static double hamiltonian_scale(const metric_t* m, const double p[4]) {
    return fabs(m->tt * p[0] * p[0]) + fabs(2.0 * m->tp * p[0] * p[3]) +
           fabs(m->rr * p[1] * p[1]) + fabs(m->thth * p[2] * p[2]) +
           fabs(m->pp * p[3] * p[3]);
}

/* kerr.h:342-348 */
static double carter_constant(double a, double th, double p_th, double E, double Lz, double m2) {
    double sn = sin(th);
    if (fabs(sn) < 1e-9) sn = 1e-9;
    const double cs2 = cos(th) * cos(th);
    return p_th * p_th + cs2 * (a * a * (m2 - E * E) + Lz * Lz / (sn * sn));
}

/* ======================================================================== */
/* Geodesics                                                                */
/* ======================================================================== */

enum { YT = 0, YR = 1, YTH = 2, YPH = 3, YPT = 4, YPR = 5, YPTH = 6, YPPH = 7 };

/* geodesic.h:50-71: Hamilton's equations for H = 1/2 g^{mu nu} p_mu p_nu. */
static void geodesic_rhs(double a, const double* y, double* d) {
    const geom_t g = geom_at(a, y[YR], y[YTH]);
    const metric_deriv_t m = metric_upper_deriv(&g);
    const double pt = y[YPT], pr = y[YPR], pth = y[YPTH], pph = y[YPPH];
    d[YT] = m.g.tt * pt + m.g.tp * pph;
    d[YR] = m.g.rr * pr;
    d[YTH] = m.g.thth * pth;
    d[YPH] = m.g.tp * pt + m.g.pp * pph;
    d[YPT] = 0.0;
    d[YPPH] = 0.0;
    d[YPR] = -0.5 * (m.dr.tt * pt * pt + 2.0 * m.dr.tp * pt * pph + m.dr.rr * pr * pr +
                     m.dr.thth * pth * pth + m.dr.pp * pph * pph);
    d[YPTH] = -0.5 * (m.dth.tt * pt * pt + 2.0 * m.dth.tp * pt * pph + m.dth.rr * pr * pr +
                      m.dth.thth * pth * pth + m.dth.pp * pph * pph);
}

/* geodesic.h:77-106: Dormand-Prince 5(4) tableau (Hairer, Norsett & Wanner II.4). */
static const double c_a21 = 1.0 / 5.0;
static const double c_a31 = 3.0 / 40.0, c_a32 = 9.0 / 40.0;
static const double c_a41 = 44.0 / 45.0, c_a42 = -56.0 / 15.0, c_a43 = 32.0 / 9.0;
static const double c_a51 = 19372.0 / 6561.0, c_a52 = -25360.0 / 2187.0,
                    c_a53 = 64448.0 / 6561.0, c_a54 = -212.0 / 729.0;
static const double c_a61 = 9017.0 / 3168.0, c_a62 = -355.0 / 33.0, c_a63 = 46732.0 / 5247.0,
                    c_a64 = 49.0 / 176.0, c_a65 = -5103.0 / 18656.0;
static const double c_b1 = 35.0 / 384.0, c_b3 = 500.0 / 1113.0, c_b4 = 125.0 / 192.0,
                    c_b5 = -2187.0 / 6784.0, c_b6 = 11.0 / 84.0;
#define C_E1 (35.0 / 384.0 - 5179.0 / 57600.0)
#define C_E3 (500.0 / 1113.0 - 7571.0 / 16695.0)
#define C_E4 (125.0 / 192.0 - 393.0 / 640.0)
#define C_E5 (-2187.0 / 6784.0 - (-92097.0 / 339200.0))
#define C_E6 (11.0 / 84.0 - 187.0 / 2100.0)
#define C_E7 (0.0 - 1.0 / 40.0)
static const double c_d1 = -12715105075.0 / 11282082432.0, c_d3 = 87487479700.0 / 32700410799.0,
                    c_d4 = -10690763975.0 / 1880347072.0, c_d5 = 701980252875.0 / 199316789632.0,
                    c_d6 = -1453857185.0 / 822651844.0, c_d7 = 69997945.0 / 29380423.0;

/* geodesic.h:109-121 */
typedef struct { double r1[8], r2[8], r3[8], r4[8], r5[8]; double h; } dense_t;
static void dense_eval(const dense_t* d, double s, double* y) {
    const double s1 = 1.0 - s;
    for (int i = 0; i < 8; ++i)
        y[i] = d->r1[i] + s * (d->r2[i] + s1 * (d->r3[i] + s * (d->r4[i] + s1 * d->r5[i])));
}

/* geodesic.h:123-204 */
typedef struct { double a, rtol, atol; double k1[8]; int have_k1; double err_prev; } stepper_t;

static void stepper_init(stepper_t* st, double a, double rtol, double atol) {
    st->a = a; st->rtol = rtol; st->atol = atol;
    st->have_k1 = 0; st->err_prev = 1e-4;
    memset(st->k1, 0, sizeof st->k1);
}

static int try_step(stepper_t* st, const double* y, double* h, double* y_out, dense_t* dense) {
    const double a = st->a;
    const double hh = *h;
    double tmp[8], k2[8], k3[8], k4[8], k5[8], k6[8], k7[8], ynew[8];
    if (!st->have_k1) { geodesic_rhs(a, y, st->k1); st->have_k1 = 1; }
    const double* k1 = st->k1;
    for (int i = 0; i < 8; ++i) tmp[i] = y[i] + hh * c_a21 * k1[i];
    geodesic_rhs(a, tmp, k2);
    for (int i = 0; i < 8; ++i) tmp[i] = y[i] + hh * (c_a31 * k1[i] + c_a32 * k2[i]);
    geodesic_rhs(a, tmp, k3);
    for (int i = 0; i < 8; ++i) tmp[i] = y[i] + hh * (c_a41 * k1[i] + c_a42 * k2[i] + c_a43 * k3[i]);
    geodesic_rhs(a, tmp, k4);
    for (int i = 0; i < 8; ++i)
        tmp[i] = y[i] + hh * (c_a51 * k1[i] + c_a52 * k2[i] + c_a53 * k3[i] + c_a54 * k4[i]);
    geodesic_rhs(a, tmp, k5);
    for (int i = 0; i < 8; ++i)
        tmp[i] = y[i] + hh * (c_a61 * k1[i] + c_a62 * k2[i] + c_a63 * k3[i] + c_a64 * k4[i] +
                              c_a65 * k5[i]);
    geodesic_rhs(a, tmp, k6);
    for (int i = 0; i < 8; ++i)
        ynew[i] = y[i] + hh * (c_b1 * k1[i] + c_b3 * k3[i] + c_b4 * k4[i] + c_b5 * k5[i] +
                               c_b6 * k6[i]);
    geodesic_rhs(a, ynew, k7);

    double err2 = 0.0;
    for (int i = 0; i < 8; ++i) {
        const double e = hh * (C_E1 * k1[i] + C_E3 * k3[i] + C_E4 * k4[i] + C_E5 * k5[i] +
                               C_E6 * k6[i] + C_E7 * k7[i]);
        const double sc = st->atol + st->rtol * dmax(fabs(y[i]), fabs(ynew[i]));
        const double q = e / sc;
        err2 += q * q;
    }
    double err = sqrt(err2 / 8.0);
    if (!isfinite(err)) err = 1e10;

    const double alpha = 0.7 / 5.0, beta = 0.4 / 5.0, safety = 0.9;
    double fac = safety * pow(dmax(err, 1e-16), -alpha) * pow(dmax(st->err_prev, 1e-4), beta);
    fac = dclamp(fac, 0.2, 5.0);

    if (err <= 1.0) {
        dense->h = hh;
        for (int i = 0; i < 8; ++i) {
            dense->r1[i] = y[i];
            dense->r2[i] = ynew[i] - y[i];
            dense->r3[i] = hh * k1[i] - dense->r2[i];
            dense->r4[i] = dense->r2[i] - hh * k7[i] - dense->r3[i];
            dense->r5[i] = hh * (c_d1 * k1[i] + c_d3 * k3[i] + c_d4 * k4[i] + c_d5 * k5[i] +
                                 c_d6 * k6[i] + c_d7 * k7[i]);
        }
        memcpy(y_out, ynew, sizeof ynew);
        memcpy(st->k1, k7, sizeof k7);
        st->err_prev = dmax(err, 1e-4);
        *h = hh * fac;
        return 1;
    }
    *h = hh * dmin(fac, 1.0);
    return 0;
}

/* geodesic.h:215-231: null momentum from a tetrad direction, lowered. */
static void make_photon(double a, double r, double th, double phi, const tetrad_t* tet,
                        const double dir[3], int past_directed, double* y) {
    const geom_t g = geom_at(a, r, th);
    const double s = past_directed ? -1.0 : +1.0;
    double pup[4];
    for (int mu = 0; mu < 4; ++mu)
        pup[mu] = tet->e[0][mu] + s * (dir[0] * tet->e[1][mu] + dir[1] * tet->e[2][mu] +
                                       dir[2] * tet->e[3][mu]);
    if (past_directed) for (int mu = 0; mu < 4; ++mu) pup[mu] = -pup[mu];
    const metric_t m = metric_lower(&g);
    y[0] = 0.0; y[1] = r; y[2] = th; y[3] = phi;
    y[4] = m.tt * pup[0] + m.tp * pup[3];
    y[5] = m.rr * pup[1];
    y[6] = m.thth * pup[2];
    y[7] = m.tp * pup[0] + m.pp * pup[3];
}

/* geodesic.h:234-251 */
typedef struct { double E, Lz, Q, norm, norm_rel; } invariants_t;
static invariants_t invariants(double a, const double* y) {
    invariants_t iv;
    iv.E = -y[YPT];
    iv.Lz = y[YPPH];
    iv.Q = carter_constant(a, y[YTH], y[YPTH], iv.E, iv.Lz, 0.0);
    const geom_t g = geom_at(a, y[YR], y[YTH]);
    const metric_t m = metric_upper(&g);
    const double p[4] = {y[YPT], y[YPR], y[YPTH], y[YPPH]};
    iv.norm = hamiltonian(&m, p);
    const double sc = hamiltonian_scale(&m, p);
    iv.norm_rel = (sc > 0.0) ? iv.norm / sc : iv.norm;
    return iv;
}

/* geodesic.h:256-262 */
static void bl_to_cartesian(double a, double r, double th, double phi, double out[3]) {
    const double rr = sqrt(r * r + a * a);
    const double sn = sin(th);
    out[0] = rr * sn * cos(phi);
    out[1] = rr * sn * sin(phi);
    out[2] = r * cos(th);
}

/* render.cpp:15-26 */
static void cartesian_velocity(double a, const double* y, const double* dy, double v[3]) {
    const double r = y[YR], th = y[YTH], ph = y[YPH];
    const double R = sqrt(r * r + a * a);
    const double sn = sin(th), cs = cos(th);
    const double sp = sin(ph), cp = cos(ph);
    const double dr = dy[YR], dth = dy[YTH], dph = dy[YPH];
    const double dR = (R > 0.0) ? r / R * dr : dr;
    v[0] = dR * sn * cp + R * cs * dth * cp - R * sn * sp * dph;
    v[1] = dR * sn * sp + R * cs * dth * sp + R * sn * cp * dph;
    v[2] = dr * cs - r * sn * dth;
}

/* render.cpp:31-34 */
static double redshift_factor(const double* y, const double u[4]) {
    const double ku = y[YPT] * u[0] + y[YPR] * u[1] + y[YPTH] * u[2] + y[YPPH] * u[3];
    return (ku > 1e-12) ? 1.0 / ku : 0.0;
}

/* ======================================================================== */
/* Novikov-Thorne disc                                                      */
/* ======================================================================== */

/* disc.h:46-64: Page & Thorne's closed form of W(r). */
static double pt_term(double xi, double xj, double xk, double a, double x, double x0) {
    if (fabs(xi) < 1e-13) return 0.0;
    return 3.0 * (xi - a) * (xi - a) / (xi * (xi - xj) * (xi - xk)) * log((x - xi) / (x0 - xi));
}
static double page_thorne_W(double a, double r, double r_isco) {
    const double x = sqrt(r);
    const double x0 = sqrt(r_isco);
    const double ac = acos(dclamp(a, -1.0, 1.0));
    const double x1 = 2.0 * cos(ac / 3.0 - ORC_PI / 3.0);
    const double x2 = 2.0 * cos(ac / 3.0 + ORC_PI / 3.0);
    const double x3 = -2.0 * cos(ac / 3.0);
    return x - x0 - 1.5 * a * log(x / x0) - pt_term(x1, x2, x3, a, x, x0) -
           pt_term(x2, x1, x3, a, x, x0) - pt_term(x3, x1, x2, a, x, x0);
}

typedef struct { double M, a; int sigma; double r_in, r_out, eta, mdot, r_g; } disc_t;

/* disc.h:73-82 */
static void disc_init(disc_t* d, double M_kg, double spin, double r_out, double eddington,
                      int prograde) {
    d->M = M_kg;
    d->a = dclamp(spin, -0.9999, 0.9999);
    d->sigma = prograde;
    d->r_in = isco_radius(dclamp(spin, -0.9999, 0.9999), prograde);
    d->r_out = dmax(r_out, isco_radius(dclamp(spin, -0.9999, 0.9999), prograde) * 1.02);
    d->eta = disc_efficiency(d->a, d->sigma);
    /* constants.h:52-60: L_Edd = 4 pi G M m_p c / sigma_T, Mdot_Edd = L_Edd / (eta c^2) */
    const double L_edd = 4.0 * ORC_PI * PH_G * M_kg * PH_M_P * PH_C / PH_SIGMA_T;
    d->mdot = eddington * (L_edd / (d->eta * PH_C * PH_C));
    d->r_g = PH_G * M_kg / (PH_C * PH_C);
}

static int disc_contains(const disc_t* d, double r) { return r >= d->r_in && r <= d->r_out; }

/* disc.h:134-143 */
static double disc_omega(const disc_t* d, double r) {
    const double r32 = r * sqrt(r);
    return d->sigma / (r32 + d->sigma * d->a);
}
static double disc_omega_prime(const disc_t* d, double r) {
    const double r32 = r * sqrt(r);
    const double dd = r32 + d->sigma * d->a;
    return -d->sigma * 1.5 * sqrt(r) / (dd * dd);
}

/* disc.h:110-121 */
static double disc_flux_dimensionless(const disc_t* d, double r) {
    if (r <= d->r_in) return 0.0;
    const double W = page_thorne_W(d->a, r, d->r_in);
    const double Om = disc_omega(d, r);
    const double dOm = disc_omega_prime(d, r);
    const double E = circular_energy(d->a, r, d->sigma);
    const double L = circular_angmom(d->a, r, d->sigma);
    const double den = (E - Om * L);
    if (!(den > 0.0)) return 0.0;
    const double F = (-dOm) / (4.0 * ORC_PI * r * den * den) * W;
    return (F > 0.0 && isfinite(F)) ? F : 0.0;
}

/* disc.h:94-104 */
static double disc_temperature(const disc_t* d, double r) {
    double F;
    if (r <= d->r_in || r > d->r_out) F = 0.0;
    else F = disc_flux_dimensionless(d, r) * d->mdot * PH_C * PH_C / (d->r_g * d->r_g);
    if (F <= 0.0) return 0.0;
    return pow(F / PH_SIGMA_SB, 0.25);
}

/* ======================================================================== */
/* Spectrum                                                                 */
/* ======================================================================== */

/* spectrum.cpp:13-22 */
static double planck_radiance(double lambda_m, double T) {
    if (T <= 0.0 || lambda_m <= 0.0) return 0.0;
    const double l = lambda_m;
    const double l5 = l * l * l * l * l;
    const double x = PH_H * PH_C / (l * PH_KB * T);
    if (x > 700.0) return 0.0;
    return (2.0 * PH_H * PH_C * PH_C) / (l5 * expm1(x));
}

/* spectrum.cpp:36-53: multi-lobe Gaussian fit of the CIE 1931 2-degree
   colour matching functions (Wyman, Sloan & Shirley 2013). */
static double lobe(double x, double mu, double s1, double s2) {
    const double t = (x - mu) * ((x < mu) ? 1.0 / s1 : 1.0 / s2);
    return exp(-0.5 * t * t);
}
static double cie_x(double nm) {
    return 1.056 * lobe(nm, 599.8, 37.9, 31.0) + 0.362 * lobe(nm, 442.0, 16.0, 26.7) -
           0.065 * lobe(nm, 501.1, 20.4, 26.2);
}
static double cie_y(double nm) {
    return 0.821 * lobe(nm, 568.8, 46.9, 40.5) + 0.286 * lobe(nm, 530.9, 16.3, 31.1);
}
static double cie_z(double nm) {
    return 1.217 * lobe(nm, 437.0, 11.8, 36.0) + 0.681 * lobe(nm, 459.0, 26.0, 13.8);
}

/* spectrum.cpp:55-73: 1 nm rectangle sum over 360..830 nm. */
static void blackbody_xyz_exact(double T, double out[3]) {
    out[0] = out[1] = out[2] = 0.0;
    if (T <= 0.0) return;
    const double lo = 360.0, hi = 830.0, dl = 1.0;
    for (double nm = lo; nm <= hi; nm += dl) {
        const double w = planck_radiance(nm * 1e-9, T) * dl * 1e-9;
        out[0] += w * cie_x(nm);
        out[1] += w * cie_y(nm);
        out[2] += w * cie_z(nm);
    }
}

/* spectrum.cpp:94-134: 4096-entry log-log table over 50 K .. 3e9 K. */
#define TABLE_N 4096
static const double kLogTMin = 1.6989700043360187;
static const double kLogTMax = 9.4771212547196626;
static double* g_lx = NULL;
static double* g_ly = NULL;
static double* g_lz = NULL;

static void table_build(void) {
    if (g_lx) return;
    double* lx = (double*)malloc(3 * TABLE_N * sizeof(double));
    for (int i = 0; i < TABLE_N; ++i) {
        const double f = (double)i / (TABLE_N - 1);
        const double T = pow(10.0, kLogTMin + f * (kLogTMax - kLogTMin));
        double v[3];
        blackbody_xyz_exact(T, v);
        lx[i] = log(dmax(v[0], 1e-300));
        lx[TABLE_N + i] = log(dmax(v[1], 1e-300));
        lx[2 * TABLE_N + i] = log(dmax(v[2], 1e-300));
    }
    g_ly = lx + TABLE_N;
    g_lz = lx + 2 * TABLE_N;
    g_lx = lx;
}

static void blackbody_xyz(double T, double o[3]) {
    table_build();
    const double lg = log10(dclamp(T, 50.0, 3.0e9));
    const double f = (lg - kLogTMin) / (kLogTMax - kLogTMin) * (TABLE_N - 1);
    const int i = iclamp((int)f, 0, TABLE_N - 2);
    const double u = f - i;
    o[0] = exp(g_lx[i] * (1.0 - u) + g_lx[i + 1] * u);
    o[1] = exp(g_ly[i] * (1.0 - u) + g_ly[i + 1] * u);
    o[2] = exp(g_lz[i] * (1.0 - u) + g_lz[i + 1] * u);
}

/* spectrum.cpp:158-162 (Ballesteros 2012) */
static double bv_to_temperature(double bv) {
    const double x = dclamp(bv, -0.4, 2.0);
    return 4600.0 * (1.0 / (0.92 * x + 1.7) + 1.0 / (0.92 * x + 0.62));
}

/* ======================================================================== */
/* Sky                                                                      */
/* ======================================================================== */

/* scene.h:27-44: splitmix64. */
typedef struct { uint64_t s; } rng_t;
static uint64_t rng_next(rng_t* r) {
    r->s += 0x9E3779B97F4A7C15ull;
    uint64_t z = r->s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double rng_uniform(rng_t* r) { return (double)(rng_next(r) >> 11) * 0x1.0p-53; }
static double rng_uniform_ab(rng_t* r, double a, double b) { return a + (b - a) * rng_uniform(r); }
static double rng_normal(rng_t* r) {
    const double u1 = dmax(rng_uniform(r), 1e-15);
    const double u2 = rng_uniform(r);
    return sqrt(-2.0 * log(u1)) * cos(2.0 * ORC_PI * u2);
}

typedef struct { double x, y, z, mag, T, irr; } star_t;

typedef struct {
    int n;
    star_t* stars;
    int* bin_start;   /* CSR over 360 x 720 bins, in catalogue order within a bin */
    int* bin_items;
    int n_lat, n_lon;
    int milky_way;
    int sky_mode;
} starfield_t;

/* scene.h:185-196: 30 degree tilt of the galactic plane. */
static void galactic_to_world(const double g[3], double w[3]) {
    const double ca = 0.8660254037844387, sa = 0.5;
    w[0] = g[0];
    w[1] = ca * g[1] - sa * g[2];
    w[2] = sa * g[1] + ca * g[2];
}
static void world_to_galactic(const double w[3], double g[3]) {
    const double ca = 0.8660254037844387, sa = 0.5;
    g[0] = w[0];
    g[1] = ca * w[1] + sa * w[2];
    g[2] = -sa * w[1] + ca * w[2];
}

/* scene.h:62-104 (BH_SKY_GALACTIC); BH_SKY_UNIFORM draws an isotropic
   direction, a magnitude by the same inverse CDF capped at m = 6.5 and a
   B-V index uniform in [-0.3, 1.8]. */
static void gen_star(rng_t* rng, int sky_mode, star_t* s) {
    double dir[3];
    if (sky_mode == BH_SKY_UNIFORM) {
        const double z = rng_uniform_ab(rng, -1.0, 1.0);
        const double ph = rng_uniform_ab(rng, 0.0, 2.0 * ORC_PI);
        const double rr = sqrt(dmax(0.0, 1.0 - z * z));
        dir[0] = rr * cos(ph); dir[1] = rr * sin(ph); dir[2] = z;
        s->x = dir[0]; s->y = dir[1]; s->z = dir[2];
        const double u = rng_uniform(rng);
        s->mag = -1.5 + log10(u * (pow(10.0, 0.45 * (6.5 - -1.5)) - 1.0) + 1.0) / 0.45;
        const double bv = rng_uniform_ab(rng, -0.3, 1.8);
        s->T = bv_to_temperature(bv);
    } else {
        if (rng_uniform(rng) < 0.45) {
            const double b = rng_normal(rng) * 0.12;
            const double l = rng_uniform_ab(rng, 0.0, 2.0 * ORC_PI);
            const double cb = cos(b);
            double gd[3] = {cb * cos(l), cb * sin(l), sin(b)};
            galactic_to_world(gd, dir);
        } else {
            const double z = rng_uniform_ab(rng, -1.0, 1.0);
            const double ph = rng_uniform_ab(rng, 0.0, 2.0 * ORC_PI);
            const double rr = sqrt(dmax(0.0, 1.0 - z * z));
            dir[0] = rr * cos(ph); dir[1] = rr * sin(ph); dir[2] = z;
        }
        s->x = dir[0]; s->y = dir[1]; s->z = dir[2];
        const double u = rng_uniform(rng);
        s->mag = -1.5 + log10(u * (pow(10.0, 0.45 * (12.0 - -1.5)) - 1.0) + 1.0) / 0.45;
        double bv = 0.55 + 0.42 * rng_normal(rng);
        if (rng_uniform(rng) < 0.10) bv = rng_uniform_ab(rng, 1.2, 1.9);
        s->T = bv_to_temperature(dclamp(bv, -0.35, 1.95));
    }
    const double F0 = 3.64e-9 * 0.089 * 1e6 * 1e-6;
    s->irr = F0 * pow(10.0, -0.4 * s->mag);
}

/* scene.h:173-181 */
static int star_bin(const starfield_t* sf, const star_t* s) {
    const double theta = acos(dclamp(s->z, -1.0, 1.0));
    const double phi = atan2(s->y, s->x);
    int ti = (int)(theta / ORC_PI * sf->n_lat);
    int pi = (int)((phi + ORC_PI) / (2.0 * ORC_PI) * sf->n_lon);
    ti = iclamp(ti, 0, sf->n_lat - 1);
    pi = ((pi % sf->n_lon) + sf->n_lon) % sf->n_lon;
    return ti * sf->n_lon + pi;
}

static void starfield_free(starfield_t* sf) {
    free(sf->stars); free(sf->bin_start); free(sf->bin_items);
    memset(sf, 0, sizeof *sf);
}

static int starfield_build(starfield_t* sf, int count, uint64_t seed, int sky_mode, int milky_way) {
    memset(sf, 0, sizeof *sf);
    sf->n = count < 0 ? 0 : count;
    sf->n_lat = 360; sf->n_lon = 720;
    sf->milky_way = milky_way;
    sf->sky_mode = sky_mode;
    const int nb = sf->n_lat * sf->n_lon;
    sf->stars = (star_t*)malloc((size_t)(sf->n > 0 ? sf->n : 1) * sizeof(star_t));
    sf->bin_start = (int*)calloc((size_t)nb + 1, sizeof(int));
    sf->bin_items = (int*)malloc((size_t)(sf->n > 0 ? sf->n : 1) * sizeof(int));
    if (!sf->stars || !sf->bin_start || !sf->bin_items) { starfield_free(sf); return -1; }
    rng_t rng = {seed};
    for (int i = 0; i < sf->n; ++i) gen_star(&rng, sky_mode, &sf->stars[i]);
    int* bins = (int*)malloc((size_t)(sf->n > 0 ? sf->n : 1) * sizeof(int));
    for (int i = 0; i < sf->n; ++i) { bins[i] = star_bin(sf, &sf->stars[i]); sf->bin_start[bins[i] + 1]++; }
    for (int b = 0; b < nb; ++b) sf->bin_start[b + 1] += sf->bin_start[b];
    int* fill = (int*)calloc((size_t)nb, sizeof(int));
    for (int i = 0; i < sf->n; ++i) sf->bin_items[sf->bin_start[bins[i]] + fill[bins[i]]++] = i;
    free(fill); free(bins);
    return 0;
}

/* Diffuse background.  BH_SKY_GALACTIC: scene.h:202-223 (band, bulge, dust
   lanes at 21.5 mag/arcsec^2, 4800 K colour).  BH_SKY_UNIFORM: the same
   surface brightness and colour everywhere. */
static void diffuse_radiance(int sky_mode, const double d[3], double out[3]) {
    const double F0 = 3.24e-10;
    const double arcsec2_per_sr = 4.2545170296152206e10;
    const double L = F0 * pow(10.0, -0.4 * 21.5) * arcsec2_per_sr;
    double amp;
    if (sky_mode == BH_SKY_UNIFORM) {
        amp = L;
    } else {
        double g[3];
        world_to_galactic(d, g);
        const double sin_b = dclamp(g[2], -1.0, 1.0);
        const double band = exp(-fabs(sin_b) / 0.055);
        const double l = atan2(g[1], g[0]);
        const double bulge = 0.55 + 0.45 * exp(-(l * l) / (2.0 * 0.45 * 0.45));
        const double lane = 0.65 + 0.35 * sin(l * 7.3 + sin_b * 41.0) * sin(l * 3.1 - sin_b * 17.0);
        amp = L * band * bulge * dmax(0.0, lane);
    }
    double c[3];
    blackbody_xyz(4800.0, c);
    const double inv = (c[1] > 0.0) ? 1.0 / c[1] : 0.0;
    out[0] = amp * c[0] * inv;
    out[1] = amp;
    out[2] = amp * c[2] * inv;
}

/* scene.h:111-158: Gaussian-PSF star lookup over the +-3 sigma bin window. */
static void sky_radiance(const starfield_t* sf, const double d[3], double sigma, double out[3]) {
    out[0] = out[1] = out[2] = 0.0;
    const double cutoff = 3.0 * sigma;
    const double inv2s2 = 1.0 / (2.0 * sigma * sigma);
    const double norm = 1.0 / (2.0 * ORC_PI * sigma * sigma);
    const int n_lat = sf->n_lat, n_lon = sf->n_lon;
    const double theta = acos(dclamp(d[2], -1.0, 1.0));
    const double phi = atan2(d[1], d[0]);
    const int it = (int)(theta / ORC_PI * n_lat);
    const double dlat = ORC_PI / n_lat;
    int span_t = (int)ceil(cutoff / dlat);
    if (span_t < 1) span_t = 1;
    const double sn = dmax(sin(theta), 1e-6);
    const double dlon = 2.0 * ORC_PI / n_lon;
    int span_p = (int)ceil(cutoff / (sn * dlon));
    if (span_p < 1) span_p = 1;
    for (int a = -span_t; a <= span_t; ++a) {
        const int ti = it + a;
        if (ti < 0 || ti >= n_lat) continue;
        const int sp = (span_p * 2 + 1 >= n_lon) ? n_lon / 2 : span_p;
        for (int b = -sp; b <= sp; ++b) {
            int pi = (int)((phi + ORC_PI) / (2.0 * ORC_PI) * n_lon) + b;
            pi = ((pi % n_lon) + n_lon) % n_lon;
            const int bin = ti * n_lon + pi;
            for (int k = sf->bin_start[bin]; k < sf->bin_start[bin + 1]; ++k) {
                const star_t* s = &sf->stars[sf->bin_items[k]];
                const double dot = dclamp(d[0] * s->x + d[1] * s->y + d[2] * s->z, -1.0, 1.0);
                const double ang = (dot > 0.9999995) ? sqrt(dmax(0.0, 2.0 * (1.0 - dot))) : acos(dot);
                if (ang > cutoff) continue;
                const double w = norm * exp(-ang * ang * inv2s2) * s->irr;
                double c[3];
                blackbody_xyz(s->T, c);
                const double inv = (c[1] > 0.0) ? 1.0 / c[1] : 0.0;
                out[0] += w * c[0] * inv;
                out[1] += w;
                out[2] += w * c[2] * inv;
            }
        }
    }
    if (sf->milky_way) {
        double mw[3];
        diffuse_radiance(sf->sky_mode, d, mw);
        out[0] += mw[0]; out[1] += mw[1]; out[2] += mw[2];
    }
}

/* scene.h:356-384 */
static void ray_direction(const bh_camera* cam, double sx, double sy, double aspect, double out[3]) {
    const double tanf = tan(0.5 * cam->fov);
    double x = sx * tanf;
    double y = sy * tanf / aspect;
    double z = 1.0;
    if (cam->roll != 0.0) {
        const double cr = cos(cam->roll), sr = sin(cam->roll);
        const double xr = cr * x - sr * y, yr = sr * x + cr * y;
        x = xr; y = yr;
    }
    const double cp = cos(cam->pitch), sp = sin(cam->pitch);
    const double y2 = cp * y - sp * z;
    const double z2 = sp * y + cp * z;
    const double cy = cos(cam->yaw), sy2 = sin(cam->yaw);
    const double x2 = cy * x + sy2 * z2;
    const double z3 = -sy2 * x + cy * z2;
    double v[3];
    v[0] = -z3;
    v[1] = -y2;
    v[2] = x2;
    const double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    out[0] = v[0] / n; out[1] = v[1] / n; out[2] = v[2] / n;
}

/* ======================================================================== */
/* Jets (jet.h:77-315) and their colour (spectrum.cpp:77-92)                */
/* ======================================================================== */

static double horizon_angular_velocity(double a) {   /* kerr.h:204-207 */
    const double rp = horizon_outer(a);
    return (rp > 0.0) ? a / (2.0 * rp) : 0.0;
}

/* jet.h:81-87 */
static double blandford_znajek_power(double a, double mdot_c2, double phi, double kappa) {
    const double OmH = horizon_angular_velocity(a);
    const double x = OmH * OmH;
    const double f = 1.0 + 1.38 * x - 9.2 * x * x;
    return (kappa / (4.0 * ORC_PI)) * phi * phi * x * dmax(0.0, f) * mdot_c2;
}

static double smoothstep01(double t) {   /* jet.h:91-94 */
    t = dclamp(t, 0.0, 1.0);
    return t * t * (3.0 - 2.0 * t);
}

static double jet_radius(const bh_jet* j, double z_abs) {
    return j->R_base * pow(dmax(z_abs, 1e-6) / j->z_base, j->k);
}
static double jet_gamma_at(const bh_jet* j, double z_abs) {
    const double t = dmin(1.0, pow(dmax(z_abs, 1e-6) / j->z_sat, j->k));
    return 1.0 + (j->gamma_max - 1.0) * t;
}
static double jet_speed_at(const bh_jet* j, double z_abs) {
    const double G = jet_gamma_at(j, z_abs);
    return sqrt(dmax(0.0, 1.0 - 1.0 / (G * G)));
}
static double jet_radial_profile(const bh_jet* j, double u) {
    const double s = (u - j->u_peak) / j->u_wid;
    const double t = u / j->spine_wid;
    return exp(-s * s) + j->spine * exp(-t * t);
}

/* jet.h:194-207 */
static double jet_shape(const bh_jet* j, double z, double rho) {
    const double az = fabs(z);
    if (az <= j->z_base || az >= j->z_top) return 0.0;
    const double R = jet_radius(j, az);
    const double f = jet_radial_profile(j, rho / R);
    if (f < 1e-9) return 0.0;
    const double g = pow(jet_gamma_at(j, az) / jet_gamma_at(j, j->z_base), -(2.0 + j->alpha)) *
                     pow(R / j->R_base, -(3.0 + j->alpha)) * pow(az / j->z_base, j->zeta);
    const double ramp = smoothstep01((az - j->z_base) / (0.5 * j->z_base)) *
                        smoothstep01((j->z_top - az) / (0.15 * j->z_top));
    return f * g * ramp;
}

/* jet.h:215-240: the plasma four-velocity, built in the ZAMO frame. */
static void jet_four_velocity(const bh_jet* j, const geom_t* g, double u[4]) {
    const tetrad_t T = zamo_tetrad(g);
    const double lapse = sqrt(g->Sigma * g->Delta / g->A);
    const double omega = 2.0 * g->a * g->r / g->A;
    const double sqrt_gpp = g->sn * sqrt(g->A / g->Sigma);
    const double z = g->r * g->cs;
    const double v = jet_speed_at(j, fabs(z));
    double v_phi = (j->Omega_F - omega) * sqrt_gpp / dmax(lapse, 1e-12);
    v_phi = dclamp(v_phi, -0.5 * v, 0.5 * v);
    const double v_pol = sqrt(dmax(0.0, v * v - v_phi * v_phi));
    const double sgn = (g->cs >= 0.0) ? 1.0 : -1.0;
    const double d_r = sgn * g->cs;
    const double d_th = -sgn * g->sn;
    const double G = 1.0 / sqrt(dmax(1e-12, 1.0 - v * v));
    for (int mu = 0; mu < 4; ++mu)
        u[mu] = G * (T.e[0][mu] + v_pol * (d_r * T.e[1][mu] + d_th * T.e[2][mu]) + v_phi * T.e[3][mu]);
}

/* jet.h:262-312 */
static void jet_configure(bh_jet* j, double spin, double mdot_c2, double r_g_m) {
    const double nu_0 = PH_C / 550e-9, nu_lo = 1.0e9, nu_hi = 1.0e17;
    j->a = spin;
    j->Omega_F = 0.5 * horizon_angular_velocity(spin);
    j->P_jet = blandford_znajek_power(spin, mdot_c2, j->phi_flux, 0.053);
    j->L_rad = j->eps_rad * j->P_jet;
    j->r_bound = sqrt(j->z_top * j->z_top + jet_radius(j, j->z_top) * jet_radius(j, j->z_top)) * 1.05;
    double C_f = 0.0;
    {
        const int N = 2000;
        const double du = 3.0 / N;
        for (int i = 0; i < N; ++i) {
            const double u = (i + 0.5) * du;
            C_f += jet_radial_profile(j, u) * u * du;
        }
    }
    double V = 0.0;
    {
        const int N = 4000;
        const double dz = (j->z_top - j->z_base) / N;
        for (int i = 0; i < N; ++i) {
            const double z = j->z_base + (i + 0.5) * dz;
            const double R = jet_radius(j, z);
            const double gz = pow(jet_gamma_at(j, z) / jet_gamma_at(j, j->z_base), -(2.0 + j->alpha)) *
                              pow(R / j->R_base, -(3.0 + j->alpha)) * pow(z / j->z_base, j->zeta);
            const double ramp = smoothstep01((z - j->z_base) / (0.5 * j->z_base)) *
                                smoothstep01((j->z_top - z) / (0.15 * j->z_top));
            V += gz * ramp * R * R * dz;
        }
        V *= 2.0 * (2.0 * ORC_PI) * C_f;
    }
    j->volume_rg3 = V;
    const double V_m3 = V * r_g_m * r_g_m * r_g_m;
    if (!(V_m3 > 0.0) || !(j->L_rad > 0.0)) { j->j_nu0 = 0.0; return; }
    const double A = j->L_rad / (4.0 * ORC_PI * V_m3);
    const double p = 1.0 - j->alpha;
    const double band = (fabs(p) > 1e-9) ? (pow(nu_hi, p) - pow(nu_lo, p)) / p : log(nu_hi / nu_lo);
    j->j_nu0 = A / (pow(nu_0, j->alpha) * band) * r_g_m;
}

/* spectrum.cpp:77-92: the colour of a unit power law I_nu ~ nu^-alpha. */
static void powerlaw_xyz(double alpha, double out[3]) {
    const double lambda_0 = 550e-9;
    out[0] = out[1] = out[2] = 0.0;
    const double lo = 360.0, hi = 830.0, dl = 1.0;
    for (double nm = lo; nm <= hi; nm += dl) {
        const double lam = nm * 1e-9;
        const double I_l = PH_C * pow(lam / lambda_0, alpha) / (lam * lam);
        const double w = I_l * dl * 1e-9;
        out[0] += w * cie_x(nm);
        out[1] += w * cie_y(nm);
        out[2] += w * cie_z(nm);
    }
}

/* render.cpp:55-62 */
static double segment_distance_to_origin(const double p0[3], const double p1[3]) {
    const double d[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    const double dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double t = 0.0;
    if (dd > 0.0) t = dclamp(-(p0[0] * d[0] + p0[1] * d[1] + p0[2] * d[2]) / dd, 0.0, 1.0);
    const double q[3] = {p0[0] + t * d[0], p0[1] + t * d[1], p0[2] + t * d[2]};
    return sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
}

/* render.cpp:44-50: four-point Gauss-Legendre on [0, 1]. */
static const double kGLx[4] = {0.06943184420297371, 0.33000947820757187, 0.66999052179242813,
                               0.93056815579702629};
static const double kGLw[4] = {0.17392742256872693, 0.32607257743127307, 0.32607257743127307,
                               0.17392742256872693};

/* render.cpp:107-122: the transfer integral over the part [0, s_end] of one step. */
static void sample_jet(const bh_jet* j, double a, const dense_t* dense, double h_step, double s_end,
                       double* acc) {
    if (s_end <= 0.0) return;
    double sum = 0.0;
    for (int q = 0; q < 4; ++q) {
        double ys[8];
        dense_eval(dense, kGLx[q] * s_end, ys);
        const double z = ys[YR] * cos(ys[YTH]);
        const double rho = sqrt(ys[YR] * ys[YR] + a * a) * sin(ys[YTH]);
        const double sh = jet_shape(j, z, rho);
        if (sh <= 0.0) continue;
        const geom_t gg = geom_at(a, ys[YR], ys[YTH]);
        double u[4];
        jet_four_velocity(j, &gg, u);
        const double gf = redshift_factor(ys, u);
        if (gf <= 0.0) continue;
        sum += kGLw[q] * sh * pow(gf, 2.0 + j->alpha);
    }
    *acc += j->j_nu0 * sum * h_step * s_end;
}

/* ======================================================================== */
/* Tracer and shading                                                       */
/* ======================================================================== */

typedef struct {
    const bh_render_config* cfg;
    disc_t disc;
    int have_disc;
    starfield_t stars;
    int have_stars;
    tetrad_t tet;
    double psf_sigma, aspect;
    int have_jet;
    double jet_colour[3];
} scene_t;

typedef struct { int what; double y[8]; double jet; int steps, attempts; double q_drift, norm_rel; } hit_t;

/* neutronstar.h:94-99 */
static void ns_surface_four_velocity(const bh_neutron_star* st, double theta, double u[4]) {
    const double sn = sin(theta);
    const double norm2 = 1.0 - 2.0 / st->R - st->Omega * st->Omega * st->R * st->R * sn * sn;
    const double ut = (norm2 > 1e-12) ? 1.0 / sqrt(norm2) : 1.0;
    u[0] = ut; u[1] = 0.0; u[2] = 0.0; u[3] = st->Omega * ut;
}

/* neutronstar.h:104-130 */
static double ns_temperature_at(const bh_neutron_star* st, double theta, double phi, double t_emit) {
    if (!st->caps) return st->T_eff;
    const double spin_phase = st->cap_phase0 + st->Omega * t_emit;
    const double m[3] = {sin(st->cap_tilt) * cos(spin_phase), sin(st->cap_tilt) * sin(spin_phase),
                         cos(st->cap_tilt)};
    const double n[3] = {sin(theta) * cos(phi), sin(theta) * sin(phi), cos(theta)};
    const double dot = n[0] * m[0] + n[1] * m[1] + n[2] * m[2];
    double ang = acos(dclamp(dot, -1.0, 1.0));
    if (st->two_caps) ang = dmin(ang, ORC_PI - ang);
    if (ang <= st->cap_radius) {
        const double edge = 0.9 * st->cap_radius;
        if (ang <= edge) return st->cap_T;
        const double u = (ang - edge) / (st->cap_radius - edge);
        const double w = 0.5 * (1.0 + cos(ORC_PI * u));
        return st->T_eff + (st->cap_T - st->T_eff) * w;
    }
    return st->T_eff;
}

/* render.cpp:69-260 */
static hit_t trace(const scene_t* sc, const double dir[3], bh_render_stats* local) {
    const bh_render_config* cfg = sc->cfg;
    const double a = cfg->spin;
    const double r_h = horizon_outer(a);
    const double r_stop = (cfg->stop_mode == BH_STOP_RELATIVE)
                              ? r_h * (1.0 + cfg->stop_epsilon)
                              : r_h * 1.0 + 1e-4 + (r_h - horizon_inner(a)) * 1e-3;
    hit_t hit;
    memset(&hit, 0, sizeof hit);
    hit.what = BH_HIT_EXHAUSTED;

    double y[8], ynew[8];
    make_photon(a, cfg->cam.r, cfg->cam.theta, cfg->cam.phi, &sc->tet, dir, 1, y);
    const invariants_t iv0 = invariants(a, y);
    const double Q0 = fabs(iv0.Q) + 1e-12;

    stepper_t st;
    stepper_init(&st, a, cfg->rtol, cfg->atol);
    double h = 0.02 * dmax(1.0, cfg->cam.r);
    memcpy(hit.y, y, sizeof y);

    double p0[3], p1[3];
    bl_to_cartesian(a, y[YR], y[YTH], y[YPH], p0);

    for (int step = 0; step < cfg->max_steps; ++step) {
        dense_t dense;
        const double hmax = 0.05 * dmax(1.0, y[YR] - r_h) + 0.01;
        if (h > hmax) h = hmax;
        int tries = 0;
        ++hit.attempts;
        while (!try_step(&st, y, &h, ynew, &dense)) {
            if (++tries > 40 || fabs(h) < 1e-14) { hit.what = BH_HIT_HORIZON; return hit; }
            ++hit.attempts;
        }
        ++local->steps;
        ++hit.steps;
        {
            const invariants_t iv = invariants(a, ynew);
            local->max_norm_error = dmax(local->max_norm_error, fabs(iv.norm_rel));
            local->max_carter_drift = dmax(local->max_carter_drift, fabs(iv.Q - iv0.Q) / Q0);
            hit.norm_rel = dmax(hit.norm_rel, fabs(iv.norm_rel));
            hit.q_drift = dmax(hit.q_drift, fabs(iv.Q - iv0.Q) / Q0);
        }
        bl_to_cartesian(a, ynew[YR], ynew[YTH], ynew[YPH], p1);
        /* render.cpp:150-152: most steps are nowhere near the jet */
        const int near_jet = sc->have_jet && segment_distance_to_origin(p0, p1) < cfg->jet.r_bound;

        /* render.cpp:158-169: neutron-star surface */
        if (cfg->star.enabled && ynew[YR] <= cfg->star.R) {
            double lo = 0.0, hi = 1.0, ys[8];
            for (int k = 0; k < 60; ++k) {
                const double mid = 0.5 * (lo + hi);
                dense_eval(&dense, mid, ys);
                if (ys[YR] <= cfg->star.R) hi = mid; else lo = mid;
            }
            const double s_end = 0.5 * (lo + hi);
            if (near_jet) sample_jet(&cfg->jet, a, &dense, dense.h, s_end, &hit.jet);
            hit.what = BH_HIT_STAR;
            dense_eval(&dense, s_end, hit.y);
            return hit;
        }
        /* render.cpp:172-177: horizon */
        if (ynew[YR] <= r_stop) {
            if (near_jet) sample_jet(&cfg->jet, a, &dense, dense.h, 1.0, &hit.jet);
            hit.what = BH_HIT_HORIZON;
            memcpy(hit.y, ynew, sizeof ynew);
            return hit;
        }
        /* render.cpp:180-199: equatorial crossing */
        if (sc->have_disc) {
            const double c0 = cos(y[YTH]);
            const double c1 = cos(ynew[YTH]);
            if (c0 * c1 < 0.0) {
                double lo = 0.0, hi = 1.0, ys[8];
                for (int k = 0; k < 60; ++k) {
                    const double mid = 0.5 * (lo + hi);
                    dense_eval(&dense, mid, ys);
                    const double cm = cos(ys[YTH]);
                    if (cm * c0 <= 0.0) hi = mid; else lo = mid;
                }
                const double s_end = 0.5 * (lo + hi);
                double yc[8];
                dense_eval(&dense, s_end, yc);
                if (disc_contains(&sc->disc, yc[YR])) {
                    if (near_jet) sample_jet(&cfg->jet, a, &dense, dense.h, s_end, &hit.jet);
                    hit.what = BH_HIT_DISC;
                    memcpy(hit.y, yc, sizeof yc);
                    return hit;
                }
            }
        }
        /* render.cpp:202-241: the Sun */
        if (cfg->sun_enabled) {
            const double* C = cfg->sun.centre;
            const double seg[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
            const double seg_len = sqrt(seg[0] * seg[0] + seg[1] * seg[1] + seg[2] * seg[2]);
            const double dc = sqrt((p0[0] - C[0]) * (p0[0] - C[0]) + (p0[1] - C[1]) * (p0[1] - C[1]) +
                                   (p0[2] - C[2]) * (p0[2] - C[2]));
            if (dc <= seg_len + cfg->sun.radius * 1.5) {
                double ys[8], q[3];
#define SUN_F(S, OUT)                                                                   \
    do {                                                                                \
        dense_eval(&dense, (S), ys);                                                    \
        bl_to_cartesian(a, ys[YR], ys[YTH], ys[YPH], q);                                \
        const double dx_ = q[0] - C[0], dy_ = q[1] - C[1], dz_ = q[2] - C[2];           \
        (OUT) = dx_ * dx_ + dy_ * dy_ + dz_ * dz_ - cfg->sun.radius * cfg->sun.radius;  \
    } while (0)
                double f0;
                SUN_F(0.0, f0);
                if (f0 <= 0.0) { hit.what = BH_HIT_SUN; memcpy(hit.y, y, sizeof y); return hit; }
                double prev_s = 0.0;
                for (int k = 1; k <= 12; ++k) {
                    const double s = (double)k / 12;
                    double fs;
                    SUN_F(s, fs);
                    if (fs <= 0.0) {
                        double lo = prev_s, hi2 = s;
                        for (int b = 0; b < 50; ++b) {
                            const double mid = 0.5 * (lo + hi2);
                            double fm;
                            SUN_F(mid, fm);
                            if (fm <= 0.0) hi2 = mid; else lo = mid;
                        }
                        const double s_end = 0.5 * (lo + hi2);
                        if (near_jet) sample_jet(&cfg->jet, a, &dense, dense.h, s_end, &hit.jet);
                        hit.what = BH_HIT_SUN;
                        dense_eval(&dense, s_end, hit.y);
                        return hit;
                    }
                    prev_s = s;
                }
#undef SUN_F
            }
        }
        /* render.cpp:244: nothing stopped the ray inside this step */
        if (near_jet) sample_jet(&cfg->jet, a, &dense, dense.h, 1.0, &hit.jet);
        /* render.cpp:247-251: escape */
        if (ynew[YR] > cfg->r_escape) {
            hit.what = BH_HIT_SKY;
            memcpy(hit.y, ynew, sizeof ynew);
            return hit;
        }
        memcpy(y, ynew, sizeof y);
        p0[0] = p1[0]; p0[1] = p1[1]; p0[2] = p1[2];
    }
    hit.what = BH_HIT_EXHAUSTED;
    memcpy(hit.y, y, sizeof y);
    return hit;
}

/* render.cpp:265-375.  Also reports g (disc hits) and the sky direction. */
static void shade_hit(const scene_t* sc, const hit_t* hit, bh_render_stats* local, double out[3],
                      double* g_out, double dir_out[3]) {
    const bh_render_config* cfg = sc->cfg;
    const double a = cfg->spin;
    out[0] = out[1] = out[2] = 0.0;
    *g_out = 0.0;
    dir_out[0] = dir_out[1] = dir_out[2] = 0.0;
    switch (hit->what) {
    case BH_HIT_HORIZON:
        ++local->captured;
        return;
    case BH_HIT_DISC: {
        ++local->disc_hits;
        const double r = hit->y[YR];
        double T_em = disc_temperature(&sc->disc, r);
        if (T_em <= 0.0) return;
        if (cfg->hotspot.enabled) {
            /* scene.h:325-334 */
            const bh_hotspot* hs = &cfg->hotspot;
            const double t_emit = cfg->observer_time + hit->y[YT];
            double f = 1.0;
            {
                const double phi_s = hs->phi0 + hs->omega * t_emit;
                const double dx = r * cos(hit->y[YPH]) - hs->r * cos(phi_s);
                const double dy = r * sin(hit->y[YPH]) - hs->r * sin(phi_s);
                const double d2 = dx * dx + dy * dy;
                f = 1.0 + hs->contrast * exp(-0.5 * d2 / (hs->sigma * hs->sigma));
            }
            T_em *= pow(f, 0.25);
        }
        double u[4];
        keplerian_four_velocity(sc->disc.a, r, sc->disc.sigma, u);
        const double g = redshift_factor(hit->y, u);
        if (g <= 0.0) return;
        *g_out = g;
        blackbody_xyz(g * T_em, out);
        return;
    }
    case BH_HIT_SUN: {
        ++local->sun_hits;
        const geom_t gm = geom_at(a, hit->y[YR], hit->y[YTH]);
        const metric_t ml = metric_lower(&gm);
        if (ml.tt >= 0.0) return;
        const double u[4] = {1.0 / sqrt(-ml.tt), 0.0, 0.0, 0.0};
        const double g = redshift_factor(hit->y, u);
        if (g <= 0.0) return;
        *g_out = g;
        double p[3], d[8], v[3];
        bl_to_cartesian(a, hit->y[YR], hit->y[YTH], hit->y[YPH], p);
        geodesic_rhs(a, hit->y, d);
        cartesian_velocity(a, hit->y, d, v);
        const double vn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (vn > 0.0) { v[0] /= vn; v[1] /= vn; v[2] /= vn; }
        /* scene.h:266-276: Eddington limb darkening */
        double limb = 1.0;
        {
            double n[3] = {p[0] - cfg->sun.centre[0], p[1] - cfg->sun.centre[1], p[2] - cfg->sun.centre[2]};
            const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            if (len > 0.0) {
                n[0] /= len; n[1] /= len; n[2] /= len;
                const double mu = dclamp(-(n[0] * v[0] + n[1] * v[1] + n[2] * v[2]), 0.0, 1.0);
                limb = (2.0 + 3.0 * mu) / 5.0;
            }
        }
        const double self_redshift = PH_G * PH_M_SUN / (PH_R_SUN * PH_C * PH_C);
        const double T_obs = g * cfg->sun.T_eff / (1.0 + self_redshift);
        blackbody_xyz(T_obs, out);
        out[0] *= limb; out[1] *= limb; out[2] *= limb;
        return;
    }
    case BH_HIT_STAR: {
        ++local->star_hits;
        const bh_neutron_star* st = &cfg->star;
        const double r = hit->y[YR], th = hit->y[YTH], ph = hit->y[YPH];
        double u[4];
        ns_surface_four_velocity(st, th, u);
        const double ku = hit->y[YPT] * u[0] + hit->y[YPPH] * u[3];
        if (!(ku > 1e-12)) return;
        const double g = 1.0 / ku;
        *g_out = g;
        const double t_emit = cfg->observer_time + hit->y[YT];
        const double T_local = ns_temperature_at(st, th, ph, t_emit);
        const double f = 1.0 - 2.0 / r;
        const double mu = (f > 0.0) ? dclamp(-hit->y[YPR] * sqrt(f) / ku, 0.0, 1.0) : 1.0;
        const double limb = (2.0 + 3.0 * mu) / 5.0;
        blackbody_xyz(g * T_local, out);
        out[0] *= limb; out[1] *= limb; out[2] *= limb;
        return;
    }
    case BH_HIT_SKY: {
        ++local->escaped;
        double d[8], v[3];
        geodesic_rhs(a, hit->y, d);
        cartesian_velocity(a, hit->y, d, v);
        const double vn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (vn <= 0.0) return;
        v[0] /= vn; v[1] /= vn; v[2] /= vn;
        dir_out[0] = v[0]; dir_out[1] = v[1]; dir_out[2] = v[2];
        if (!sc->have_stars) return;
        sky_radiance(&sc->stars, v, sc->psf_sigma, out);
        return;
    }
    default:
        ++local->exhausted;
        return;
    }
}

static int scene_init(scene_t* sc, const bh_render_config* cfg) {
    memset(sc, 0, sizeof *sc);
    if (!cfg || cfg->width <= 0 || cfg->height <= 0) return BH_ERR_INVALID_ARG;
    sc->cfg = cfg;
    if (cfg->jet_enabled) {
        sc->have_jet = 1;
        powerlaw_xyz(cfg->jet.alpha, sc->jet_colour);   /* render.cpp:417 */
    }
    if (cfg->disc_enabled) {
        disc_init(&sc->disc, cfg->M_kg, cfg->spin, cfg->disc_r_out, cfg->eddington, cfg->disc_sense);
        sc->have_disc = 1;
    }
    if (cfg->stars_enabled) {
        if (starfield_build(&sc->stars, cfg->star_count, cfg->seed, cfg->sky_mode, cfg->milky_way) != 0)
            return BH_ERR_OUT_OF_MEMORY;
        sc->have_stars = 1;
    }
    const geom_t gcam = geom_at(cfg->spin, cfg->cam.r, cfg->cam.theta);
    sc->tet = zamo_tetrad(&gcam);
    sc->aspect = (double)cfg->width / cfg->height;
    const double px_ang = cfg->cam.fov / cfg->width;
    sc->psf_sigma = 0.55 * px_ang;
    return BH_OK;
}

static void scene_free(scene_t* sc) {
    if (sc->have_stars) starfield_free(&sc->stars);
}

static void stats_add(bh_render_stats* s, const bh_render_stats* b) {
    s->rays += b->rays; s->steps += b->steps; s->captured += b->captured;
    s->disc_hits += b->disc_hits; s->sun_hits += b->sun_hits; s->star_hits += b->star_hits;
    s->jet_rays += b->jet_rays; s->escaped += b->escaped; s->exhausted += b->exhausted;
    s->total_flux += b->total_flux;
    s->max_norm_error = dmax(s->max_norm_error, b->max_norm_error);
    s->max_carter_drift = dmax(s->max_carter_drift, b->max_carter_drift);
}

/* render.cpp:433-463: the samples of pixel (xx, yy): per-sample results to
   rays[0 .. S^2) when rays is not NULL, the pixel's average to *pixel when
   that is not NULL, counters and flux into *local. */
static void trace_pixel(const scene_t* sc, int xx, int yy, bh_render_stats* local, bh_ray_result* rays,
                        bh_xyz* pixel) {
    const bh_render_config* cfg = sc->cfg;
    const int S = cfg->sqrt_spp > 1 ? cfg->sqrt_spp : 1;
    const double inv_S = 1.0 / S;
    rng_t rng = {cfg->seed ^ ((uint64_t)yy << 32) ^ ((uint64_t)xx * 0x9E3779B97F4A7C15ull)};
    double acc[3] = {0.0, 0.0, 0.0};
    size_t ridx = 0;
    for (int sy = 0; sy < S; ++sy) {
        for (int sx = 0; sx < S; ++sx) {
            const double jx = (sx + rng_uniform(&rng)) * inv_S;
            const double jy = (sy + rng_uniform(&rng)) * inv_S;
            const double u = (2.0 * (xx + jx) / cfg->width - 1.0);
            const double v = (1.0 - 2.0 * (yy + jy) / cfg->height);
            double dir[3];
            ray_direction(&cfg->cam, u, v, sc->aspect, dir);
            ++local->rays;
            const hit_t hit = trace(sc, dir, local);
            double c[3], g, sdir[3];
            shade_hit(sc, &hit, local, c, &g, sdir);
            if (hit.jet > 0.0) {   /* render.cpp:384-392 */
                ++local->jet_rays;
                c[0] += sc->jet_colour[0] * hit.jet;
                c[1] += sc->jet_colour[1] * hit.jet;
                c[2] += sc->jet_colour[2] * hit.jet;
            }
            acc[0] += c[0]; acc[1] += c[1]; acc[2] += c[2];
            if (rays) {
                bh_ray_result* o = &rays[ridx++];
                o->what = hit.what;
                o->steps = hit.steps;
                memcpy(o->y, hit.y, sizeof hit.y);
                o->g = g;
                o->dir[0] = sdir[0]; o->dir[1] = sdir[1]; o->dir[2] = sdir[2];
                o->xyz.x = c[0]; o->xyz.y = c[1]; o->xyz.z = c[2];
                o->attempts = hit.attempts;
                o->reserved = 0;
                o->max_norm = hit.norm_rel;
                o->max_q = hit.q_drift;
                o->jet = hit.jet;
            }
        }
    }
    const double wgt = 1.0 / (S * S);
    if (pixel) {
        pixel->x = acc[0] * wgt; pixel->y = acc[1] * wgt; pixel->z = acc[2] * wgt;
    }
    local->total_flux += acc[1] * wgt;
}

/* render.cpp:428-463: the pixel loop over a window, one result per sample. */
static int run_window(const bh_render_config* cfg, int x0, int y0, int w, int h,
                      bh_ray_result* rays, bh_xyz* pixels, bh_render_stats* stats) {
    scene_t sc;
    int rc = scene_init(&sc, cfg);
    if (rc != BH_OK) return rc;
    if (x0 < 0 || y0 < 0 || w < 0 || h < 0 || x0 + w > cfg->width || y0 + h > cfg->height) {
        scene_free(&sc);
        return BH_ERR_INVALID_ARG;
    }
    bh_render_stats local;
    memset(&local, 0, sizeof local);
    const int S = cfg->sqrt_spp > 1 ? cfg->sqrt_spp : 1;
    size_t ridx = 0;
    for (int yy = y0; yy < y0 + h; ++yy) {
        for (int xx = x0; xx < x0 + w; ++xx) {
            trace_pixel(&sc, xx, yy, &local, rays ? &rays[ridx] : NULL,
                        pixels ? &pixels[(size_t)(yy - y0) * w + (xx - x0)] : NULL);
            ridx += (size_t)S * S;
        }
    }
    if (stats) stats_add(stats, &local);
    scene_free(&sc);
    return BH_OK;
}

/* The pixel loop over a list of whole rows on `threads` workers, each taking
   the next row from a shared counter (render.cpp:420-477's pool, for
   per-sample results of large parts of a frame).  Samples of the k-th listed
   row go to out[(k * width + x) * S^2 + s]. */
typedef struct {
    const scene_t* sc;
    const int* rows;
    int nrows;
    int next;
    pthread_mutex_t lock;
    bh_ray_result* out;
    bh_render_stats stats;
} rows_job_t;

static void* rows_worker(void* arg) {
    rows_job_t* job = (rows_job_t*)arg;
    const bh_render_config* cfg = job->sc->cfg;
    const int S = cfg->sqrt_spp > 1 ? cfg->sqrt_spp : 1;
    bh_render_stats local;
    memset(&local, 0, sizeof local);
    for (;;) {
        pthread_mutex_lock(&job->lock);
        const int k = job->next++;
        pthread_mutex_unlock(&job->lock);
        if (k >= job->nrows) break;
        for (int xx = 0; xx < cfg->width; ++xx)
            trace_pixel(job->sc, xx, job->rows[k], &local,
                        &job->out[((size_t)k * cfg->width + xx) * S * S], NULL);
    }
    pthread_mutex_lock(&job->lock);
    stats_add(&job->stats, &local);
    pthread_mutex_unlock(&job->lock);
    return NULL;
}

int orc_trace_rows(const bh_render_config* cfg, const int* rows, int nrows, int threads, bh_ray_result* out,
                   bh_render_stats* stats) {
    if (!cfg || nrows < 0 || (nrows > 0 && (!rows || !out))) return BH_ERR_INVALID_ARG;
    for (int k = 0; k < nrows; ++k)
        if (rows[k] < 0 || rows[k] >= cfg->height) return BH_ERR_INVALID_ARG;
    scene_t sc;
    int rc = scene_init(&sc, cfg);
    if (rc != BH_OK) return rc;
    table_build();   /* the lazily built blackbody table, before any worker reads it */
    rows_job_t job;
    memset(&job, 0, sizeof job);
    job.sc = &sc;
    job.rows = rows;
    job.nrows = nrows;
    job.out = out;
    pthread_mutex_init(&job.lock, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tid[256];
    int started = 0;
    for (int t = 0; t < threads; ++t) {
        if (pthread_create(&tid[t], NULL, rows_worker, &job) != 0) break;
        ++started;
    }
    if (started == 0) rows_worker(&job);
    for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
    pthread_mutex_destroy(&job.lock);
    if (stats) stats_add(stats, &job.stats);
    scene_free(&sc);
    return BH_OK;
}

/* ======================================================================== */
/* Exported entry points                                                    */
/* ======================================================================== */

static geom_t geom_pub(double a, double r, double th) { return geom_at(a, r, th); }

static void metric_out(const metric_t* m, double* o) {
    o[0] = m->tt; o[1] = m->tp; o[2] = m->rr; o[3] = m->thth; o[4] = m->pp;
}

void orc_metric_upper(double a, double r, double th, double out5[5]) {
    const geom_t g = geom_pub(a, r, th);
    const metric_t m = metric_upper(&g);
    metric_out(&m, out5);
}
void orc_metric_lower(double a, double r, double th, double out5[5]) {
    const geom_t g = geom_pub(a, r, th);
    const metric_t m = metric_lower(&g);
    metric_out(&m, out5);
}
void orc_metric_upper_deriv(double a, double r, double th, double out15[15]) {
    const geom_t g = geom_pub(a, r, th);
    const metric_deriv_t m = metric_upper_deriv(&g);
    metric_out(&m.g, out15);
    metric_out(&m.dr, out15 + 5);
    metric_out(&m.dth, out15 + 10);
}
double orc_horizon_outer(double a) { return horizon_outer(a); }
double orc_horizon_inner(double a) { return horizon_inner(a); }
double orc_isco_radius(double a, int sigma) { return isco_radius(a, sigma); }
double orc_photon_circular_orbit(double a, int sigma) { return photon_circular_orbit(a, sigma); }
double orc_circular_energy(double a, double r, int sigma) { return circular_energy(a, r, sigma); }
double orc_circular_angmom(double a, double r, int sigma) { return circular_angmom(a, r, sigma); }
double orc_disc_efficiency(double a, int sigma) { return disc_efficiency(a, sigma); }
void orc_keplerian_four_velocity(double a, double r, int sigma, double out4[4]) {
    keplerian_four_velocity(a, r, sigma, out4);
}
void orc_zamo_tetrad(double a, double r, double th, double out16[16]) {
    const geom_t g = geom_pub(a, r, th);
    const tetrad_t t = zamo_tetrad(&g);
    memcpy(out16, t.e, sizeof t.e);
}
double orc_carter_constant(double a, double th, double p_th, double E, double Lz) {
    return carter_constant(a, th, p_th, E, Lz, 0.0);
}
void orc_geodesic_rhs(double a, const double y[8], double dy[8]) { geodesic_rhs(a, y, dy); }
void orc_make_photon(double a, double r, double th, double phi, const double dir[3], double y_out[8]) {
    const geom_t g = geom_pub(a, r, th);
    const tetrad_t t = zamo_tetrad(&g);
    make_photon(a, r, th, phi, &t, dir, 1, y_out);
}
void orc_invariants(double a, const double y[8], double out5[5]) {
    const invariants_t iv = invariants(a, y);
    out5[0] = iv.E; out5[1] = iv.Lz; out5[2] = iv.Q; out5[3] = iv.norm; out5[4] = iv.norm_rel;
}
long orc_integrate(double a, const double y0[8], double h0, double rtol, double atol, int max_steps,
                   double r_in, double r_out, double y_out[8]) {
    /* validate.cpp:253-271 with a radial stop */
    stepper_t st;
    stepper_init(&st, a, rtol, atol);
    double y[8], ynew[8], h = h0;
    dense_t seg;
    memcpy(y, y0, sizeof y);
    long n = 0;
    for (int i = 0; i < max_steps; ++i) {
        int tries = 0, failed = 0;
        while (!try_step(&st, y, &h, ynew, &seg)) {
            if (++tries > 60) { failed = 1; break; }
        }
        if (failed) break;
        ++n;
        if (ynew[YR] < r_in || ynew[YR] > r_out) { memcpy(y, ynew, sizeof y); break; }
        memcpy(y, ynew, sizeof y);
    }
    memcpy(y_out, y, sizeof y);
    return n;
}
double orc_page_thorne_W(double a, double r, double r_isco) { return page_thorne_W(a, r, r_isco); }
double orc_disc_temperature(double M_kg, double spin, double r_out, double eddington, int sense, double r) {
    disc_t d;
    disc_init(&d, M_kg, spin, r_out, eddington, sense);
    return disc_temperature(&d, r);
}
double orc_planck_radiance(double lambda_m, double T) { return planck_radiance(lambda_m, T); }
void orc_blackbody_xyz_exact(double T, double out3[3]) { blackbody_xyz_exact(T, out3); }
void orc_blackbody_xyz(double T, double out3[3]) { blackbody_xyz(T, out3); }
double orc_bv_to_temperature(double bv) { return bv_to_temperature(bv); }
void orc_blackbody_table(double* out) {
    table_build();
    memcpy(out, g_lx, 3 * TABLE_N * sizeof(double));
}

int orc_star_catalogue(int count, uint64_t seed, int sky_mode, double* out6) {
    if (count < 0 || !out6) return BH_ERR_INVALID_ARG;
    rng_t rng = {seed};
    for (int i = 0; i < count; ++i) {
        star_t s;
        gen_star(&rng, sky_mode, &s);
        double* o = out6 + 6 * (size_t)i;
        o[0] = s.x; o[1] = s.y; o[2] = s.z; o[3] = s.mag; o[4] = s.T; o[5] = s.irr;
    }
    return BH_OK;
}

int orc_sky_radiance(int count, uint64_t seed, int sky_mode, int milky_way, const double* dirs, int n,
                     double sigma, double* out3) {
    starfield_t sf;
    if (starfield_build(&sf, count, seed, sky_mode, milky_way) != 0) return BH_ERR_OUT_OF_MEMORY;
    for (int i = 0; i < n; ++i) sky_radiance(&sf, dirs + 3 * (size_t)i, sigma, out3 + 3 * (size_t)i);
    starfield_free(&sf);
    return BH_OK;
}

void orc_ray_direction(const bh_camera* cam, double sx, double sy, double aspect, double out3[3]) {
    ray_direction(cam, sx, sy, aspect, out3);
}

int orc_trace_rays(const bh_render_config* cfg, int x0, int y0, int w, int h, bh_ray_result* out,
                   bh_render_stats* stats) {
    return run_window(cfg, x0, y0, w, h, out, NULL, stats);
}

int orc_render_window(const bh_render_config* cfg, int x0, int y0, int w, int h, bh_xyz* out,
                      bh_render_stats* stats) {
    return run_window(cfg, x0, y0, w, h, NULL, out, stats);
}


/* ---- display transform (image.cpp:22-191, spectrum.cpp:137-152) ------------ */

static int cmp_double(const void* a, const void* b) {
    const double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

/* image.cpp:22-45: the 99.9th and 99.99th percentiles (order statistics
   k = (size_t)(q (n - 1)) of the positive finite luminances) set the
   exposure.  A sort gives the same order statistic as nth_element. */
double orc_auto_exposure(const bh_xyz* px, long n, double key) {
    double* lum = (double*)malloc((size_t)(n > 0 ? n : 1) * sizeof(double));
    size_t m = 0;
    for (long i = 0; i < n; ++i)
        if (px[i].y > 0.0 && isfinite(px[i].y)) lum[m++] = px[i].y;
    if (m == 0) {
        free(lum);
        return 1.0;
    }
    qsort(lum, m, sizeof(double), cmp_double);
    size_t k1 = (size_t)(0.999 * (double)(m - 1));
    if (k1 > m - 1) k1 = m - 1;
    size_t k2 = (size_t)(0.9999 * (double)(m - 1));
    if (k2 > m - 1) k2 = m - 1;
    const double hi = lum[k1], peak = lum[k2];
    free(lum);
    double e = 1.0;
    if (hi > 0.0) e = key / hi;
    if (peak > 0.0) {
        const double c = 3.0 * key / peak;
        if (c < e) e = c;
    }
    return e;
}

static int clampi(int v, int lo, int hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

/* One separable Gaussian blur with clamped edges (image.cpp:60-91). */
static void glare_blur(const bh_xyz* src, int w, int h, double sigma, bh_xyz* dst) {
    int r = (int)ceil(3.0 * sigma);
    if (r < 1) r = 1;
    double* k = (double*)malloc((size_t)(2 * r + 1) * sizeof(double));
    double sum = 0.0;
    for (int i = -r; i <= r; ++i) {
        k[i + r] = exp(-0.5 * (i * i) / (sigma * sigma));
        sum += k[i + r];
    }
    for (int i = 0; i < 2 * r + 1; ++i) k[i] /= sum;
    bh_xyz* tmp = (bh_xyz*)malloc((size_t)w * h * sizeof(bh_xyz));
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            bh_xyz a = {0.0, 0.0, 0.0};
            for (int i = -r; i <= r; ++i) {
                const bh_xyz* q = &src[(size_t)y * w + clampi(x + i, 0, w - 1)];
                a.x += k[i + r] * q->x;
                a.y += k[i + r] * q->y;
                a.z += k[i + r] * q->z;
            }
            tmp[(size_t)y * w + x] = a;
        }
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            bh_xyz a = {0.0, 0.0, 0.0};
            for (int i = -r; i <= r; ++i) {
                const bh_xyz* q = &tmp[(size_t)clampi(y + i, 0, h - 1) * w + x];
                a.x += k[i + r] * q->x;
                a.y += k[i + r] * q->y;
                a.z += k[i + r] * q->z;
            }
            dst[(size_t)y * w + x] = a;
        }
    free(tmp);
    free(k);
}

/* image.cpp:47-104: a narrow (radius) and a wide (3 radius) Gaussian. */
void orc_add_glare(bh_xyz* px, int w, int h, double strength, double radius_px) {
    if (strength <= 0.0 || radius_px <= 0.0) return;
    const size_t n = (size_t)w * h;
    bh_xyz* nearp = (bh_xyz*)malloc(n * sizeof(bh_xyz));
    bh_xyz* farp = (bh_xyz*)malloc(n * sizeof(bh_xyz));
    glare_blur(px, w, h, radius_px, nearp);
    glare_blur(px, w, h, radius_px * 3.0, farp);
    const double core = 1.0 - strength;
    const double a = 0.7 * strength, b = 0.3 * strength;
    for (size_t i = 0; i < n; ++i) {
        px[i].x = px[i].x * core + nearp[i].x * a + farp[i].x * b;
        px[i].y = px[i].y * core + nearp[i].y * a + farp[i].y * b;
        px[i].z = px[i].z * core + nearp[i].z * a + farp[i].z * b;
    }
    free(nearp);
    free(farp);
}

static double clampd_(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

static double aces_curve(double x) {   /* Narkowicz's ACES fit, image.cpp:106-110 */
    const double a = 2.51, b = 0.03, c = 2.43, d = 0.59, e = 0.14;
    return clampd_((x * (a * x + b)) / (x * (c * x + d) + e), 0.0, 1.0);
}

static double srgb_encode(double v) {  /* image.cpp:112-115 */
    v = clampd_(v, 0.0, 1.0);
    return (v <= 0.0031308) ? 12.92 * v : 1.055 * pow(v, 1.0 / 2.4) - 0.055;
}

/* image.cpp:117-191 with spectrum.cpp:137-152 (XYZ -> linear sRGB, gamut clamp). */
void orc_develop(const bh_xyz* px, long n, double exposure, int tonemap, double log_decades,
                 uint8_t* out) {
    const double log_k = pow(10.0, clampd_(log_decades, 1.0, 20.0));
    for (long i = 0; i < n; ++i) {
        bh_xyz c = px[i];
        if (!isfinite(c.x) || !isfinite(c.y) || !isfinite(c.z)) c.x = c.y = c.z = 0.0;
        c.x *= exposure;
        c.y *= exposure;
        c.z *= exposure;
        double v[3];
        v[0] = 3.2404542 * c.x - 1.5371385 * c.y - 0.4985314 * c.z;
        v[1] = -0.9692660 * c.x + 1.8760108 * c.y + 0.0415560 * c.z;
        v[2] = 0.0556434 * c.x - 0.2040259 * c.y + 1.0572252 * c.z;
        double m = v[0];
        if (v[1] < m) m = v[1];
        if (v[2] < m) m = v[2];
        if (!(m >= 0.0)) {
            v[0] -= m;
            v[1] -= m;
            v[2] -= m;
        }
        for (int ch = 0; ch < 3; ++ch)
            if (v[ch] < 0.0) v[ch] = 0.0;
        for (int ch = 0; ch < 3; ++ch) {
            double x = v[ch];
            switch (tonemap) {
            case 0: x = clampd_(x, 0.0, 1.0); break;
            case 1: x = x / (1.0 + x); break;
            case 2: x = aces_curve(x); break;
            case 3: {
                const double denom = log10(1.0 + log_k);
                x = clampd_(log10(1.0 + log_k * (x < 0.0 ? 0.0 : x)) / denom, 0.0, 1.0);
                break;
            }
            default: {
                const double cap = 0.12, wt = 0.5;
                const double denom = log10(1.0 + log_k);
                const double f = aces_curve(x);
                const double l = clampd_(log10(1.0 + log_k * (x < 0.0 ? 0.0 : x)) / denom, 0.0, 1.0);
                const double lift = cap * tanh(wt * l / cap);
                x = clampd_(f + lift * (1.0 - f), 0.0, 1.0);
                break;
            }
            }
            v[ch] = x;
        }
        for (int ch = 0; ch < 3; ++ch) out[i * 3 + ch] = (uint8_t)lround(255.0 * srgb_encode(v[ch]));
    }
}


/* ---- jets ---------------------------------------------------------------- */
void orc_jet_configure(bh_jet* jet, double spin, double mdot_c2, double r_g_m) {
    jet_configure(jet, spin, mdot_c2, r_g_m);
}
void orc_powerlaw_xyz(double alpha, double out3[3]) { powerlaw_xyz(alpha, out3); }
double orc_jet_shape(const bh_jet* jet, double z, double rho) { return jet_shape(jet, z, rho); }
void orc_jet_four_velocity(const bh_jet* jet, double a, double r, double th, double out4[4]) {
    const geom_t g = geom_at(a, r, th);
    jet_four_velocity(jet, &g, out4);
}
