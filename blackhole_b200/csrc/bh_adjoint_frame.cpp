// bh_adjoint_frame.cpp - Per-frame derivatives for the discrete adjoint.
//
// The camera tetrad and metric (kerr.h:44-77, 270-293) as functions of the
// spin and the camera's polar angle, and the disc constants (disc.h:46-82:
// ISCO radius, the Page-Thorne W roots and coefficients, the accretion rate
// through the efficiency) as functions of the spin, evaluated once with dual
// numbers: their values are the frame constants of make_frame, their tangents
// the derivatives the per-ray adjoint contracts with.
#include "bh_adjoint.h"

#include <cmath>

#include "bh_dual.cuh"

namespace bhg {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kG = 6.67430e-11;
constexpr double kC = 2.99792458e8;
constexpr double kSigmaT = 6.6524587321e-29;
constexpr double kMp = 1.67262192369e-27;

template <class T>
T isco_t(const T& a, int sigma) {
    const T a2 = a * a;
    const T Z1 = 1.0 + cbrt(1.0 - a2) * (cbrt(1.0 + a) + cbrt(1.0 - a));
    const T Z2 = sqrt(3.0 * a2 + Z1 * Z1);
    T q = (3.0 - Z1) * (3.0 + Z1 + 2.0 * Z2);
    if (q.v < 0.0) q = T(0.0);
    return 3.0 + Z2 - static_cast<double>(sigma) * sqrt(q);
}

template <class T>
T circular_energy_t(const T& a, const T& r, int sigma) {
    const T sr = sqrt(r);
    const T num = r * r - 2.0 * r + static_cast<double>(sigma) * a * sr;
    const T den = r * sqrt(r * r - 3.0 * r + 2.0 * static_cast<double>(sigma) * a * sr);
    return num / den;
}

}  // namespace

int make_adjoint_frame(const bh_render_config& c, const FrameParams& F, AdjointFrame& X, std::string& err) {
    X = AdjointFrame{};
    if (c.sun_enabled || c.star.enabled || c.hotspot.enabled || c.jet_enabled) {
        err = "the adjoint covers disc and sky scenes (no Sun, neutron star, hot spot or jet)";
        return BH_ERR_UNSUPPORTED;
    }
    if (!(F.a2 < 1.0)) {
        err = "the adjoint needs |spin| < 1";
        return BH_ERR_INVALID_ARG;
    }
    X.checkpoint_interval = 16;
    X.checkpoint_slots = 64;

    // Camera: slot 0 = spin, slot 1 = polar angle.
    using D2 = Dual<2>;
    const D2 a = D2::var(c.spin, kParSpin);
    const D2 th = D2::var(c.cam.theta, kParIncl);
    const double r = c.cam.r;
    D2 sn = sin(th);
    if (std::fabs(sn.v) < 1e-9) sn = D2(sn.v < 0.0 ? -1e-9 : 1e-9);
    const D2 cs = cos(th);
    const D2 a2 = a * a;
    const D2 sn2 = sn * sn, cs2 = cs * cs;
    const D2 Sigma = r * r + a2 * cs2;
    const D2 Delta = r * r - 2.0 * r + a2;
    const D2 A = (r * r + a2) * (r * r + a2) - a2 * Delta * sn2;
    const D2 alpha = sqrt(Sigma * Delta / A);
    const D2 omega = 2.0 * a * r / A;
    const D2 tet[5] = {1.0 / alpha, omega / alpha, sqrt(Delta / Sigma), 1.0 / sqrt(Sigma), sqrt(Sigma / A) / sn};
    const D2 ml[5] = {-(1.0 - 2.0 * r / Sigma), -2.0 * a * r * sn2 / Sigma, Sigma / Delta, Sigma, A * sn2 / Sigma};
    for (int i = 0; i < 5; ++i)
        for (int q = 0; q < 2; ++q) {
            X.d_tet[i][q] = tet[i].d[q];
            X.d_ml[i][q] = ml[i].d[q];
        }

    // Disc: one slot, the spin (zero where the disc clamps it).
    if (F.disc_enabled) {
        using D1 = Dual<1>;
        const bool free_spin = std::fabs(c.spin) < 0.9999;
        D1 ad(F.disc_a);
        ad.d[0] = free_spin ? 1.0 : 0.0;
        const int sg = F.disc_sigma;
        const D1 r_in = isco_t(ad, sg);
        const D1 x0 = sqrt(r_in);
        const D1 ac = acos(ad);
        const D1 xr[3] = {2.0 * cos(ac / 3.0 - kPi / 3.0), 2.0 * cos(ac / 3.0 + kPi / 3.0), -2.0 * cos(ac / 3.0)};
        const int jk[3][2] = {{1, 2}, {0, 2}, {0, 1}};
        X.d_disc_a = ad.d[0];
        X.d_x0 = x0.d[0];
        for (int i = 0; i < 3; ++i) {
            const D1 xi = xr[i], xj = xr[jk[i][0]], xk = xr[jk[i][1]];
            X.d_pt_x[i] = xi.d[0];
            X.d_pt_den[i] = (x0 - xi).d[0];
            X.d_pt_c[i] = (F.pt_c[i] == 0.0)
                              ? 0.0
                              : (3.0 * (xi - ad) * (xi - ad) / (xi * (xi - xj) * (xi - xk))).d[0];
        }
        const D1 eta = 1.0 - circular_energy_t(ad, r_in, sg);
        const double L_edd = 4.0 * kPi * kG * c.M_kg * kMp * kC / kSigmaT;
        const D1 per_edd = L_edd / (eta * kC * kC);
        X.d_mdot_da = c.eddington * per_edd.d[0];
        X.d_mdot_dedd = per_edd.v;
    }
    return BH_OK;
}

}  // namespace bhg
