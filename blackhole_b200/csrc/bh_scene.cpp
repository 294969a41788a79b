// bh_scene.cpp - Host-side scene preparation (see bh_scene.h).
//
// The formulas below keep the reference's operand order: this file is
// compiled by the host compiler without FMA contraction, so the frame
// constants, star catalogue and blackbody table come out bit-identical to the
// ones the reference builds (the tests check the catalogue and table).
#include "bh_scene.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace bhg {

namespace {

constexpr double kPi = 3.14159265358979323846;
// constants.h:20-46
constexpr double kG = 6.67430e-11;
constexpr double kC = 2.99792458e8;
constexpr double kH = 6.62607015e-34;
constexpr double kKB = 1.380649e-23;
constexpr double kSigmaT = 6.6524587321e-29;
constexpr double kMp = 1.67262192369e-27;
constexpr double kMsun = 1.98847e30;
constexpr double kRsun = 6.957e8;
constexpr double kTsun = 5772.0;
constexpr double kMixedRtolFloor = 1e-6;
constexpr double kMixedAtolFloor = 1e-8;
// The reference's step cap hmax = kHmaxA max(1, r - r_h) + kHmaxB (render.cpp:130-131).
constexpr double kHmaxA = 0.05;
constexpr double kHmaxB = 0.01;
// The mixed path's own step cap, kHmaxLoose max(1, r - r_h), where it drops the reference's.
constexpr double kHmaxLoose = 0.3;

double clampd(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }
double maxd(double a, double b) { return (a < b) ? b : a; }

// ---- Kerr quantities at one point (kerr.h:44-59, 69-77, 187-194, 223-293) ----
struct G {
    double r, sn, cs, sn2, cs2, Sigma, Delta, A, a, a2;
};
G geom(double a, double r, double th) {
    G g;
    g.a = a;
    g.a2 = a * a;
    g.r = r;
    g.sn = std::sin(th);
    if (std::fabs(g.sn) < 1e-9) g.sn = (g.sn < 0.0 ? -1e-9 : 1e-9);
    g.cs = std::cos(th);
    g.sn2 = g.sn * g.sn;
    g.cs2 = g.cs * g.cs;
    g.Sigma = r * r + g.a2 * g.cs2;
    g.Delta = r * r - 2.0 * r + g.a2;
    g.A = (r * r + g.a2) * (r * r + g.a2) - g.a2 * g.Delta * g.sn2;
    return g;
}
double horizon_outer(double a) { const double d = 1.0 - a * a; return 1.0 + std::sqrt(maxd(0.0, d)); }
double horizon_inner(double a) { const double d = 1.0 - a * a; return 1.0 - std::sqrt(maxd(0.0, d)); }
double isco_radius(double a, int sigma) {
    const double a2 = a * a;
    const double Z1 = 1.0 + std::cbrt(1.0 - a2) * (std::cbrt(1.0 + a) + std::cbrt(1.0 - a));
    const double Z2 = std::sqrt(3.0 * a2 + Z1 * Z1);
    const double s = std::sqrt(maxd(0.0, (3.0 - Z1) * (3.0 + Z1 + 2.0 * Z2)));
    return 3.0 + Z2 - static_cast<double>(sigma) * s;
}
double circular_energy(double a, double r, int sigma) {
    const double sr = std::sqrt(r);
    const double num = r * r - 2.0 * r + sigma * a * sr;
    const double den = r * std::sqrt(r * r - 3.0 * r + 2.0 * sigma * a * sr);
    return num / den;
}

// ---- spectrum.cpp:13-73 ------------------------------------------------------
double planck(double l, double T) {
    if (T <= 0.0 || l <= 0.0) return 0.0;
    const double l5 = l * l * l * l * l;
    const double x = kH * kC / (l * kKB * T);
    if (x > 700.0) return 0.0;
    return (2.0 * kH * kC * kC) / (l5 * std::expm1(x));
}
// CIE 1931 multi-lobe fit (Wyman, Sloan & Shirley 2013).
double lobe(double x, double mu, double s1, double s2) {
    const double t = (x - mu) * ((x < mu) ? 1.0 / s1 : 1.0 / s2);
    return std::exp(-0.5 * t * t);
}
double cie_x(double nm) {
    return 1.056 * lobe(nm, 599.8, 37.9, 31.0) + 0.362 * lobe(nm, 442.0, 16.0, 26.7) -
           0.065 * lobe(nm, 501.1, 20.4, 26.2);
}
double cie_y(double nm) { return 0.821 * lobe(nm, 568.8, 46.9, 40.5) + 0.286 * lobe(nm, 530.9, 16.3, 31.1); }
double cie_z(double nm) { return 1.217 * lobe(nm, 437.0, 11.8, 36.0) + 0.681 * lobe(nm, 459.0, 26.0, 13.8); }
void bb_exact(double T, double o[3]) {
    o[0] = o[1] = o[2] = 0.0;
    if (T <= 0.0) return;
    const double lo = 360.0, hi = 830.0, dl = 1.0;
    for (double nm = lo; nm <= hi; nm += dl) {
        const double w = planck(nm * 1e-9, T) * dl * 1e-9;
        o[0] += w * cie_x(nm);
        o[1] += w * cie_y(nm);
        o[2] += w * cie_z(nm);
    }
}
constexpr double kLogTMin = 1.6989700043360187;
constexpr double kLogTMax = 9.4771212547196626;

double bv_to_temperature(double bv) {  // spectrum.cpp:158-162 (Ballesteros 2012)
    const double x = clampd(bv, -0.4, 2.0);
    return 4600.0 * (1.0 / (0.92 * x + 1.7) + 1.0 / (0.92 * x + 0.62));
}

// spectrum.cpp:77-92: CIE colour of a unit power law I_nu ~ nu^-alpha.
void powerlaw_xyz(double alpha, double out[3]) {
    constexpr double lambda_0 = 550e-9;
    out[0] = out[1] = out[2] = 0.0;
    constexpr double lo = 360.0, hi = 830.0, dl = 1.0;
    for (double nm = lo; nm <= hi; nm += dl) {
        const double lam = nm * 1e-9;
        const double I_l = kC * std::pow(lam / lambda_0, alpha) / (lam * lam);
        const double w = I_l * dl * 1e-9;
        out[0] += w * cie_x(nm);
        out[1] += w * cie_y(nm);
        out[2] += w * cie_z(nm);
    }
}

// ---- jet.h:77-315 (the host half: power and emissivity normalisation) ---------
double smoothstep01(double t) {
    t = clampd(t, 0.0, 1.0);
    return t * t * (3.0 - 2.0 * t);
}
double jet_radius(const bh_jet& j, double z_abs) {
    return j.R_base * std::pow(maxd(z_abs, 1e-6) / j.z_base, j.k);
}
double jet_gamma_at(const bh_jet& j, double z_abs) {
    const double t = std::min(1.0, std::pow(maxd(z_abs, 1e-6) / j.z_sat, j.k));
    return 1.0 + (j.gamma_max - 1.0) * t;
}
double jet_radial_profile(const bh_jet& j, double u) {
    const double s = (u - j.u_peak) / j.u_wid;
    const double t = u / j.spine_wid;
    return std::exp(-s * s) + j.spine * std::exp(-t * t);
}

// ---- scene.h:27-44 -------------------------------------------------------------
struct Rng {
    uint64_t s;
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * 0x1.0p-53; }
    double uniform(double a, double b) { return a + (b - a) * uniform(); }
    double normal() {
        const double u1 = maxd(uniform(), 1e-15), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
    }
};

struct Star { double x, y, z, mag, T, irr; };

// scene.h:62-104 for BH_SKY_GALACTIC; BH_SKY_UNIFORM is isotropic, m <= 6.5
// by the same inverse CDF, B-V uniform in [-0.3, 1.8].
Star gen_star(Rng& rng, int sky_mode) {
    Star s;
    double dir[3];
    if (sky_mode == BH_SKY_UNIFORM) {
        const double z = rng.uniform(-1.0, 1.0);
        const double ph = rng.uniform(0.0, 2.0 * kPi);
        const double rr = std::sqrt(maxd(0.0, 1.0 - z * z));
        dir[0] = rr * std::cos(ph); dir[1] = rr * std::sin(ph); dir[2] = z;
        s.x = dir[0]; s.y = dir[1]; s.z = dir[2];
        const double u = rng.uniform();
        s.mag = -1.5 + std::log10(u * (std::pow(10.0, 0.45 * (6.5 - -1.5)) - 1.0) + 1.0) / 0.45;
        const double bv = rng.uniform(-0.3, 1.8);
        s.T = bv_to_temperature(bv);
    } else {
        if (rng.uniform() < 0.45) {
            const double b = rng.normal() * 0.12;
            const double l = rng.uniform(0.0, 2.0 * kPi);
            const double cb = std::cos(b);
            const double gd[3] = {cb * std::cos(l), cb * std::sin(l), std::sin(b)};
            const double ca = 0.8660254037844387, sa = 0.5;   // scene.h:185-190
            dir[0] = gd[0];
            dir[1] = ca * gd[1] - sa * gd[2];
            dir[2] = sa * gd[1] + ca * gd[2];
        } else {
            const double z = rng.uniform(-1.0, 1.0);
            const double ph = rng.uniform(0.0, 2.0 * kPi);
            const double rr = std::sqrt(maxd(0.0, 1.0 - z * z));
            dir[0] = rr * std::cos(ph); dir[1] = rr * std::sin(ph); dir[2] = z;
        }
        s.x = dir[0]; s.y = dir[1]; s.z = dir[2];
        const double u = rng.uniform();
        s.mag = -1.5 + std::log10(u * (std::pow(10.0, 0.45 * (12.0 - -1.5)) - 1.0) + 1.0) / 0.45;
        double bv = 0.55 + 0.42 * rng.normal();
        if (rng.uniform() < 0.10) bv = rng.uniform(1.2, 1.9);
        s.T = bv_to_temperature(clampd(bv, -0.35, 1.95));
    }
    const double F0 = 3.64e-9 * 0.089 * 1e6 * 1e-6;
    s.irr = F0 * std::pow(10.0, -0.4 * s.mag);
    return s;
}

int bin_of(const Star& s) {  // scene.h:173-181
    const double theta = std::acos(clampd(s.z, -1.0, 1.0));
    const double phi = std::atan2(s.y, s.x);
    int ti = static_cast<int>(theta / kPi * kLat);
    int pi = static_cast<int>((phi + kPi) / (2.0 * kPi) * kLon);
    ti = std::clamp(ti, 0, kLat - 1);
    pi = ((pi % kLon) + kLon) % kLon;
    return ti * kLon + pi;
}

}  // namespace

void build_blackbody_table(std::vector<double>& tab) {
    tab.assign(3 * kTableN, 0.0);
    for (int i = 0; i < kTableN; ++i) {
        const double f = static_cast<double>(i) / (kTableN - 1);
        const double T = std::pow(10.0, kLogTMin + f * (kLogTMax - kLogTMin));
        double v[3];
        bb_exact(T, v);
        tab[i] = std::log(maxd(v[0], 1e-300));
        tab[kTableN + i] = std::log(maxd(v[1], 1e-300));
        tab[2 * kTableN + i] = std::log(maxd(v[2], 1e-300));
    }
}

void blackbody_xyz_host(const std::vector<double>& t, double T, double o[3]) {
    const double lg = std::log10(clampd(T, 50.0, 3.0e9));
    const double f = (lg - kLogTMin) / (kLogTMax - kLogTMin) * (kTableN - 1);
    const int i = std::clamp(static_cast<int>(f), 0, kTableN - 2);
    const double u = f - i;
    o[0] = std::exp(t[i] * (1.0 - u) + t[i + 1] * u);
    o[1] = std::exp(t[kTableN + i] * (1.0 - u) + t[kTableN + i + 1] * u);
    o[2] = std::exp(t[2 * kTableN + i] * (1.0 - u) + t[2 * kTableN + i + 1] * u);
}

int build_sky(int count, uint64_t seed, int sky_mode, const std::vector<double>& tab, HostSky& out,
              std::string& err) {
    if (count < 0) { err = "star_count must be >= 0"; return BH_ERR_INVALID_ARG; }
    if (sky_mode != BH_SKY_GALACTIC && sky_mode != BH_SKY_UNIFORM) {
        err = "unknown sky_mode";
        return BH_ERR_INVALID_ARG;
    }
    std::vector<Star> stars(static_cast<size_t>(count));
    Rng rng{seed};
    for (int i = 0; i < count; ++i) stars[i] = gen_star(rng, sky_mode);
    const int nb = kLat * kLon;
    std::vector<int> bins(static_cast<size_t>(count));
    out.bin_start.assign(nb + 1, 0);
    for (int i = 0; i < count; ++i) { bins[i] = bin_of(stars[i]); out.bin_start[bins[i] + 1]++; }
    for (int b = 0; b < nb; ++b) out.bin_start[b + 1] += out.bin_start[b];
    std::vector<int> fill(nb, 0);
    out.pos.assign(static_cast<size_t>(count), double4{0, 0, 0, 0});
    out.col.assign(static_cast<size_t>(count), double4{0, 0, 0, 0});
    for (int i = 0; i < count; ++i) {
        const int k = out.bin_start[bins[i]] + fill[bins[i]]++;   // catalogue order within a bin
        const Star& s = stars[i];
        out.pos[k] = double4{s.x, s.y, s.z, s.irr};
        double c[3];
        blackbody_xyz_host(tab, s.T, c);
        const double inv = (c[1] > 0.0) ? 1.0 / c[1] : 0.0;
        out.col[k] = double4{c[0], c[2], inv, 0.0};
    }
    // Diffuse background colour and brightness (scene.h:214-222).
    double c[3];
    blackbody_xyz_host(tab, 4800.0, c);
    out.mw_x = c[0];
    out.mw_z = c[2];
    out.mw_inv = (c[1] > 0.0) ? 1.0 / c[1] : 0.0;
    const double F0 = 3.24e-10;
    const double arcsec2_per_sr = 4.2545170296152206e10;
    out.diffuse_L = F0 * std::pow(10.0, -0.4 * 21.5) * arcsec2_per_sr;
    return BH_OK;
}

int star_catalogue(int count, uint64_t seed, int sky_mode, double* out6) {
    if (count < 0 || (count > 0 && !out6)) return BH_ERR_INVALID_ARG;
    if (sky_mode != BH_SKY_GALACTIC && sky_mode != BH_SKY_UNIFORM) return BH_ERR_INVALID_ARG;
    Rng rng{seed};
    for (int i = 0; i < count; ++i) {
        const Star s = gen_star(rng, sky_mode);
        double* o = out6 + 6 * static_cast<size_t>(i);
        o[0] = s.x; o[1] = s.y; o[2] = s.z; o[3] = s.mag; o[4] = s.T; o[5] = s.irr;
    }
    return BH_OK;
}

namespace {
// The binary32 copies of F's step-control constants (FrameParams::f_*).
void set_binary32_copies(FrameParams& F) {
    F.f_hmax_a = static_cast<float>(F.hmax_a);
    F.f_hmax_b = static_cast<float>(F.hmax_b);
    F.f_r_h = static_cast<float>(F.r_h);
    F.f_atol = static_cast<float>(F.atol);
    F.f_rtol = static_cast<float>(F.rtol);
    F.f_land_limit = static_cast<float>(F.land_limit);
    F.f_r_stop = static_cast<float>(F.r_stop);
    F.f_r_escape = static_cast<float>(F.r_escape);
    F.f_r_promote = static_cast<float>(F.r_promote);
    F.f_pad = 0.f;
}
}  // namespace

int make_frame(const bh_render_config& c, FrameParams& F, std::string& err) {
    std::memset(&F, 0, sizeof F);
    if (c.width <= 0 || c.height <= 0) { err = "width and height must be positive"; return BH_ERR_INVALID_ARG; }
    if (c.width > (1 << 16) || c.height > (1 << 16)) { err = "width/height above 65536"; return BH_ERR_INVALID_ARG; }
    const int S = std::max(1, c.sqrt_spp);
    if (S > 64) { err = "sqrt_spp above 64"; return BH_ERR_INVALID_ARG; }
    if (c.precision != BH_PRECISION_FP64 && c.precision != BH_PRECISION_MIXED) {
        err = "unknown precision";
        return BH_ERR_INVALID_ARG;
    }
    if (c.stop_mode != BH_STOP_REFERENCE && c.stop_mode != BH_STOP_RELATIVE) {
        err = "unknown stop_mode";
        return BH_ERR_INVALID_ARG;
    }
    if (c.sky_mode != BH_SKY_GALACTIC && c.sky_mode != BH_SKY_UNIFORM) {
        err = "unknown sky_mode";
        return BH_ERR_INVALID_ARG;
    }
    if (!(c.cam.r > 0.0) || !std::isfinite(c.cam.r) || !std::isfinite(c.cam.fov) || !std::isfinite(c.spin)) {
        err = "camera radius, fov and spin must be finite (r > 0)";
        return BH_ERR_INVALID_ARG;
    }
    double rtol = c.rtol, atol = c.atol;
    if (c.precision == BH_PRECISION_MIXED) {
        // binary32 stages cannot resolve a local error below ~1e-7 of the
        // state, so the mixed path's tolerances default to floors above that.
        rtol = (c.mixed_rtol > 0.0) ? c.mixed_rtol : maxd(c.rtol, kMixedRtolFloor);
        atol = (c.mixed_atol > 0.0) ? c.mixed_atol : maxd(c.atol, kMixedAtolFloor);
    }
    if (!(rtol >= 0.0) || !(atol >= 0.0)) { err = "tolerances must be >= 0"; return BH_ERR_INVALID_ARG; }
    if (c.stars_enabled && c.star_count < 0) { err = "star_count must be >= 0"; return BH_ERR_INVALID_ARG; }

    const double a = c.spin;
    F.a = a;
    F.a2 = a * a;
    F.r_plus = horizon_outer(a);
    F.r_minus = horizon_inner(a);
    F.factored_delta = (F.a2 < 1.0) ? 1 : 0;
    F.r_h = F.r_plus;
    F.r_stop = (c.stop_mode == BH_STOP_RELATIVE) ? F.r_plus * (1.0 + c.stop_epsilon)
                                                 : F.r_plus * 1.0 + 1e-4 + (F.r_plus - F.r_minus) * 1e-3;
    F.r_escape = c.r_escape;
    F.rtol = rtol;
    F.atol = atol;
    F.rtol_ref = c.rtol;
    F.atol_ref = c.atol;
    F.h0 = 0.02 * maxd(1.0, c.cam.r);
    // The step cap (render.cpp:130-131).  The mixed path may drop it where no
    // event needs it: the disc-plane and horizon tests look at step ends,
    // which the error control keeps close together near the hole, while the
    // Sun's probes, the neutron star's surface test and the jet's quadrature
    // sample within each step.
    if (c.mixed_step_limit < BH_STEP_LIMIT_AUTO || c.mixed_step_limit > BH_STEP_LIMIT_NONE) {
        err = "unknown mixed_step_limit";
        return BH_ERR_INVALID_ARG;
    }
    const bool needs_cap = c.sun_enabled || c.star.enabled || c.jet_enabled;
    const bool capped = c.precision != BH_PRECISION_MIXED || c.mixed_step_limit == BH_STEP_LIMIT_REFERENCE ||
                        (c.mixed_step_limit == BH_STEP_LIMIT_AUTO && needs_cap);
    // Without the reference's cap the mixed path keeps a looser one,
    // h <= 0.3 max(1, r - r_h): far out the error control alone lets the
    // step grow past the scale on which the strong field sets in, and the
    // attempts that overshoot are rejected.  Measured on the CPU
    // restatement at rtol 1e-6 (edge-on frame, every 32nd row): 58.4 attempts
    // per ray instead of 64.9 (with 50.9 accepted steps instead of 51.3),
    // the direction error unchanged (p99 2.6e-6 rad); over 120 random scenes
    // 8% fewer attempts and fewer rays beyond 1e-4 rad.  BH_STEP_LIMIT_NONE
    // leaves the error control alone.
    const bool none = c.precision == BH_PRECISION_MIXED && c.mixed_step_limit == BH_STEP_LIMIT_NONE;
    F.hmax_a = capped ? kHmaxA : (none ? 1e30 : kHmaxLoose);
    F.hmax_b = capped ? kHmaxB : (none ? 1e30 : 0.0);
    // The final state of an escaping ray is the end of the step that crosses
    // r_escape (render.cpp:247-251); under the reference's cap that end lies
    // within hmax(r_escape) beyond it.  An uncapped step may end far beyond,
    // where a ray from a camera close to the hole has bent further, so the
    // mixed path shortens a step from inside r_escape that would end beyond
    // r_escape + hmax(r_escape) to end near r_escape + hmax(r_escape) / 2.
    const double hm_escape = kHmaxA * maxd(1.0, c.r_escape - F.r_h) + kHmaxB;
    F.land_escape = (c.precision == BH_PRECISION_MIXED && !capped) ? 1 : 0;
    F.land_limit = c.r_escape + hm_escape;
    F.land_target = c.r_escape + 0.5 * hm_escape;
    if (c.mixed_capture != BH_CAPTURE_AUTO && c.mixed_capture != BH_CAPTURE_REFERENCE) {
        err = "unknown mixed_capture";
        return BH_ERR_INVALID_ARG;
    }
    F.early_capture = (c.precision == BH_PRECISION_MIXED && c.mixed_capture == BH_CAPTURE_AUTO &&
                       !c.star.enabled && !c.jet_enabled) ? 1 : 0;
    // The mixed path integrates the southern hemisphere as its mirror image
    // (Kerr is symmetric under th -> pi - th, p_th -> -p_th), so that a ray
    // near either pole has a small angle, which binary32 resolves; the Sun,
    // the neutron star's caps and the jets are not mirror-symmetric, so
    // scenes with them keep the true angle.
    F.mirror_ok = (c.precision == BH_PRECISION_MIXED && !c.sun_enabled && !c.star.enabled && !c.jet_enabled) ? 1 : 0;
    if (c.mixed_near_critical != BH_NEAR_CRITICAL_AUTO && c.mixed_near_critical != BH_NEAR_CRITICAL_BINARY32) {
        err = "unknown mixed_near_critical";
        return BH_ERR_INVALID_ARG;
    }
    F.fp64_near_critical = (c.precision == BH_PRECISION_MIXED && c.mixed_near_critical == BH_NEAR_CRITICAL_AUTO) ? 1 : 0;
    // Innermost (prograde equatorial) photon orbit, kerr.h:217-220 with |a|:
    // a photon from far away that is moving inwards below it has no radial
    // turning point left and falls into the hole.
    F.r_promote = (F.a2 < 1.0) ? 2.0 * (1.0 + std::cos((2.0 / 3.0) * std::acos(-std::fabs(a)))) : 0.0;
    F.max_steps = c.max_steps;
    set_binary32_copies(F);

    // Camera (scene.h:356-384, render.cpp:409-414).
    F.cam_r = c.cam.r;
    F.cam_th = c.cam.theta;
    F.cam_ph = c.cam.phi;
    F.tanf = std::tan(0.5 * c.cam.fov);
    F.aspect = static_cast<double>(c.width) / c.height;
    F.has_roll = (c.cam.roll != 0.0) ? 1 : 0;
    F.cr = std::cos(c.cam.roll);
    F.sr = std::sin(c.cam.roll);
    F.cp = std::cos(c.cam.pitch);
    F.sp = std::sin(c.cam.pitch);
    F.cy = std::cos(c.cam.yaw);
    F.sy = std::sin(c.cam.yaw);
    F.S = S;
    F.inv_S = 1.0 / S;
    F.inv_SS = 1.0 / (S * S);
    const G g = geom(a, c.cam.r, c.cam.theta);
    if (!(g.Delta > 0.0) || !(g.A > 0.0)) {
        err = "camera must be outside the horizon";
        return BH_ERR_INVALID_ARG;
    }
    // ZAMO tetrad (kerr.h:270-293)
    const double alpha = std::sqrt(g.Sigma * g.Delta / g.A);
    const double omega = 2.0 * g.a * g.r / g.A;
    F.tet00 = 1.0 / alpha;
    F.tet03 = omega / alpha;
    F.tet11 = std::sqrt(g.Delta / g.Sigma);
    F.tet22 = 1.0 / std::sqrt(g.Sigma);
    F.tet33 = std::sqrt(g.Sigma / g.A) / g.sn;
    // metric_lower at the camera (kerr.h:69-77)
    F.ml_tt = -(1.0 - 2.0 * g.r / g.Sigma);
    F.ml_tp = -2.0 * g.a * g.r * g.sn2 / g.Sigma;
    F.ml_rr = g.Sigma / g.Delta;
    F.ml_thth = g.Sigma;
    F.ml_pp = g.A * g.sn2 / g.Sigma;
    {
        // carter_constant's own clamp (kerr.h:344-346)
        double sn = std::sin(c.cam.theta);
        if (std::fabs(sn) < 1e-9) sn = 1e-9;
        F.cam_sn2 = sn * sn;
        F.cam_cs2 = std::cos(c.cam.theta) * std::cos(c.cam.theta);
    }
    F.seed = c.seed;
    F.width = c.width;
    F.height = c.height;
    F.n_rays = static_cast<long long>(c.width) * c.height * S * S;

    // Novikov-Thorne disc (disc.h:73-82, W constants of disc.h:46-60).
    F.disc_enabled = c.disc_enabled ? 1 : 0;
    if (c.disc_enabled) {
        const double ad = clampd(a, -0.9999, 0.9999);
        const int sg = c.disc_sense;
        if (sg != 1 && sg != -1) { err = "disc_sense must be +1 or -1"; return BH_ERR_INVALID_ARG; }
        F.disc_a = ad;
        F.disc_sigma = sg;
        F.r_in = isco_radius(ad, sg);
        F.r_out = maxd(c.disc_r_out, isco_radius(ad, sg) * 1.02);
        const double eta = 1.0 - circular_energy(ad, isco_radius(ad, sg), sg);
        const double L_edd = 4.0 * kPi * kG * c.M_kg * kMp * kC / kSigmaT;
        F.disc_mdot = c.eddington * (L_edd / (eta * kC * kC));
        F.disc_eta = eta;
        const double r_g = kG * c.M_kg / (kC * kC);
        F.disc_rg2 = r_g * r_g;
        F.x0 = std::sqrt(F.r_in);
        const double ac = std::acos(clampd(ad, -1.0, 1.0));
        const double x[3] = {2.0 * std::cos(ac / 3.0 - kPi / 3.0), 2.0 * std::cos(ac / 3.0 + kPi / 3.0),
                             -2.0 * std::cos(ac / 3.0)};
        const int jk[3][2] = {{1, 2}, {0, 2}, {0, 1}};
        for (int i = 0; i < 3; ++i) {
            const double xi = x[i], xj = x[jk[i][0]], xk = x[jk[i][1]];
            F.pt_x[i] = xi;
            F.pt_den[i] = F.x0 - xi;
            F.pt_c[i] = (std::fabs(xi) < 1e-13) ? 0.0 : 3.0 * (xi - ad) * (xi - ad) / (xi * (xi - xj) * (xi - xk));
        }
    }

    // Sky (render.cpp:413-414, scene.h:114-124).
    F.stars_enabled = c.stars_enabled ? 1 : 0;
    F.milky_way = c.milky_way ? 1 : 0;
    F.sky_mode = c.sky_mode;
    F.psf_sigma = 0.55 * (c.cam.fov / c.width);
    F.cutoff = 3.0 * F.psf_sigma;
    // Stars whose direction cosine lies below this are farther than the
    // cutoff for certain (the margin covers the rounding of acos), so their
    // acos need not be taken.
    F.cut_dot = (F.cutoff * 1.000001 < kPi) ? std::cos(F.cutoff * 1.000001) : -1.0;
    F.inv2s2 = 1.0 / (2.0 * F.psf_sigma * F.psf_sigma);
    F.psf_norm = 1.0 / (2.0 * kPi * F.psf_sigma * F.psf_sigma);
    F.span_t = std::max(1, static_cast<int>(std::ceil(F.cutoff / (kPi / kLat))));

    // Surfaces.
    F.sun_enabled = c.sun_enabled ? 1 : 0;
    for (int i = 0; i < 3; ++i) F.sun_c[i] = c.sun.centre[i];
    F.sun_R = c.sun.radius;
    F.sun_R2 = c.sun.radius * c.sun.radius;
    F.sun_T_eff = c.sun.T_eff;
    F.sun_redshift_div = 1.0 + kG * kMsun / (kRsun * kC * kC);   // scene.h:239-240
    F.ns_enabled = c.star.enabled ? 1 : 0;
    F.ns_R = c.star.R;
    F.ns_T_eff = c.star.T_eff;
    F.ns_Omega = c.star.Omega;
    F.ns_caps = c.star.caps ? 1 : 0;
    F.ns_two_caps = c.star.two_caps ? 1 : 0;
    F.ns_cap_tilt = c.star.cap_tilt;
    F.ns_cap_radius = c.star.cap_radius;
    F.ns_cap_T = c.star.cap_T;
    F.ns_cap_phase0 = c.star.cap_phase0;

    F.hs_enabled = c.hotspot.enabled ? 1 : 0;
    F.hs_r = c.hotspot.r;
    F.hs_phi0 = c.hotspot.phi0;
    F.hs_sigma = c.hotspot.sigma;
    F.hs_contrast = c.hotspot.contrast;
    F.hs_omega = c.hotspot.omega;
    F.observer_time = c.observer_time;

    // Jet: the model as configured (render() reads cfg.jet as given).
    F.jet_enabled = c.jet_enabled ? 1 : 0;
    if (c.jet_enabled) {
        const bh_jet& j = c.jet;
        if (!(j.z_base > 0.0) || !(j.z_sat > 0.0) || !(j.R_base > 0.0) || !(j.u_wid > 0.0) ||
            !(j.spine_wid > 0.0) || !(j.z_top > 0.0)) {
            err = "jet z_base, z_top, z_sat, R_base, u_wid and spine_wid must be positive";
            return BH_ERR_INVALID_ARG;
        }
        F.jet_z_base = j.z_base;
        F.jet_z_top = j.z_top;
        F.jet_R_base = j.R_base;
        F.jet_k = j.k;
        F.jet_gamma_max = j.gamma_max;
        F.jet_z_sat = j.z_sat;
        F.jet_alpha = j.alpha;
        F.jet_u_peak = j.u_peak;
        F.jet_u_wid = j.u_wid;
        F.jet_spine = j.spine;
        F.jet_spine_wid = j.spine_wid;
        F.jet_zeta = j.zeta;
        F.jet_Omega_F = j.Omega_F;
        F.jet_j_nu0 = j.j_nu0;
        F.jet_r_bound = j.r_bound;
        powerlaw_xyz(j.alpha, F.jet_col);   // render.cpp:417
    }
    return BH_OK;
}

FrameParams binary64_treatment(const FrameParams& F) {
    FrameParams G = F;
    G.rtol = F.rtol_ref;
    G.atol = F.atol_ref;
    G.hmax_a = kHmaxA;
    G.hmax_b = kHmaxB;
    G.land_escape = 0;
    G.early_capture = 0;
    G.mirror_ok = 0;
    set_binary32_copies(G);
    return G;
}

void jet_configure(bh_jet& j, double spin, double mdot_c2, double r_g_m) {
    // kerr.h:204-207 and jet.h:81-87
    const double rp = horizon_outer(spin);
    const double OmH = (rp > 0.0) ? spin / (2.0 * rp) : 0.0;
    j.a = spin;
    j.Omega_F = 0.5 * OmH;
    {
        const double x = OmH * OmH;
        const double f = 1.0 + 1.38 * x - 9.2 * x * x;
        const double kappa = 0.053, phi = j.phi_flux;
        j.P_jet = (kappa / (4.0 * kPi)) * phi * phi * x * std::max(0.0, f) * mdot_c2;
    }
    j.L_rad = j.eps_rad * j.P_jet;
    j.r_bound = std::sqrt(j.z_top * j.z_top + jet_radius(j, j.z_top) * jet_radius(j, j.z_top)) * 1.05;
    double C_f = 0.0;
    {
        constexpr int N = 2000;
        const double du = 3.0 / N;
        for (int i = 0; i < N; ++i) {
            const double u = (i + 0.5) * du;
            C_f += jet_radial_profile(j, u) * u * du;
        }
    }
    double V = 0.0;
    {
        constexpr int N = 4000;
        const double dz = (j.z_top - j.z_base) / N;
        for (int i = 0; i < N; ++i) {
            const double z = j.z_base + (i + 0.5) * dz;
            const double R = jet_radius(j, z);
            const double gz = std::pow(jet_gamma_at(j, z) / jet_gamma_at(j, j.z_base), -(2.0 + j.alpha)) *
                              std::pow(R / j.R_base, -(3.0 + j.alpha)) * std::pow(z / j.z_base, j.zeta);
            const double ramp = smoothstep01((z - j.z_base) / (0.5 * j.z_base)) *
                                smoothstep01((j.z_top - z) / (0.15 * j.z_top));
            V += gz * ramp * R * R * dz;
        }
        V *= 2.0 * (2.0 * kPi) * C_f;
    }
    j.volume_rg3 = V;
    const double V_m3 = V * r_g_m * r_g_m * r_g_m;
    if (!(V_m3 > 0.0) || !(j.L_rad > 0.0)) {
        j.j_nu0 = 0.0;
        return;
    }
    const double A = j.L_rad / (4.0 * kPi * V_m3);
    constexpr double nu_0 = kC / 550e-9, nu_lo = 1.0e9, nu_hi = 1.0e17;
    const double p = 1.0 - j.alpha;
    const double band = (std::fabs(p) > 1e-9) ? (std::pow(nu_hi, p) - std::pow(nu_lo, p)) / p
                                              : std::log(nu_hi / nu_lo);
    j.j_nu0 = A / (std::pow(nu_0, j.alpha) * band) * r_g_m;
}

int setup_jet(bh_render_config& c) {
    if (!c.jet_enabled) return BH_OK;
    if (c.star.enabled || !c.disc_enabled) {   // no horizon, or no accretion flow
        c.jet_enabled = 0;
        return BH_OK;
    }
    c.jet.z_sat = std::min(c.jet.z_sat, 0.7 * c.jet.z_top);
    const double ad = clampd(c.spin, -0.9999, 0.9999);
    const int sg = c.disc_sense;
    const double eta = 1.0 - circular_energy(ad, isco_radius(ad, sg), sg);
    const double L_edd = 4.0 * kPi * kG * c.M_kg * kMp * kC / kSigmaT;
    const double mdot = c.eddington * (L_edd / (eta * kC * kC));
    const double r_g = kG * c.M_kg / (kC * kC);
    jet_configure(c.jet, c.spin, mdot * kC * kC, r_g);
    if (!(c.jet.P_jet > 0.0)) c.jet_enabled = 0;
    return BH_OK;
}

void default_config(bh_render_config& c) {
    std::memset(&c, 0, sizeof c);
    c.struct_size = sizeof(bh_render_config);
    c.abi_version = BH_GPU_ABI_VERSION;
    c.M_kg = 10.0 * kMsun;
    c.spin = 0.9;
    c.cam.r = 60.0;
    c.cam.theta = kPi / 2.0;
    c.cam.phi = 0.0;
    c.cam.fov = 0.6;
    c.width = 1280;
    c.height = 720;
    c.sqrt_spp = 2;
    c.disc_enabled = 1;
    c.disc_r_out = 24.0;
    c.eddington = 0.1;
    c.disc_sense = 1;
    c.stars_enabled = 1;
    c.star_count = 250000;
    c.seed = 20240921ull;
    c.sun.radius = 1.0;
    c.sun.T_eff = kTsun;
    c.hotspot.r = 8.0;
    c.hotspot.sigma = 0.6;
    c.hotspot.contrast = 25.0;
    c.hotspot.sense = 1;
    c.star.M_kg = 1.4 * kMsun;
    c.star.R_m = 12000.0;
    c.star.R = 5.8;
    c.star.T_eff = 1.0e6;
    c.star.cap_tilt = 60.0 * kPi / 180.0;
    c.star.cap_radius = 20.0 * kPi / 180.0;
    c.star.cap_T = 3.0e6;
    c.star.two_caps = 1;
    c.rtol = 1e-9;
    c.atol = 1e-11;
    c.r_escape = 4000.0;
    c.max_steps = 20000;
    c.precision = BH_PRECISION_FP64;
    c.sky_mode = BH_SKY_GALACTIC;
    c.stop_mode = BH_STOP_REFERENCE;
    c.milky_way = 1;
    // jet.h:96-146
    c.jet.z_base = 3.0;
    c.jet.z_top = 120.0;
    c.jet.R_base = 1.6;
    c.jet.k = 0.58;
    c.jet.gamma_max = 10.0;
    c.jet.z_sat = 80.0;
    c.jet.alpha = 0.7;
    c.jet.u_peak = 0.82;
    c.jet.u_wid = 0.17;
    c.jet.spine = 0.06;
    c.jet.spine_wid = 0.40;
    c.jet.zeta = 2.0;
    c.jet.eps_rad = 0.02;
    c.jet.phi_flux = 50.0;
}

}  // namespace bhg
