// ref_harness.cpp - C entry points onto the reference renderer itself.
//
// TEST INFRASTRUCTURE.  This translation unit includes the reference's
// render.cpp (and through it kerr.h, geodesic.h, disc.h, scene.h) and is
// linked with the reference's spectrum.cpp, all compiled unmodified from the
// reference tree into oracle/_ref/libbh_ref.so by oracle/Makefile.  It gives
// the tests and the CPU baseline access to:
//   - ref_render:        the reference's own bh::render (render.cpp:396-497);
//   - ref_render_rows:   the reference's trace() + shade() over a set of rows,
//                        in a row-atomic std::thread pool like render() uses
//                        (render.cpp:420-477), for bounded timing samples;
//   - ref_trace_rays:    per-sample trace()/shade() results of a pixel window;
//   - ref_* functions:   the known-answer quantities of validate.cpp.
// Nothing here is shipped or called by the GPU library.

// Standard headers first, so that the access override below touches only the
// reference's own classes (StarField keeps its catalogue private).
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#define private public
#include "render.cpp"
#undef private
#include "image.h"

#include "../include/bh_gpu.h"
#include "ref_config.h"

namespace {

int check_cfg(const bh_render_config* c) {
    if (!c || c->width <= 0 || c->height <= 0) return BH_ERR_INVALID_ARG;
    // The reference has one sky and one stop rule.
    if (c->sky_mode != BH_SKY_GALACTIC || c->stop_mode != BH_STOP_REFERENCE)
        return BH_ERR_UNSUPPORTED;
    return BH_OK;
}

void stats_out(const bh::RenderStats& s, bh_render_stats* o) {
    if (!o) return;
    o->rays += s.rays;
    o->steps += s.steps;
    o->captured += s.captured;
    o->disc_hits += s.disc_hits;
    o->sun_hits += s.sun_hits;
    o->star_hits += s.star_hits;
    o->jet_rays += s.jet_rays;
    o->escaped += s.escaped;
    o->exhausted += s.exhausted;
    o->total_flux += s.total_flux;
    o->max_norm_error = std::max(o->max_norm_error, s.max_norm_error);
    o->max_carter_drift = std::max(o->max_carter_drift, s.max_carter_drift);
    o->seconds = s.seconds;
}

// Everything render() builds before its pixel loop (render.cpp:396-418).
struct Scene {
    bh::RenderConfig cfg;
    std::unique_ptr<bh::NovikovThorneDisc> disc;
    std::unique_ptr<bh::StarField> stars;
    bh::Tetrad tet;
    double aspect, psf_sigma;
    spec::XYZ jet_colour;
    explicit Scene(const bh_render_config& c, bool milky_way) : cfg(to_ref(c)) {
        if (cfg.disc_enabled)
            disc = std::make_unique<bh::NovikovThorneDisc>(cfg.M_kg, cfg.spin, cfg.disc_r_out,
                                                           cfg.eddington, cfg.disc_sense);
        if (cfg.stars_enabled)
            stars = std::make_unique<bh::StarField>(cfg.star_count, cfg.seed, milky_way);
        const bh::Geom gcam = bh::geom_at(cfg.spin, cfg.cam.r, cfg.cam.theta);
        tet = bh::zamo_tetrad(gcam);
        aspect = static_cast<double>(cfg.width) / cfg.height;
        psf_sigma = 0.55 * (cfg.cam.fov / cfg.width);
        jet_colour = cfg.jet.enabled ? spec::powerlaw_xyz(cfg.jet.alpha) : spec::XYZ{};   // render.cpp:417
    }
};

}  // namespace

extern "C" {

int ref_render(const bh_render_config* c, bh_xyz* out, bh_render_stats* st) {
    const int rc = check_cfg(c);
    if (rc != BH_OK) return rc;
    if (!c->milky_way && c->stars_enabled) return BH_ERR_UNSUPPORTED;
    const bh::RenderConfig cfg = to_ref(*c);
    bh::RenderStats s;
    const img::Image im = bh::render(cfg, s);
    if (out) std::memcpy(out, im.pixels.data(), im.pixels.size() * sizeof(spec::XYZ));
    stats_out(s, st);
    return BH_OK;
}

// The pixel loop of render.cpp:428-463 restricted to the listed rows, on
// `threads` workers pulling rows from an atomic counter.  Pixels go to
// out[k * width + x] for the k-th listed row.  Scene setup (disc, star
// catalogue, spectrum table) is done before the clock starts and reported in
// st->seconds separately from tracing: *setup_seconds gets the setup time.
int ref_render_rows(const bh_render_config* c, const int* rows, int nrows, int threads,
                    bh_xyz* out, bh_render_stats* st, double* setup_seconds) {
    const int rc = check_cfg(c);
    if (rc != BH_OK) return rc;
    if (nrows < 0 || (nrows > 0 && !rows)) return BH_ERR_INVALID_ARG;
    for (int k = 0; k < nrows; ++k)
        if (rows[k] < 0 || rows[k] >= c->height) return BH_ERR_INVALID_ARG;
    const auto t_setup = std::chrono::steady_clock::now();
    Scene sc(*c, c->milky_way != 0);
    (void)spec::blackbody_xyz(5000.0);  // build the magic-static table outside the clock
    const auto t_start = std::chrono::steady_clock::now();
    if (setup_seconds)
        *setup_seconds = std::chrono::duration<double>(t_start - t_setup).count();

    int nthreads = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
    if (nthreads <= 0) nthreads = 1;
    std::atomic<int> next{0};
    std::vector<bh::RenderStats> per_thread(nthreads);
    const bh::RenderConfig& cfg = sc.cfg;
    auto worker = [&](int tid) {
        bh::RenderStats& local = per_thread[tid];
        const int S = std::max(1, cfg.sqrt_spp);
        const double inv_S = 1.0 / S;
        for (;;) {
            const int k = next.fetch_add(1);
            if (k >= nrows) break;
            const int y = rows[k];
            for (int x = 0; x < cfg.width; ++x) {
                bh::Rng rng(cfg.seed ^ (static_cast<uint64_t>(y) << 32) ^
                            (static_cast<uint64_t>(x) * 0x9E3779B97F4A7C15ull));
                spec::XYZ acc{};
                for (int sy = 0; sy < S; ++sy)
                    for (int sx = 0; sx < S; ++sx) {
                        const double jx = (sx + rng.uniform()) * inv_S;
                        const double jy = (sy + rng.uniform()) * inv_S;
                        const double u = (2.0 * (x + jx) / cfg.width - 1.0);
                        const double v = (1.0 - 2.0 * (y + jy) / cfg.height);
                        double dir[3];
                        cfg.cam.ray_direction(u, v, sc.aspect, dir);
                        ++local.rays;
                        const bh::Hit hit = bh::trace(cfg, sc.disc.get(), dir, sc.tet, local);
                        const spec::XYZ col = bh::shade(cfg, sc.disc.get(), sc.stars.get(), hit,
                                                        sc.psf_sigma, sc.jet_colour, local);
                        acc.x += col.x; acc.y += col.y; acc.z += col.z;
                    }
                const double w = 1.0 / (S * S);
                if (out) out[static_cast<size_t>(k) * cfg.width + x] = {acc.x * w, acc.y * w, acc.z * w};
                local.total_flux += acc.y * w;
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker, t);
    for (auto& th : pool) th.join();
    bh::RenderStats total;
    for (const auto& s : per_thread) {
        total.rays += s.rays; total.steps += s.steps; total.captured += s.captured;
        total.disc_hits += s.disc_hits; total.sun_hits += s.sun_hits; total.star_hits += s.star_hits;
        total.jet_rays += s.jet_rays; total.escaped += s.escaped; total.exhausted += s.exhausted;
        total.total_flux += s.total_flux;
        total.max_norm_error = std::max(total.max_norm_error, s.max_norm_error);
        total.max_carter_drift = std::max(total.max_carter_drift, s.max_carter_drift);
    }
    total.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    stats_out(total, st);
    return BH_OK;
}

}  // extern "C"

namespace {

// The samples of pixel (x, y) through the reference's trace() and shade():
// per-sample results into out[0 .. S^2), counters and flux into `local`.
void trace_pixel(const Scene& sc, int x, int y, bh::RenderStats& local, bh_ray_result* out) {
    const bh::RenderConfig& cfg = sc.cfg;
    const int S = std::max(1, cfg.sqrt_spp);
    const double inv_S = 1.0 / S;
    size_t idx = 0;
    bh::Rng rng(cfg.seed ^ (static_cast<uint64_t>(y) << 32) ^
                (static_cast<uint64_t>(x) * 0x9E3779B97F4A7C15ull));
    spec::XYZ acc{};
    for (int sy = 0; sy < S; ++sy)
        for (int sx = 0; sx < S; ++sx) {
            const double jx = (sx + rng.uniform()) * inv_S;
            const double jy = (sy + rng.uniform()) * inv_S;
            const double u = (2.0 * (x + jx) / cfg.width - 1.0);
            const double v = (1.0 - 2.0 * (y + jy) / cfg.height);
            double dir[3];
            cfg.cam.ray_direction(u, v, sc.aspect, dir);
            ++local.rays;
            bh::RenderStats rs;   // this ray's own counters and drift maxima
            const bh::Hit hit = bh::trace(cfg, sc.disc.get(), dir, sc.tet, rs);
            local.steps += rs.steps;
            local.max_norm_error = std::max(local.max_norm_error, rs.max_norm_error);
            local.max_carter_drift = std::max(local.max_carter_drift, rs.max_carter_drift);
            const spec::XYZ col = bh::shade(cfg, sc.disc.get(), sc.stars.get(), hit,
                                            sc.psf_sigma, sc.jet_colour, local);
            acc.x += col.x; acc.y += col.y; acc.z += col.z;
            bh_ray_result& o = out[idx++];
            std::memset(&o, 0, sizeof o);
            o.what = static_cast<int32_t>(hit.what);
            o.steps = static_cast<int32_t>(rs.steps);
            o.max_norm = rs.max_norm_error;
            o.max_q = rs.max_carter_drift;
            o.jet = hit.jet;
            for (int i = 0; i < 8; ++i) o.y[i] = hit.y[i];
            o.xyz.x = col.x; o.xyz.y = col.y; o.xyz.z = col.z;
            // The fields shade_hit computes on the way (render.cpp:275-325).
            if (hit.what == bh::Hit::What::Disc && sc.disc) {
                const double r = hit.y[bh::Y_R];
                if (sc.disc->temperature(r) > 0.0) {
                    const double g = bh::redshift_factor(hit.y, sc.disc->four_velocity(r));
                    o.g = (g > 0.0) ? g : 0.0;
                }
            } else if (hit.what == bh::Hit::What::Sky) {
                const bh::State d = bh::geodesic_rhs(cfg.spin, hit.y);
                double v3[3];
                bh::cartesian_velocity(cfg.spin, hit.y, d, v3);
                const double vn = std::sqrt(v3[0] * v3[0] + v3[1] * v3[1] + v3[2] * v3[2]);
                if (vn > 0.0)
                    for (int i = 0; i < 3; ++i) o.dir[i] = v3[i] / vn;
            } else if (hit.what == bh::Hit::What::Sun) {
                const bh::Geom gm = bh::geom_at(cfg.spin, hit.y[bh::Y_R], hit.y[bh::Y_TH]);
                const bh::MetricLower ml = bh::metric_lower(gm);
                if (ml.tt < 0.0) {
                    const std::array<double, 4> u = {1.0 / std::sqrt(-ml.tt), 0.0, 0.0, 0.0};
                    const double g = bh::redshift_factor(hit.y, u);
                    o.g = (g > 0.0) ? g : 0.0;
                }
            } else if (hit.what == bh::Hit::What::Star) {
                const auto u = cfg.star.surface_four_velocity(hit.y[bh::Y_TH]);
                const double ku = hit.y[bh::Y_PT] * u[0] + hit.y[bh::Y_PPH] * u[3];
                if (ku > 1e-12) o.g = 1.0 / ku;
            }
        }
    const double w = 1.0 / (S * S);
    local.total_flux += acc.y * w;
}

void add_stats(bh::RenderStats& total, const bh::RenderStats& s) {
    total.rays += s.rays; total.steps += s.steps; total.captured += s.captured;
    total.disc_hits += s.disc_hits; total.sun_hits += s.sun_hits; total.star_hits += s.star_hits;
    total.jet_rays += s.jet_rays; total.escaped += s.escaped; total.exhausted += s.exhausted;
    total.total_flux += s.total_flux;
    total.max_norm_error = std::max(total.max_norm_error, s.max_norm_error);
    total.max_carter_drift = std::max(total.max_carter_drift, s.max_carter_drift);
}

}  // namespace

extern "C" {

// Per-sample trace()/shade() results of a pixel window, single-threaded.
int ref_trace_rays(const bh_render_config* c, int x0, int y0, int w, int h, bh_ray_result* out,
                   bh_render_stats* st) {
    const int rc = check_cfg(c);
    if (rc != BH_OK) return rc;
    if (x0 < 0 || y0 < 0 || w < 0 || h < 0 || x0 + w > c->width || y0 + h > c->height)
        return BH_ERR_INVALID_ARG;
    Scene sc(*c, c->milky_way != 0);
    bh::RenderStats local;
    const int S = std::max(1, sc.cfg.sqrt_spp);
    size_t idx = 0;
    for (int y = y0; y < y0 + h; ++y)
        for (int x = x0; x < x0 + w; ++x) {
            trace_pixel(sc, x, y, local, out + idx);
            idx += static_cast<size_t>(S) * S;
        }
    stats_out(local, st);
    return BH_OK;
}

// Per-sample results of whole rows on `threads` workers pulling rows from an
// atomic counter, as render() shares rows out (render.cpp:420-477): sample s
// of pixel x of the k-th listed row at out[(k * width + x) * S^2 + s].
int ref_trace_rows(const bh_render_config* c, const int* rows, int nrows, int threads, bh_ray_result* out,
                   bh_render_stats* st) {
    const int rc = check_cfg(c);
    if (rc != BH_OK) return rc;
    if (nrows < 0 || (nrows > 0 && (!rows || !out))) return BH_ERR_INVALID_ARG;
    for (int k = 0; k < nrows; ++k)
        if (rows[k] < 0 || rows[k] >= c->height) return BH_ERR_INVALID_ARG;
    Scene sc(*c, c->milky_way != 0);
    (void)spec::blackbody_xyz(5000.0);  // the magic-static table, before the workers
    int nthreads = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
    if (nthreads <= 0) nthreads = 1;
    const int S = std::max(1, sc.cfg.sqrt_spp);
    std::atomic<int> next{0};
    std::vector<bh::RenderStats> per_thread(nthreads);
    auto worker = [&](int tid) {
        for (;;) {
            const int k = next.fetch_add(1);
            if (k >= nrows) break;
            for (int x = 0; x < sc.cfg.width; ++x)
                trace_pixel(sc, x, rows[k], per_thread[tid],
                            out + (static_cast<size_t>(k) * sc.cfg.width + x) * S * S);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker, t);
    for (auto& th : pool) th.join();
    bh::RenderStats total;
    for (const auto& s : per_thread) add_stats(total, s);
    stats_out(total, st);
    return BH_OK;
}

// ---- known-answer quantities (validate.cpp sections 1, 3, 4, 6, 7) --------

void ref_metric_upper_deriv(double a, double r, double th, double out15[15]) {
    const bh::MetricUpperDeriv d = bh::metric_upper_deriv(a, r, th);
    const bh::MetricUpper* m[3] = {&d.g, &d.dr, &d.dth};
    for (int k = 0; k < 3; ++k) {
        out15[5 * k + 0] = m[k]->tt;
        out15[5 * k + 1] = m[k]->tp;
        out15[5 * k + 2] = m[k]->rr;
        out15[5 * k + 3] = m[k]->thth;
        out15[5 * k + 4] = m[k]->pp;
    }
}
void ref_metric_lower(double a, double r, double th, double out5[5]) {
    const bh::MetricLower m = bh::metric_lower(a, r, th);
    out5[0] = m.tt; out5[1] = m.tp; out5[2] = m.rr; out5[3] = m.thth; out5[4] = m.pp;
}
void ref_geodesic_rhs(double a, const double y[8], double dy[8]) {
    bh::State s;
    for (int i = 0; i < 8; ++i) s[i] = y[i];
    const bh::State d = bh::geodesic_rhs(a, s);
    for (int i = 0; i < 8; ++i) dy[i] = d[i];
}
double ref_isco_radius(double a, int sigma) { return bh::isco_radius(a, sigma); }
double ref_photon_circular_orbit(double a, int sigma) { return bh::photon_circular_orbit(a, sigma); }
double ref_disc_efficiency(double a, int sigma) { return bh::disc_efficiency(a, sigma); }
double ref_horizon_outer(double a) { return bh::horizon_outer(a); }
double ref_page_thorne_W(double a, double r, double r_isco) { return bh::page_thorne_W(a, r, r_isco); }
double ref_disc_temperature(double M_kg, double spin, double r_out, double eddington, int sense,
                            double r) {
    const bh::NovikovThorneDisc d(M_kg, spin, r_out, eddington, sense);
    return d.temperature(r);
}
void ref_blackbody_xyz(double T, double out3[3]) {
    const spec::XYZ c = spec::blackbody_xyz(T);
    out3[0] = c.x; out3[1] = c.y; out3[2] = c.z;
}
void ref_blackbody_xyz_exact(double T, double out3[3]) {
    const spec::XYZ c = spec::blackbody_xyz_exact(T);
    out3[0] = c.x; out3[1] = c.y; out3[2] = c.z;
}
void ref_make_photon(double a, double r, double th, double phi, const double dir[3], double y[8]) {
    const bh::Geom g = bh::geom_at(a, r, th);
    const bh::Tetrad tet = bh::zamo_tetrad(g);
    const bh::State s = bh::make_photon(a, r, th, phi, tet, dir, true);
    for (int i = 0; i < 8; ++i) y[i] = s[i];
}
void ref_invariants(double a, const double y[8], double out5[5]) {
    bh::State s;
    for (int i = 0; i < 8; ++i) s[i] = y[i];
    const bh::Invariants iv = bh::invariants(a, s);
    out5[0] = iv.E; out5[1] = iv.Lz; out5[2] = iv.Q; out5[3] = iv.norm; out5[4] = iv.norm_rel;
}
// The star catalogue exactly as StarField builds it (scene.h:62-107).
int ref_star_catalogue(int count, uint64_t seed, double* out6) {
    if (count < 0 || !out6) return BH_ERR_INVALID_ARG;
    const bh::StarField sf(count, seed, true);
    for (int i = 0; i < count; ++i) {
        const auto& s = sf.stars_[static_cast<size_t>(i)];
        double* o = out6 + 6 * static_cast<size_t>(i);
        o[0] = s.x; o[1] = s.y; o[2] = s.z; o[3] = s.mag; o[4] = s.temperature; o[5] = s.irradiance;
    }
    return BH_OK;
}
int ref_sky_radiance(int count, uint64_t seed, int milky_way, const double* dirs, int n, double sigma,
                     double* out3) {
    const bh::StarField sf(count, seed, milky_way != 0);
    for (int i = 0; i < n; ++i) {
        const spec::XYZ c = sf.radiance(dirs + 3 * static_cast<size_t>(i), sigma);
        out3[3 * i] = c.x; out3[3 * i + 1] = c.y; out3[3 * i + 2] = c.z;
    }
    return BH_OK;
}

// Jets: Jet::configure, the power-law colour, the shape and the four-velocity.
namespace {
bh::Jet jet_of(const bh_jet& j) {
    bh::Jet o;
    o.z_base = j.z_base; o.z_top = j.z_top; o.R_base = j.R_base; o.k = j.k;
    o.gamma_max = j.gamma_max; o.z_sat = j.z_sat; o.alpha = j.alpha;
    o.u_peak = j.u_peak; o.u_wid = j.u_wid; o.spine = j.spine; o.spine_wid = j.spine_wid;
    o.zeta = j.zeta; o.eps_rad = j.eps_rad; o.phi_flux = j.phi_flux;
    o.a = j.a; o.Omega_F = j.Omega_F; o.P_jet = j.P_jet; o.L_rad = j.L_rad; o.j_nu0 = j.j_nu0;
    o.r_bound = j.r_bound; o.volume_rg3 = j.volume_rg3;
    return o;
}
}  // namespace

void ref_jet_configure(bh_jet* jet, double spin, double mdot_c2, double r_g_m) {
    bh::Jet j = jet_of(*jet);
    j.configure(spin, mdot_c2, r_g_m);
    jet->a = j.a; jet->Omega_F = j.Omega_F; jet->P_jet = j.P_jet; jet->L_rad = j.L_rad;
    jet->j_nu0 = j.j_nu0; jet->r_bound = j.r_bound; jet->volume_rg3 = j.volume_rg3;
}
void ref_powerlaw_xyz(double alpha, double out3[3]) {
    const spec::XYZ c = spec::powerlaw_xyz(alpha);
    out3[0] = c.x; out3[1] = c.y; out3[2] = c.z;
}
double ref_jet_shape(const bh_jet* jet, double z, double rho) { return jet_of(*jet).shape(z, rho); }
void ref_jet_four_velocity(const bh_jet* jet, double a, double r, double th, double out4[4]) {
    const auto u = jet_of(*jet).four_velocity(bh::geom_at(a, r, th));
    for (int i = 0; i < 4; ++i) out4[i] = u[i];
}

// The display transform (image.cpp:22-191), through the reference's own img::.
namespace {
img::Image to_image(const bh_xyz* px, int w, int h) {
    img::Image im(w, h);
    for (size_t i = 0; i < im.pixels.size(); ++i) im.pixels[i] = {px[i].x, px[i].y, px[i].z};
    return im;
}
}  // namespace

double ref_auto_exposure(const bh_xyz* px, int w, int h, double key) {
    return img::auto_exposure(to_image(px, w, h), key);
}
void ref_add_glare(bh_xyz* px, int w, int h, double strength, double radius_px) {
    img::Image im = to_image(px, w, h);
    img::add_glare(im, strength, radius_px);
    for (size_t i = 0; i < im.pixels.size(); ++i) px[i] = {im.pixels[i].x, im.pixels[i].y, im.pixels[i].z};
}
void ref_develop(const bh_xyz* px, int w, int h, double exposure, int tonemap, double log_decades,
                 uint8_t* out) {
    const std::vector<uint8_t> rgb =
        img::develop(to_image(px, w, h), exposure, static_cast<img::ToneMap>(tonemap), log_decades);
    std::memcpy(out, rgb.data(), rgb.size());
}

}  // extern "C"
