// render_gpu.cpp - bh::render_gpu: the reference's render() surface over the
// C-ABI of libbh_gpu.so.  See render_gpu.h.
#include "render_gpu.h"

#include <algorithm>
#include <cstddef>
#include <type_traits>

namespace bh {

// The copy below names every field of the reference's RenderConfig as it is
// (render.h:15-53 and the structs it holds): a field renamed or removed there
// stops this file compiling, and one added changes the struct's size, which
// these asserts catch (x86-64 System V layout of the structs as of
// render.h:15-53, scene.h:232-236/306-313/343-351, neutronstar.h:43-70,
// jet.h:96-146).
static_assert(std::is_trivially_copyable<RenderConfig>::value, "RenderConfig is plain data");
static_assert(sizeof(RenderConfig) == 560, "bh::RenderConfig changed: update gpu_config()");
static_assert(sizeof(Jet) == 176, "bh::Jet changed: update gpu_config()");
static_assert(sizeof(NeutronStar) == 104, "bh::NeutronStar changed: update gpu_config()");
static_assert(sizeof(HotSpot) == 56, "bh::HotSpot changed: update gpu_config()");
static_assert(sizeof(Camera) == 7 * sizeof(double), "bh::Camera changed: update gpu_config()");
static_assert(sizeof(RenderStats) == 104, "bh::RenderStats changed: update render_gpu()");
// img::Image's pixels are written in place as bh_xyz.
static_assert(sizeof(spec::XYZ) == sizeof(bh_xyz), "spec::XYZ and bh_xyz differ");
static_assert(offsetof(spec::XYZ, y) == offsetof(bh_xyz, y) && offsetof(spec::XYZ, z) == offsetof(bh_xyz, z),
              "spec::XYZ and bh_xyz differ");

bh_render_config gpu_config(const RenderConfig& c, int precision) {
    bh_render_config g;
    bh_render_config_default(&g);
    g.M_kg = c.M_kg;
    g.spin = c.spin;
    g.cam.r = c.cam.r;
    g.cam.theta = c.cam.theta;
    g.cam.phi = c.cam.phi;
    g.cam.fov = c.cam.fov;
    g.cam.yaw = c.cam.yaw;
    g.cam.pitch = c.cam.pitch;
    g.cam.roll = c.cam.roll;
    g.width = c.width;
    g.height = c.height;
    g.sqrt_spp = c.sqrt_spp;
    g.disc_enabled = c.disc_enabled ? 1 : 0;
    g.disc_r_out = c.disc_r_out;
    g.eddington = c.eddington;
    g.disc_sense = c.disc_sense;
    g.stars_enabled = c.stars_enabled ? 1 : 0;
    g.star_count = c.star_count;
    g.seed = c.seed;
    g.sun_enabled = c.sun_enabled ? 1 : 0;
    for (int i = 0; i < 3; ++i) g.sun.centre[i] = c.sun.centre[i];
    g.sun.radius = c.sun.radius;
    g.sun.T_eff = c.sun.T_eff;
    g.hotspot.enabled = c.hotspot.enabled ? 1 : 0;
    g.hotspot.sense = c.hotspot.sense;
    g.hotspot.r = c.hotspot.r;
    g.hotspot.phi0 = c.hotspot.phi0;
    g.hotspot.sigma = c.hotspot.sigma;
    g.hotspot.contrast = c.hotspot.contrast;
    g.hotspot.omega = c.hotspot.omega;
    g.star.enabled = c.star.enabled ? 1 : 0;
    g.star.caps = c.star.caps ? 1 : 0;
    g.star.M_kg = c.star.M_kg;
    g.star.R_m = c.star.R_m;
    g.star.R = c.star.R;
    g.star.T_eff = c.star.T_eff;
    g.star.spin_hz = c.star.spin_hz;
    g.star.Omega = c.star.Omega;
    g.star.cap_tilt = c.star.cap_tilt;
    g.star.cap_radius = c.star.cap_radius;
    g.star.cap_T = c.star.cap_T;
    g.star.cap_phase0 = c.star.cap_phase0;
    g.star.two_caps = c.star.two_caps ? 1 : 0;
    g.jet_enabled = c.jet.enabled ? 1 : 0;   // the jet as main.cpp configured it
    g.jet.z_base = c.jet.z_base;
    g.jet.z_top = c.jet.z_top;
    g.jet.R_base = c.jet.R_base;
    g.jet.k = c.jet.k;
    g.jet.gamma_max = c.jet.gamma_max;
    g.jet.z_sat = c.jet.z_sat;
    g.jet.alpha = c.jet.alpha;
    g.jet.u_peak = c.jet.u_peak;
    g.jet.u_wid = c.jet.u_wid;
    g.jet.spine = c.jet.spine;
    g.jet.spine_wid = c.jet.spine_wid;
    g.jet.zeta = c.jet.zeta;
    g.jet.eps_rad = c.jet.eps_rad;
    g.jet.phi_flux = c.jet.phi_flux;
    g.jet.a = c.jet.a;
    g.jet.Omega_F = c.jet.Omega_F;
    g.jet.P_jet = c.jet.P_jet;
    g.jet.L_rad = c.jet.L_rad;
    g.jet.j_nu0 = c.jet.j_nu0;
    g.jet.r_bound = c.jet.r_bound;
    g.jet.volume_rg3 = c.jet.volume_rg3;
    g.observer_time = c.observer_time;
    g.rtol = c.rtol;
    g.atol = c.atol;
    g.r_escape = c.r_escape;
    g.max_steps = c.max_steps;
    g.threads = c.threads;
    g.quiet = c.quiet ? 1 : 0;
    g.precision = precision;
    return g;
}

namespace {

struct ThreadContext {
    bh_ctx* ctx = nullptr;
    ~ThreadContext() {
        if (ctx) bh_gpu_destroy(ctx);
    }
};

thread_local ThreadContext t_ctx;

bh_ctx* context() {
    if (!t_ctx.ctx) {
        const int rc = bh_gpu_create(0, &t_ctx.ctx);
        if (rc != BH_OK) {
            t_ctx.ctx = nullptr;
            throw GpuError(rc, "bh_gpu_create: no usable sm_100 GPU (status " + std::to_string(rc) + ")");
        }
    }
    return t_ctx.ctx;
}

}  // namespace

img::Image render_gpu(const RenderConfig& cfg, RenderStats& stats, int precision) {
    const bh_render_config g = gpu_config(cfg, precision);
    bh_ctx* ctx = context();
    img::Image im(std::max(cfg.width, 0), std::max(cfg.height, 0));
    bh_render_stats s{};
    const int rc = bh_gpu_render(ctx, &g, reinterpret_cast<bh_xyz*>(im.pixels.data()), &s);
    if (rc != BH_OK) throw GpuError(rc, bh_gpu_last_error(ctx));
    // render.cpp:481-495: counters and flux added, drifts maximised, the
    // time overwritten.
    stats.rays += s.rays;
    stats.steps += s.steps;
    stats.captured += s.captured;
    stats.disc_hits += s.disc_hits;
    stats.sun_hits += s.sun_hits;
    stats.star_hits += s.star_hits;
    stats.jet_rays += s.jet_rays;
    stats.escaped += s.escaped;
    stats.exhausted += s.exhausted;
    stats.total_flux += s.total_flux;
    stats.max_norm_error = std::max(stats.max_norm_error, s.max_norm_error);
    stats.max_carter_drift = std::max(stats.max_carter_drift, s.max_carter_drift);
    stats.seconds = s.seconds;
    return im;
}

void release_gpu() {
    if (t_ctx.ctx) {
        bh_gpu_destroy(t_ctx.ctx);
        t_ctx.ctx = nullptr;
    }
}

}  // namespace bh
