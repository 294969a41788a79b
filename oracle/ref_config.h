// ref_config.h - bh_render_config -> the reference's bh::RenderConfig.
//
// TEST INFRASTRUCTURE, shared by the harnesses that call the reference
// (ref_harness.cpp) and the drop-in adapter (adapter_check.cpp): every field
// the reference has (render.h:15-53, scene.h:232-236, 306-313, 343-351,
// neutronstar.h:43-70, jet.h:96-146), copied one for one.  Include after the
// reference's render.h.
#pragma once

namespace {

// force_quiet: the harnesses never print the reference's progress.
bh::RenderConfig to_ref(const bh_render_config& c, bool force_quiet = true) {
    bh::RenderConfig r;
    r.M_kg = c.M_kg;
    r.spin = c.spin;
    r.cam.r = c.cam.r;
    r.cam.theta = c.cam.theta;
    r.cam.phi = c.cam.phi;
    r.cam.fov = c.cam.fov;
    r.cam.yaw = c.cam.yaw;
    r.cam.pitch = c.cam.pitch;
    r.cam.roll = c.cam.roll;
    r.width = c.width;
    r.height = c.height;
    r.sqrt_spp = c.sqrt_spp;
    r.disc_enabled = c.disc_enabled != 0;
    r.disc_r_out = c.disc_r_out;
    r.eddington = c.eddington;
    r.disc_sense = c.disc_sense;
    r.stars_enabled = c.stars_enabled != 0;
    r.star_count = c.star_count;
    r.seed = c.seed;
    r.sun_enabled = c.sun_enabled != 0;
    for (int i = 0; i < 3; ++i) r.sun.centre[i] = c.sun.centre[i];
    r.sun.radius = c.sun.radius;
    r.sun.T_eff = c.sun.T_eff;
    r.hotspot.enabled = c.hotspot.enabled != 0;
    r.hotspot.r = c.hotspot.r;
    r.hotspot.phi0 = c.hotspot.phi0;
    r.hotspot.sigma = c.hotspot.sigma;
    r.hotspot.contrast = c.hotspot.contrast;
    r.hotspot.omega = c.hotspot.omega;
    r.hotspot.sense = c.hotspot.sense;
    r.star.enabled = c.star.enabled != 0;
    r.star.caps = c.star.caps != 0;
    r.star.M_kg = c.star.M_kg;
    r.star.R_m = c.star.R_m;
    r.star.R = c.star.R;
    r.star.T_eff = c.star.T_eff;
    r.star.spin_hz = c.star.spin_hz;
    r.star.Omega = c.star.Omega;
    r.star.cap_tilt = c.star.cap_tilt;
    r.star.cap_radius = c.star.cap_radius;
    r.star.cap_T = c.star.cap_T;
    r.star.cap_phase0 = c.star.cap_phase0;
    r.star.two_caps = c.star.two_caps != 0;
    r.jet.enabled = c.jet_enabled != 0;
    r.jet.z_base = c.jet.z_base;
    r.jet.z_top = c.jet.z_top;
    r.jet.R_base = c.jet.R_base;
    r.jet.k = c.jet.k;
    r.jet.gamma_max = c.jet.gamma_max;
    r.jet.z_sat = c.jet.z_sat;
    r.jet.alpha = c.jet.alpha;
    r.jet.u_peak = c.jet.u_peak;
    r.jet.u_wid = c.jet.u_wid;
    r.jet.spine = c.jet.spine;
    r.jet.spine_wid = c.jet.spine_wid;
    r.jet.zeta = c.jet.zeta;
    r.jet.eps_rad = c.jet.eps_rad;
    r.jet.phi_flux = c.jet.phi_flux;
    r.jet.a = c.jet.a;
    r.jet.Omega_F = c.jet.Omega_F;
    r.jet.P_jet = c.jet.P_jet;
    r.jet.L_rad = c.jet.L_rad;
    r.jet.j_nu0 = c.jet.j_nu0;
    r.jet.r_bound = c.jet.r_bound;
    r.jet.volume_rg3 = c.jet.volume_rg3;
    r.observer_time = c.observer_time;
    r.rtol = c.rtol;
    r.atol = c.atol;
    r.r_escape = c.r_escape;
    r.max_steps = c.max_steps;
    r.threads = c.threads;
    r.quiet = force_quiet || c.quiet != 0;
    return r;
}

}  // namespace
