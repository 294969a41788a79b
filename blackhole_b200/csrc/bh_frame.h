// bh_frame.h - Per-frame and per-scene parameters shared by host and device.
//
// FrameParams holds everything the trace and shade kernels need for one frame,
// precomputed on the host once per frame (the work render() does before its
// pixel loop, render.cpp:396-418).  A batch launch reads an array of them.
#pragma once

#include <cstdint>

namespace bhg {

constexpr int kTableN = 4096;        // blackbody table entries (spectrum.cpp:97)
constexpr int kLat = 360;            // star bins in theta (scene.h:63)
constexpr int kLon = 720;            // star bins in phi

struct FrameParams {
    // ---- spacetime and integration ------------------------------------
    double a, a2;
    double r_plus, r_minus;          // horizons (kerr.h:187-194); r_minus used when a2 < 1
    double r_h;                      // r_plus, the hmax reference (render.cpp:72)
    double r_stop;                   // horizon stop radius
    double r_escape;
    double rtol, atol;               // tolerances of this frame's precision
    double h0;                       // first trial step, 0.02 max(1, r_cam) (render.cpp:86)
    double hmax_a, hmax_b;           // step cap hmax_a max(1, r - r_h) + hmax_b (render.cpp:130-131)
    double rtol_ref, atol_ref;       // the binary64 path's tolerances (the config's rtol, atol)
    double r_promote;                // innermost photon orbit: an ingoing ray below it is falling in
    double land_limit, land_target;  // mixed: a step from inside r_escape that would end beyond land_limit
                                     // is shortened to end near land_target (see land_escape)
    // binary32 copies of the constants the mixed kernel's step control reads
    // every attempt (no conversion in the step loop)
    float f_hmax_a, f_hmax_b, f_r_h, f_atol, f_rtol;
    float f_land_limit, f_r_stop, f_r_escape, f_r_promote, f_pad;
    int32_t early_capture;           // mixed: end such a ray as captured there
    int32_t mirror_ok;               // mixed: integrate th > pi/2 as its mirror pi - th
    int32_t fp64_near_critical;      // mixed: near-critical rays traced in binary64
    int32_t max_steps;
    int32_t factored_delta;          // Delta = (r - r+)(r - r-) when a^2 < 1

    // ---- camera (scene.h:356-384) and photon set-up (geodesic.h:215-231) ----
    double cam_r, cam_th, cam_ph;
    double tanf, aspect;
    double cr, sr, cp, sp, cy, sy;
    int32_t has_roll;
    int32_t S;                       // sqrt_spp
    double inv_S, inv_SS;
    double tet00, tet03, tet11, tet22, tet33;     // ZAMO tetrad, non-zero legs
    double cam_sn2, cam_cs2;         // sin^2, cos^2 of the camera theta as carter_constant clamps them
    double ml_tt, ml_tp, ml_rr, ml_thth, ml_pp;   // g_{mu nu} at the camera
    uint64_t seed;
    int32_t width, height;
    long long ray_begin;             // first global ray id of this frame
    long long n_rays;                // width * height * S^2
    long long pixel_begin;           // first pixel of this frame in the batch pixel buffer

    // ---- Novikov-Thorne disc (disc.h) -----------------------------------
    int32_t disc_enabled;
    int32_t disc_sigma;
    double disc_a;                   // spin clamped to +-0.9999 (disc.h:75)
    double r_in, r_out;
    double x0;                       // sqrt(r_in)
    double pt_x[3];                  // roots x1, x2, x3 of x^3 - 3x + 2a (disc.h:50-52)
    double pt_c[3];                  // 3 (xi-a)^2 / (xi (xi-xj)(xi-xk)), 0 where |xi| < 1e-13
    double pt_den[3];                // x0 - xi
    double disc_mdot;                // kg/s (disc.h:79)
    double disc_eta;                 // radiative efficiency 1 - E(r_isco) (disc.h:77-78)
    double disc_rg2;                 // r_g^2 in m^2 (disc.h:96)

    // ---- sky ------------------------------------------------------------
    int32_t stars_enabled;
    int32_t milky_way;
    int32_t sky_mode;
    int32_t pad0;
    double psf_sigma;                // 0.55 fov / width (render.cpp:413-414)
    double cutoff, inv2s2, psf_norm; // scene.h:114-118
    double cut_dot;                  // cos(1.000001 cutoff): a star with d.s below it is outside the cutoff
    int32_t span_t;                  // scene.h:124
    int32_t pad1;

    // ---- surfaces -------------------------------------------------------
    int32_t sun_enabled;
    int32_t ns_enabled;
    double sun_c[3], sun_R, sun_R2, sun_T_eff, sun_redshift_div;
    double ns_R, ns_T_eff, ns_Omega, ns_cap_tilt, ns_cap_radius, ns_cap_T, ns_cap_phase0;
    int32_t ns_caps, ns_two_caps;

    // ---- hot spot (scene.h:306-335) ---------------------------------------
    int32_t hs_enabled;
    int32_t pad2;
    double hs_r, hs_phi0, hs_sigma, hs_contrast, hs_omega;
    double observer_time;
    int32_t precision_tag;           // BH_PRECISION_* of the launch
    int32_t land_escape;             // mixed: land the escaping step within the reference's cap of r_escape

    // ---- jet (jet.h:96-315; sampled per step, render.cpp:107-122) ------------
    int32_t jet_enabled;
    int32_t pad4;
    double jet_z_base, jet_z_top, jet_R_base, jet_k, jet_gamma_max, jet_z_sat;
    double jet_alpha, jet_u_peak, jet_u_wid, jet_spine, jet_spine_wid, jet_zeta;
    double jet_Omega_F, jet_j_nu0, jet_r_bound;
    double jet_col[3];               // powerlaw_xyz(alpha) (spectrum.cpp:77-92)
};

// Read-only sky data shared by all frames of a launch.
struct SkyData {
    const double4* star_pos;         // x, y, z, irradiance; sorted by bin (CSR order)
    const double4* star_col;         // blackbody_xyz(T): x, z, 1/y (or 0), unused
    const int32_t* bin_start;        // kLat*kLon + 1 offsets
    const double* table;             // ln X, ln Y, ln Z, each kTableN entries
    double mw_x, mw_z, mw_inv;       // blackbody_xyz(4800 K): x, z, 1/y
    double diffuse_L;                // 21.5 mag/arcsec^2 in W m^-2 sr^-1
    int32_t n_stars;
    int32_t pad;
};

// Trace result of one ray (written once when the ray terminates).
struct HitRecord {
    double y[8];
    double max_norm;                 // worst |norm_rel| along the ray
    double max_q;                    // worst Carter drift along the ray
    int32_t what;
    int32_t steps;
    int32_t attempts;
    int32_t pad;
};

// Per-frame reduction target (device side), reduced into bh_render_stats.
struct FrameStats {
    unsigned long long rays, steps, attempts;
    unsigned long long captured, disc_hits, sun_hits, star_hits, escaped, exhausted, jet_rays;
    unsigned long long max_norm_bits, max_q_bits;   // non-negative doubles as ordered bits
    double total_flux;
};

// Work-queue state of one launch.
struct QueueState {
    unsigned long long next;         // next unclaimed global ray id
    unsigned long long attempts;     // step attempts of finished rays
    unsigned long long budget;       // 0 = none
    unsigned long long deferred;     // rays handed from binary32 to binary64
    unsigned long long resume_next;  // next unclaimed deferred ray
    unsigned long long select_next;  // next near-critical ray the binary64 kernel takes (list or scan)
    unsigned long long selected;     // near-critical rays the classification pass listed
    unsigned long long select_next2; // next listed ray of the binary64 pass after the binary32 kernels
    int32_t abort;                   // set by the host (1) or by the budget check (2)
    int32_t status;
};

}  // namespace bhg
