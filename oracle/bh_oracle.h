/*
 * bh_oracle.h - CPU oracle of the per-pixel geodesic render path.
 *
 * TEST INFRASTRUCTURE.  This is a plain-C FP64 restatement of the reference
 * renderer's algorithm (kerr.h, geodesic.h, disc.h, scene.h, spectrum.cpp,
 * render.cpp), used only by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline leg of bench.py, as the checker.  It is never linked into, or
 * called by, the GPU library.
 *
 * The same entry points with the prefix ref_ exist in oracle/_ref/libbh_ref.so,
 * built from the reference sources themselves; tests pin this restatement
 * against those bit for bit.
 */
#ifndef BH_ORACLE_H
#define BH_ORACLE_H

#include "../include/bh_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Kerr geometry (kerr.h). out5 = {tt, tp, rr, thth, pp}. */
void   orc_metric_upper(double a, double r, double th, double out5[5]);
void   orc_metric_lower(double a, double r, double th, double out5[5]);
/* out15 = {g[5], d_r g[5], d_th g[5]} */
void   orc_metric_upper_deriv(double a, double r, double th, double out15[15]);
double orc_horizon_outer(double a);
double orc_horizon_inner(double a);
double orc_isco_radius(double a, int sigma);
double orc_photon_circular_orbit(double a, int sigma);
double orc_circular_energy(double a, double r, int sigma);
double orc_circular_angmom(double a, double r, int sigma);
double orc_disc_efficiency(double a, int sigma);
void   orc_keplerian_four_velocity(double a, double r, int sigma, double out4[4]);
void   orc_zamo_tetrad(double a, double r, double th, double out16[16]);
double orc_carter_constant(double a, double th, double p_th, double E, double Lz);

/* Geodesics (geodesic.h). */
void   orc_geodesic_rhs(double a, const double y[8], double dy[8]);
void   orc_make_photon(double a, double r, double th, double phi, const double dir[3],
                       double y_out[8]);
/* out5 = {E, Lz, Q, norm, norm_rel} */
void   orc_invariants(double a, const double y[8], double out5[5]);
/* Integrate with the DP5(4) stepper until r < r_in or r > r_out or max_steps;
   returns accepted steps, writes the final state. */
long   orc_integrate(double a, const double y0[8], double h0, double rtol, double atol,
                     int max_steps, double r_in, double r_out, double y_out[8]);

/* Disc (disc.h). */
double orc_page_thorne_W(double a, double r, double r_isco);
double orc_disc_temperature(double M_kg, double spin, double r_out, double eddington,
                            int sense, double r);

/* Spectrum (spectrum.cpp). */
double orc_planck_radiance(double lambda_m, double T);
void   orc_blackbody_xyz_exact(double T, double out3[3]);
void   orc_blackbody_xyz(double T, double out3[3]);
double orc_bv_to_temperature(double bv);
/* ln X, ln Y, ln Z of the 4096-entry table (spectrum.cpp:101-121). */
void   orc_blackbody_table(double* out);

/* Star catalogue: out6 per star = {x, y, z, mag, T, irradiance}. */
int    orc_star_catalogue(int count, uint64_t seed, int sky_mode, double* out6);
/* Sky radiance along a unit direction (stars + diffuse) for a catalogue. */
int    orc_sky_radiance(int count, uint64_t seed, int sky_mode, int milky_way,
                        const double* dirs, int n, double sigma, double* out3);

/* Camera (scene.h:356-384). */
void   orc_ray_direction(const bh_camera* cam, double sx, double sy, double aspect,
                         double out3[3]);

/* The render path (render.cpp).  Per-sample results of the pixel window
   [x0, x0+w) x [y0, y0+h), ordered by pixel then sample, as bh_gpu_trace_rays. */
int    orc_trace_rays(const bh_render_config* cfg, int x0, int y0, int w, int h,
                      bh_ray_result* out, bh_render_stats* stats);
/* Per-sample results of whole rows (rows[0..nrows)) on `threads` workers:
   sample s of pixel x of the k-th listed row at out[(k * width + x) * S^2 + s]. */
int    orc_trace_rows(const bh_render_config* cfg, const int* rows, int nrows, int threads,
                      bh_ray_result* out, bh_render_stats* stats);
/* Pixels of the same window (w*h, row-major).  stats are added into. */
int    orc_render_window(const bh_render_config* cfg, int x0, int y0, int w, int h,
                         bh_xyz* out, bh_render_stats* stats);

/* Jets (jet.h:77-315, spectrum.cpp:77-92). */
void   orc_jet_configure(bh_jet* jet, double spin, double mdot_c2, double r_g_m);
void   orc_powerlaw_xyz(double alpha, double out3[3]);
double orc_jet_shape(const bh_jet* jet, double z, double rho);
void   orc_jet_four_velocity(const bh_jet* jet, double a, double r, double th, double out4[4]);

/* Display transform (image.cpp:22-191).  tonemap: 0 Linear, 1 Reinhard,
   2 ACES, 3 Log, 4 HDR (img::ToneMap order). */
double orc_auto_exposure(const bh_xyz* px, long n, double key);
void   orc_add_glare(bh_xyz* px, int w, int h, double strength, double radius_px);
void   orc_develop(const bh_xyz* px, long n, double exposure, int tonemap, double log_decades,
                   uint8_t* out);

#ifdef __cplusplus
}
#endif

#endif
