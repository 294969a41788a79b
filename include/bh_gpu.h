/*
 * bh_gpu.h - C-ABI of the B200 geodesic render library (libbh_gpu.so).
 *
 * This is the drop-in boundary for the reference renderer's per-pixel loop:
 *
 *     img::Image bh::render(const RenderConfig& cfg, RenderStats& stats);   (render.h:72)
 *
 * The POD structs below mirror bh::RenderConfig (render.h:15-53), bh::Camera
 * (scene.h:343-351), bh::RenderStats (render.h:55-69) and the img::Image pixel
 * layout (image.h:18-27: row-major vector<spec::XYZ>, spec::XYZ = 3 doubles,
 * spectrum.h:23-25).  No C++ or CUDA types cross this boundary: plain pointers,
 * sizes and status codes only.
 *
 * Conventions
 *  - Every entry point that can fail returns 0 (BH_OK) or a negative bh_status.
 *    The message of the last failure on a context is bh_gpu_last_error().
 *  - Host buffers are owned by the caller.  A context owns its device memory
 *    (ray buffers, star catalogue, spectrum table) and reuses it across calls.
 *  - One context per host thread; a context drives one GPU.  Calls on one
 *    context are serialised by the caller (like a CUDA stream).
 *  - Stats follow bh::render: counters and the two drift maxima are ADDED
 *    into *stats (render.cpp:481-494); `seconds` is overwritten (render.cpp:495).
 *  - There is no CPU fallback: without a usable GPU, bh_gpu_create fails with
 *    BH_ERR_NO_DEVICE.
 */
#ifndef BH_GPU_H
#define BH_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BH_GPU_ABI_VERSION 3

/* Status codes. */
enum {
    BH_OK = 0,
    BH_ERR_INVALID_ARG = -1,   /* a config field or pointer is out of range        */
    BH_ERR_CUDA = -2,          /* a CUDA runtime call failed                       */
    BH_ERR_BUDGET = -3,        /* the per-launch step budget ran out               */
    BH_ERR_ABORTED = -4,       /* bh_gpu_request_abort() stopped the launch        */
    BH_ERR_NO_DEVICE = -5,     /* no CUDA device, or not an sm_100 part            */
    BH_ERR_UNSUPPORTED = -6,   /* a feature of the config that is not built        */
    BH_ERR_OUT_OF_MEMORY = -7  /* device allocation failed                         */
};

/* Termination class of a ray; same order as Hit::What (render.cpp:37). */
enum {
    BH_HIT_HORIZON = 0,
    BH_HIT_DISC = 1,
    BH_HIT_SUN = 2,
    BH_HIT_STAR = 3,      /* neutron-star surface */
    BH_HIT_SKY = 4,
    BH_HIT_EXHAUSTED = 5
};

/* Arithmetic of the integrator (extension; the reference is FP64 only). */
enum {
    BH_PRECISION_FP64 = 0,   /* every operation in IEEE binary64                   */
    BH_PRECISION_MIXED = 1   /* binary32 state and stages; binary64 for Delta and
                                Sigma, the error norm, accept/reject, h, root
                                refinement and the invariant diagnostics           */
};

/* Background sky (extension). */
enum {
    BH_SKY_GALACTIC = 0,     /* the reference catalogue: 45% galactic band, m <= 12,
                                normal B-V, plus the band-modulated Milky Way
                                (scene.h:62-107, 202-223)                          */
    BH_SKY_UNIFORM = 1       /* isotropic stars, m <= 6.5, B-V uniform in
                                [-0.3, 1.8], plus a uniform 21.5 mag/arcsec^2
                                background                                          */
};

/* Horizon stop radius (extension). */
enum {
    BH_STOP_REFERENCE = 0,   /* r_+ + 1e-4 + 1e-3 (r_+ - r_-)    (render.cpp:73)    */
    BH_STOP_RELATIVE = 1     /* r_+ (1 + stop_epsilon)                               */
};

/* The step-size limiter of the MIXED path.  The reference caps every step at
   hmax = 0.05 max(1, r - r_+) + 0.01 (render.cpp:130-131) on top of the error
   control; the binary64 path always does.
     BH_STEP_LIMIT_AUTO       the reference cap when the Sun, a neutron star
                              or a jet is in the scene (their hit tests and
                              the jet's quadrature sample each step), a looser
                              cap h <= 0.3 max(1, r - r_+) otherwise;
     BH_STEP_LIMIT_REFERENCE  the reference cap;
     BH_STEP_LIMIT_NONE       steps set by the error control alone.
   Without the reference cap, a step that leaves the escape sphere is
   shortened to end within the reference cap's step of r_escape, where the
   reference's last step ends. */
enum { BH_STEP_LIMIT_AUTO = 0, BH_STEP_LIMIT_REFERENCE = 1, BH_STEP_LIMIT_NONE = 2 };

/* How the MIXED path ends a ray that moves inwards inside the innermost
   circular photon orbit.  Such a photon has no radial turning point left
   (every turning point of a photon lies outside its spherical photon orbit,
   and the prograde equatorial one is the innermost), so it reaches the
   horizon; the disc lies outside the ISCO, further out still.
     BH_CAPTURE_AUTO       ended there as captured (BH_HIT_HORIZON, with the
                           state where it was ended) unless a neutron star or
                           a jet is in the scene (a surface or emission on the
                           way in); traced to the stop radius in binary64
                           otherwise;
     BH_CAPTURE_REFERENCE  always traced to the stop radius in binary64. */
enum { BH_CAPTURE_AUTO = 0, BH_CAPTURE_REFERENCE = 1 };

/* Which rays the MIXED path traces in binary64 from the start.  A photon whose
   radial potential R(r) = (r^2 + a^2 - a b)^2 - Delta (q + (b - a)^2) (b = L_z/E,
   q = Q/E^2) dips to just below zero at its minimum r* escapes after circling
   close to the photon shell, and every pass multiplies a change of its state
   by ~e^(2 pi): no binary32 state resolves where it leaves to.
     BH_NEAR_CRITICAL_AUTO      ingoing rays with -0.1 < R(r*)/r*^4 < 0 are
                                traced in binary64 under the binary64 path's
                                tolerances and step cap (their results are
                                the binary64 frame's), by a kernel that runs
                                beside the binary32 one;
     BH_NEAR_CRITICAL_BINARY32  every ray starts in binary32. */
enum { BH_NEAR_CRITICAL_AUTO = 0, BH_NEAR_CRITICAL_BINARY32 = 1 };

typedef struct bh_xyz {      /* spec::XYZ (spectrum.h:23-25), W m^-2 sr^-1 */
    double x, y, z;
} bh_xyz;

typedef struct bh_camera {   /* bh::Camera (scene.h:343-351) */
    double r, theta, phi;    /* Boyer-Lindquist position                    */
    double fov;              /* horizontal field of view, radians           */
    double yaw, pitch, roll;
} bh_camera;

typedef struct bh_sun {      /* bh::SunBody (scene.h:232-236) */
    double centre[3];        /* pseudo-Cartesian, gravitational radii */
    double radius;
    double T_eff;
} bh_sun;

typedef struct bh_hotspot {  /* bh::HotSpot (scene.h:306-313) */
    int32_t enabled;
    int32_t sense;
    double r, phi0, sigma, contrast, omega;
} bh_hotspot;

typedef struct bh_neutron_star {  /* bh::NeutronStar (neutronstar.h:43-70) */
    int32_t enabled;
    int32_t caps;
    double M_kg, R_m, R;     /* R in gravitational radii */
    double T_eff;
    double spin_hz, Omega;
    double cap_tilt, cap_radius, cap_T, cap_phase0;
    int32_t two_caps;
    int32_t reserved;
} bh_neutron_star;

/* bh::Jet (jet.h:96-315) without its `enabled` flag, which is
   bh_render_config.jet_enabled.  The first block is the prescribed model; the
   second is what Jet::configure (jet.h:262-312) sets from the spin and the
   accretion rate: fill it with bh_jet_configure or bh_render_config_setup_jet
   before rendering (a zero j_nu0 renders no jet). */
typedef struct bh_jet {
    double z_base, z_top, R_base, k;       /* geometry: R(z) = R_base (z / z_base)^k, GM/c^2  */
    double gamma_max, z_sat;               /* bulk Lorentz factor law                          */
    double alpha;                          /* synchrotron index, S_nu ~ nu^-alpha              */
    double u_peak, u_wid, spine, spine_wid;/* limb-brightened radial profile                   */
    double zeta;                           /* re-acceleration index                            */
    double eps_rad, phi_flux;              /* radiated fraction, horizon flux (MAD = 50)       */
    /* ---- set by configure ---- */
    double a, Omega_F, P_jet, L_rad, j_nu0, r_bound, volume_rg3;
} bh_jet;

/* bh::RenderConfig (render.h:15-53) plus the GPU extensions at the end. */
typedef struct bh_render_config {
    uint32_t struct_size;    /* sizeof(bh_render_config) as the caller compiled it */
    uint32_t abi_version;    /* BH_GPU_ABI_VERSION                                 */

    double M_kg;
    double spin;
    bh_camera cam;
    int32_t width, height;
    int32_t sqrt_spp;

    int32_t disc_enabled;
    double disc_r_out;
    double eddington;
    int32_t disc_sense;
    int32_t stars_enabled;
    int32_t star_count;
    int32_t sun_enabled;
    uint64_t seed;
    bh_sun sun;
    bh_hotspot hotspot;
    bh_neutron_star star;
    int32_t jet_enabled;     /* bh::Jet::enabled; the model is `jet` below */
    int32_t reserved0;

    double observer_time;

    double rtol, atol;
    double r_escape;
    int32_t max_steps;

    int32_t threads;         /* accepted and ignored (the GPU launch replaces the pool) */
    int32_t quiet;           /* accepted and ignored */

    /* ---- extensions ------------------------------------------------------ */
    int32_t precision;       /* BH_PRECISION_*                                   */
    int32_t sky_mode;        /* BH_SKY_*                                         */
    int32_t stop_mode;       /* BH_STOP_*                                        */
    int32_t milky_way;       /* diffuse background on (1) / off (0)              */
    double stop_epsilon;     /* BH_STOP_RELATIVE only                            */
    double mixed_rtol;       /* tolerances of the MIXED path; 0 = max(rtol, 1e-6) */
    double mixed_atol;       /*                               0 = max(atol, 1e-8) */
    bh_jet jet;              /* bh::RenderConfig::jet (render.h:37)              */
    int32_t mixed_step_limit;/* BH_STEP_LIMIT_* of the MIXED path (AUTO)           */
    int32_t mixed_capture;   /* BH_CAPTURE_* of the MIXED path (AUTO)              */
    int32_t mixed_near_critical; /* BH_NEAR_CRITICAL_* of the MIXED path (AUTO)    */
} bh_render_config;

/* bh::RenderStats (render.h:55-69) plus extensions. */
typedef struct bh_render_stats {
    long long rays;
    long long steps;         /* accepted integration steps */
    long long captured;
    long long disc_hits;
    long long sun_hits;
    long long star_hits;
    long long jet_rays;
    long long escaped;
    long long exhausted;
    double max_norm_error;   /* worst |g^ab p_a p_b| / sum |terms| along any ray */
    double max_carter_drift; /* worst |Q - Q0| / (|Q0| + 1e-12)                  */
    double seconds;
    double total_flux;       /* sum of pixel luminance Y                         */
    /* ---- extensions ---- */
    long long attempts;      /* step attempts, accepted + rejected               */
    double kernel_ms;        /* device time of the trace kernel                  */
    double shade_ms;         /* device time of the shade kernel                  */
    long long h2d_bytes;     /* host->device bytes the call copied               */
    long long d2h_bytes;     /* device->host bytes the call copied               */
} bh_render_stats;

/* Per-sample result, for parity checks (the fields trace() and shade() see). */
typedef struct bh_ray_result {
    int32_t what;            /* BH_HIT_*                                         */
    int32_t steps;           /* accepted steps of this ray                       */
    double y[8];             /* final state (t, r, th, phi, p_t, p_r, p_th, p_phi) */
    double g;                /* redshift factor of a disc hit, else 0           */
    double dir[3];           /* unit sky direction of an escaped ray, else 0    */
    bh_xyz xyz;              /* radiance of this sample                          */
    int32_t attempts;        /* step attempts (accepted + rejected)             */
    int32_t reserved;
    double max_norm;         /* worst relative null norm along the ray          */
    double max_q;            /* worst relative Carter drift along the ray       */
    double jet;              /* jet emission picked up, Hit::jet (render.cpp:41) */
} bh_ray_result;

/* Launch shape of the persistent trace kernel (the autotuner's search space). */
typedef struct bh_launch_params {
    int32_t block_size;      /* threads per block, multiple of 32, 64..512       */
    int32_t rays_per_thread; /* rays a lane takes per queue visit, 1..4          */
    int32_t refill;          /* lanes that must be idle before a warp refills   */
    int32_t blocks_per_sm;   /* 0 = as many as fit                              */
    int32_t reg_variant;     /* 1: tight register cap (more warps per SM),
                                2: wide cap (fewer spills)                      */
} bh_launch_params;

typedef struct bh_ctx bh_ctx;

int  bh_gpu_abi_version(void);

/* The reference's defaults (render.h:15-53, scene.h:343-351, jet.h:96-146) plus
   BH_PRECISION_FP64, BH_SKY_GALACTIC, BH_STOP_REFERENCE, milky_way = 1. */
void bh_render_config_default(bh_render_config* cfg);

/* Jet::configure (jet.h:262-312): Blandford-Znajek power of spin `spin` for
   an accretion flow of mdot_c2 watts around a hole of gravitational radius
   r_g_m metres, and the emissivity normalisation that radiates eps_rad of it. */
void bh_jet_configure(bh_jet* jet, double spin, double mdot_c2, double r_g_m);

/* The CLI's jet set-up (main.cpp:399-423) on a config: with jet_enabled, jets
   are switched off for a neutron star or without a disc (no accretion flow),
   z_sat is capped at 0.7 z_top, the jet is configured from the disc's
   accretion rate, and switched off when the hole has no rotational power. */
int  bh_render_config_setup_jet(bh_render_config* cfg);

int  bh_gpu_create(int device, bh_ctx** out);
void bh_gpu_destroy(bh_ctx* ctx);
const char* bh_gpu_last_error(const bh_ctx* ctx);

/* Replaces bh::render (render.cpp:396-497): trace and shade every sample of
   the frame, write W*H pixels (row-major, averaged over sqrt_spp^2 samples)
   into the caller's host buffer and add the frame's counters into *stats
   (stats may be NULL). */
int  bh_gpu_render(bh_ctx* ctx, const bh_render_config* cfg,
                   bh_xyz* out_pixels, bh_render_stats* stats);

/* The same frame, written into a device buffer of W*H bh_xyz on `stream`
   (a cudaStream_t, or NULL for the legacy default stream).  Returns once the work
   is enqueued when stats == NULL; with stats it synchronises. */
int  bh_gpu_render_device(bh_ctx* ctx, const bh_render_config* cfg,
                          bh_xyz* d_pixels, bh_render_stats* stats, void* stream);

/* Per-sample results of a whole frame: W*H*sqrt_spp^2 entries, ordered by
   pixel (row-major) and then by sample (sy, sx) as in render.cpp:439-456. */
int  bh_gpu_trace_rays(bh_ctx* ctx, const bh_render_config* cfg,
                       bh_ray_result* out, bh_render_stats* stats);

/* Many frames of any size in one persistent launch (replaces the serial frame
   loop of main.cpp:952-989).  outs[i] receives frame i's pixels; stats[i]
   (optional array) receives frame i's counters.  All frames must share the
   precision, sky and star settings of cfgs[0].  The batch runs as one CUDA
   graph (staging copies, trace, shade, stats), captured on the first call and
   replayed while the batch shape (frame count and sizes, launch parameters,
   buffers) is unchanged; kernel_ms is then the device time of the whole graph
   and shade_ms is 0. */
int  bh_gpu_render_batch(bh_ctx* ctx, const bh_render_config* cfgs, int n,
                         bh_xyz* const* outs, bh_render_stats* stats);

/* Launch shape of the trace kernel of `precision` (BH_PRECISION_*, or -1 for
   both) used by the next calls; zero fields keep the current value.  The
   binary64 pass that finishes mixed-precision rays uses the FP64 shape. */
int  bh_gpu_set_launch(bh_ctx* ctx, int precision, const bh_launch_params* p);
int  bh_gpu_get_launch(const bh_ctx* ctx, int precision, bh_launch_params* p);

/* Autotuner: render `cfg` twice per launch shape of the search space (block
   size 64..512, rays per thread 1..8, refill threshold 8..32 idle lanes,
   both register caps), keep the shape with the shortest trace-kernel time for
   cfg->precision, and return it in *best (and its time in *best_ms).  Extension;
   no counterpart in the reference. */
int  bh_gpu_autotune(bh_ctx* ctx, const bh_render_config* cfg, bh_launch_params* best, double* best_ms);

/* The same search on a batch of frames through bh_gpu_render_batch (each
   shape timed on the captured batch graph; *best_ms is its device time).
   The search space: block size 64..512, rays per thread 1..8, refill
   threshold 8..32 idle lanes (a refill claims n_idle x rays_per_thread rays,
   8 to 256, in one atomic), both register caps.  Extension; no counterpart
   in the reference. */
int  bh_gpu_autotune_batch(bh_ctx* ctx, const bh_render_config* cfgs, int n, bh_launch_params* best,
                           double* best_ms);

/* Step budget of one launch (total step attempts over all rays; 0 = none).
   A launch that exceeds it stops taking rays and returns BH_ERR_BUDGET. */
int  bh_gpu_set_step_budget(bh_ctx* ctx, long long budget);

/* Ask the next or running launch on this context to stop taking rays; it then
   returns BH_ERR_ABORTED.  Safe to call from another host thread. */
void bh_gpu_request_abort(bh_ctx* ctx);
void bh_gpu_clear_abort(bh_ctx* ctx);

/* One ray's trace result, without shading: final state (t, r, th, phi, p_t,
   p_r, p_th, p_phi), the worst relative null norm and Carter drift along the
   ray, its termination class (BH_HIT_*), accepted steps and step attempts. */
typedef struct bh_trace_record {
    double y[8];
    double max_norm;
    double max_q;
    int32_t what;
    int32_t steps;
    int32_t attempts;
    int32_t reserved;
} bh_trace_record;

/* Largest ray count (width * height * sqrt_spp^2) bh_gpu_trace_noalloc takes. */
#define BH_NOALLOC_MAX_RAYS 65536

/* Trace the rays of `cfg` into the caller's device buffer d_out (n_rays
   bh_trace_record) on `stream` (a cudaStream_t; NULL = the legacy default
   stream), WITHOUT allocating: for callers that cannot call cudaMalloc -
   hosts whose GPU memory belongs to their own allocator or fixed budget
   (engines, frameworks with a caching allocator, plug-in hosts that forbid
   device allocation in the render callback), and real-time loops that cannot
   afford the implicit device synchronisation cudaMalloc/cudaFree may cause.
   It allocates no device memory, and on success no host memory either.
   The kernel's scratch (work-queue counters, frame constants, and for
   BH_PRECISION_MIXED the list of rays handed to binary64) lives in one
   statically allocated 6.3 MiB device array of this library, so a call
   takes at most BH_NOALLOC_MAX_RAYS rays and returns BH_ERR_INVALID_ARG
   above that.  Every GPU that loads the library holds the array until exit.
   The first call on a device looks the array's device address up, and with
   CUDA's lazy module loading (the default) it is also the call that loads
   this library's kernels and places the array on that device, which may
   allocate and synchronise the device: make that first call once during
   set-up, outside the real-time path and before any stream capture.  Every
   call clears the counters it needs at zero, and all calls share the one
   array, so calls whose work overlaps on the GPU (other streams, other host
   threads) race - serialise them.  The calling thread's current device is
   the same on return as on entry.
   A config with a jet returns BH_ERR_UNSUPPORTED (the jet's emission is a
   per-ray sum this entry point has no scratch for).
   Stars, disc temperature and pixels are not computed (no shading): the
   records equal the trace part of bh_gpu_trace_rays for the same config and
   default launch shape.  Records are in work order: ray id = p * S^2 + k for
   sample k = sy * S + sx of pixel p, with pixels numbered in bands of four
   rows, column by column inside a band (band b = p / (4 W) covers rows
   4b .. 4b + h - 1, h = min(4, H - 4b); x = (p - 4Wb) / h, y = 4b + (p - 4Wb) % h).
   Returns once the work is enqueued.  No counterpart in the reference. */
int  bh_gpu_trace_noalloc(int device, const bh_render_config* cfg, bh_trace_record* d_out, void* stream);

/* Result of the discrete adjoint (bh_gpu_adjoint). */
typedef struct bh_grad4 {
    double loss;             /* sum over pixels of (Y - target)^2, Y the CIE Y of the frame */
    double d_spin;           /* dLoss / d(spin), edge term included               */
    double d_inclination;    /* dLoss / d(camera polar angle cam.theta), per radian, edge term included */
    double d_eddington;      /* dLoss / d(eddington)                              */
    double d_r_out;          /* dLoss / d(disc_r_out): the edge term alone        */
    double kernel_ms;        /* device time of the render, adjoint, edge pass and reductions */
    long long rays;
    long long steps;         /* accepted steps of the adjoint's forward pass      */
    long long replayed_steps;/* accepted steps recomputed by the reverse pass     */
    long long disc_rays;
    long long sky_rays;
    int32_t max_checkpoint_interval;
    int32_t reserved;
    double edge_spin;        /* the edge term's part of d_spin                    */
    double edge_inclination; /* the edge term's part of d_inclination             */
    long long edge_candidates;/* equatorial crossings examined for an edge       */
    long long edge_cells;    /* edges found crossing a sample's cell              */
    long long edge_steps;    /* accepted steps integrated by the edge pass        */
    double held_spin;        /* per-ray spin terms of images of order >= 3, not in d_spin */
    double held_inclination; /* the same for the inclination                     */
    long long high_order_rays;/* rays whose event came after a third equatorial crossing */
} bh_grad4;

/* The luminance loss of `cfg` against `target` (W*H floats, row-major, the
   CIE Y in W m^-2 sr^-1 of each pixel) and its gradient with respect to the
   spin, the camera inclination, the Eddington ratio and the disc's outer
   radius.  The frame is rendered in binary64 (whatever cfg->precision says);
   the gradient is the discrete adjoint of that render: each ray's accepted
   DP5 step sequence is replayed backwards from checkpoints (every 16 accepted
   steps, 64 per ray in flight; the interval doubles for longer rays), with
   the step sizes and each ray's termination class held fixed.  To that the
   edge term is added: the motion of the disc's outer edge (r_out) and inner
   edge (the ISCO) across the image, which a point-sampled frame shows only
   as samples changing class.  It is the derivative of the frame averaged
   over each sample's cell of the pixel: for every sample whose first or
   second equatorial crossing lies near an edge (within twice the spread of
   the neighbouring samples' same crossing), (luminance jump across the edge)
   x (length of the edge in the cell) / |image-plane gradient of the
   crossing radius|, times the edge's speed, the gradient and the speed
   coming from a reverse sweep of that crossing radius.  d_r_out is that term
   alone; edge_spin and edge_inclination are its part of d_spin and
   d_inclination.  The derivative covers the images of the first two
   equatorial crossings (the direct image and the first lensed image):
   images of order three and higher are rings thinner than a sample's cell
   at ordinary resolutions, whose per-sample derivative holds over a small
   part of the cell, so their per-ray spin and inclination terms are
   reported apart (held_spin, held_inclination) and their edges are left
   out.  Scenes with the Sun, a neutron star, a hot spot or a jet return
   BH_ERR_UNSUPPORTED.  No counterpart in the reference. */
int  bh_gpu_adjoint(bh_ctx* ctx, const bh_render_config* cfg, const float* target, bh_grad4* out);

/* bh_gpu_adjoint plus, when not NULL, each ray's gradient contribution
   (4 doubles: spin, inclination, eddington, r_out; the per-ray discrete
   adjoint, without the edge term) and its luminance, in bh_gpu_trace_rays
   order (pixel row-major, then sample). */
int  bh_gpu_adjoint_rays(bh_ctx* ctx, const bh_render_config* cfg, const float* target, bh_grad4* out,
                         double* ray_grad, double* ray_Y);

/* Tone curves of the display transform, in img::ToneMap order (image.h:16). */
enum {
    BH_TONEMAP_LINEAR = 0,
    BH_TONEMAP_REINHARD = 1,
    BH_TONEMAP_ACES = 2,
    BH_TONEMAP_LOG = 3,
    BH_TONEMAP_HDR = 4
};

/* The display settings of the reference CLI (main.cpp:20-29, 905-909). */
typedef struct bh_display {
    double exposure;         /* > 0: this multiplier; <= 0: metered (img::auto_exposure) */
    double key;              /* auto_exposure's key (1.0)                          */
    double glare;            /* add_glare strength in [0, 1]; 0 = off (the default) */
    double glare_radius;     /* add_glare radius in pixels (3.0)                   */
    double log_decades;      /* decades of the Log and HDR curves (16.0)           */
    int32_t tonemap;         /* BH_TONEMAP_* (BH_TONEMAP_HDR)                      */
    int32_t reserved;
} bh_display;

void bh_display_default(bh_display* d);

/* Replaces img::add_glare + img::auto_exposure + img::develop (image.cpp:22-191)
   on a caller's frame: `pixels` (W*H bh_xyz, row-major, host) is glared (on a
   device copy: the caller's buffer is not changed), metered unless
   d->exposure > 0, and developed into out_rgb (W*H*3 bytes, host; may be NULL
   to meter only).  *exposure_used (may be NULL) receives the multiplier. */
int  bh_gpu_develop(bh_ctx* ctx, const bh_xyz* pixels, int width, int height, const bh_display* d,
                    uint8_t* out_rgb, double* exposure_used);

/* bh_gpu_render and the display transform in one call, the frame never
   leaving the device as XYZ: the sequence of main.cpp:905-909 with 3 bytes per
   pixel copied back instead of 24.  out_rgb may be NULL (meter only, as the
   animation's probe frame, main.cpp:931-944). */
int  bh_gpu_render_rgb(bh_ctx* ctx, const bh_render_config* cfg, const bh_display* d, uint8_t* out_rgb,
                       double* exposure_used, bh_render_stats* stats);

/* An animation's frames (main.cpp:931-989): all frames traced in one
   persistent launch, then each one glared and developed on the device into
   outs_rgb[i] (W_i*H_i*3 bytes, host).  With d->exposure > 0 every frame uses
   that exposure (the reference locks it from a probe frame, main.cpp:931-944);
   otherwise each frame is metered on its own.  exposure_used (n doubles) and
   stats (n entries, as bh_gpu_render_batch) may be NULL. */
int  bh_gpu_render_batch_rgb(bh_ctx* ctx, const bh_render_config* cfgs, int n, const bh_display* d,
                             uint8_t* const* outs_rgb, double* exposure_used, bh_render_stats* stats);

/* What bh_gpu_eval evaluates. */
enum {
    BH_EVAL_RHS = 0,              /* in: n states of 8 doubles (t, r, th, phi, p_t, p_r, p_th, p_phi);
                                     out: n x 8 derivatives d/d lambda (the trace kernels' right-hand
                                     side in cfg->precision; dp_t = dp_phi = 0) */
    BH_EVAL_DISC_TEMPERATURE = 1, /* in: n radii (M); out: n Novikov-Thorne effective temperatures (K)
                                     of cfg's disc, as the shading evaluates them */
    BH_EVAL_BLACKBODY = 2,        /* in: n temperatures (K); out: n x 3 CIE XYZ (W m^-2 sr^-1) from the
                                     device's blackbody table */
    BH_EVAL_FRAME = 3             /* in: unused (n = 1); out: 8 frame constants of cfg: r_+, r_-, r_in
                                     (the ISCO), r_out, the efficiency 1 - E_isco, the accretion rate
                                     (kg/s), the stop radius, the escape radius */
};

/* The device functions of the render path evaluated at caller-given inputs
   (host buffers), for known-answer tests of the GPU arithmetic against
   closed forms and the reference's own checks (validate.cpp sections 1, 3,
   6, 7).  Synchronous.  No counterpart in the reference. */
int  bh_gpu_eval(bh_ctx* ctx, const bh_render_config* cfg, int what, const double* in, long long n, double* out);

/* Measured FMA throughput of `device` in TFLOP/s (2 FLOP per FMA) for
   BH_PRECISION_FP64 (binary64) or BH_PRECISION_MIXED (binary32): the ALU
   roofline of the trace kernel.  Extension; no counterpart in the reference. */
int  bh_gpu_fma_peak(int device, int precision, double* tflops);

/* The star catalogue the render path uploads for (count, seed, sky_mode): six
   doubles per star (x, y, z, magnitude, temperature K, irradiance W m^-2) in
   generation order, as StarField builds it (scene.h:62-104).  Host-side; needs
   no GPU.  Replaces nothing: exposes the catalogue for inspection. */
int  bh_star_catalogue(int count, uint64_t seed, int sky_mode, double* out6);

/* ln X, ln Y, ln Z of the 4096-entry blackbody table the GPU reads
   (spectrum.cpp:94-121), 3*4096 doubles.  Host-side; needs no GPU. */
int  bh_blackbody_table(double* out);

#ifdef __cplusplus
}
#endif

#endif /* BH_GPU_H */
