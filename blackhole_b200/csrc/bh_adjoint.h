// bh_adjoint.h - Frame constants of the discrete adjoint (host and device).
//
// The adjoint differentiates the luminance loss of one frame with respect to
// four scene parameters: the spin a, the camera inclination (its polar angle
// theta, radians), the accretion rate in Eddington units and the disc's outer
// radius.  Everything per frame that depends on a parameter carries its
// derivative here, computed on the host with dual numbers; the per-ray part
// runs on the device (bh_adjoint.cuh).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/bh_gpu.h"
#include "bh_frame.h"

namespace bhg {

// Index of a parameter in the tangent arrays below.
enum { kParSpin = 0, kParIncl = 1 };

struct AdjointFrame {
    // d/d(spin) and d/d(inclination) of the camera's non-zero ZAMO tetrad legs
    // (tet00, tet03, tet11, tet22, tet33) and of g_{mu nu} at the camera
    // (tt, t phi, rr, theta theta, phi phi).
    double d_tet[5][2];
    double d_ml[5][2];
    // d/d(spin) of the disc constants; the disc's spin is clamped to
    // +-0.9999 (disc.h:75), beyond which they do not move.
    double d_disc_a;
    double d_x0;
    double d_pt_x[3], d_pt_c[3], d_pt_den[3];
    double d_mdot_da;                // d(accretion rate in kg/s) / d(spin), through the efficiency
    double d_mdot_dedd;              // d(accretion rate) / d(Eddington ratio)
    int32_t checkpoint_interval;     // accepted steps between stored states (doubles when full)
    int32_t checkpoint_slots;        // stored states per ray in flight
};

// Checks that the scene is one the adjoint covers (a disc and/or a sky; no
// Sun, neutron star or hot spot) and fills the derivatives.  Returns a
// bh_status; `F` must come from make_frame for the same config.
int make_adjoint_frame(const bh_render_config& c, const FrameParams& F, AdjointFrame& X, std::string& err);

// One adjoint launch over the rays of one frame.
struct AdjointLaunch {
    FrameParams frame;               // binary64 frame constants (ray_begin 0)
    AdjointFrame X;
    SkyData sky;
    const bh_xyz* pixels;            // the rendered frame, row-major W x H (device)
    const float* target;             // target luminance, row-major W x H (device)
    double* ray_grad;                // 4 per ray, pixel-major then sample (device)
    double* ray_Y;                   // luminance per ray in the same order, or nullptr
    double* ckpt;                    // grid * block * checkpoint_slots * 8 doubles
    // The edge pass: per crossing slot (2 per ray, slot = 2 * ray + crossing,
    // rays in work order) the radius of the ray's first two equatorial
    // crossings as the render found them (0: none; zeroed before the
    // render), the candidate list ((slot << 2) | kEdge* bits) and 3 edge
    // contributions per slot.
    double* xing_r;
    unsigned long long* cand;
    double* edge_out;
    // 1 for a ray whose event came after its third or later equatorial
    // crossing (an image of order three or higher), in ray_grad order
    unsigned char* high_order;
    // next job, accepted, replayed, disc rays, sky rays, max interval, edge
    // candidates, edge-pass steps, edge cells, high-order rays
    unsigned long long* counters;
    // loss; the four per-ray gradient sums (spin and inclination over the
    // rays of image order one and two); the three edge sums; the spin and
    // inclination sums over the rays of order three and higher
    double* sums;
    long long n_rays;
    int grid, block;
};

constexpr int kAdjCounters = 10;
constexpr int kAdjSums = 10;

// Enqueues the edge pass's candidate selection over the sample grid, the
// adjoint kernel (edge terms, then the rays) and the deterministic reduction
// of the per-ray gradients, the edge contributions and the loss; `counters`
// and `edge_out` must be zeroed before.
cudaError_t launch_adjoint(const AdjointLaunch& L, cudaStream_t stream);
// Resident blocks of the adjoint kernel per SM at `block_size` threads.
int adjoint_blocks_per_sm(int block_size);

}  // namespace bhg
