// bh_scene.h - Host-side scene preparation for the GPU render path.
//
// Everything the reference computes once per frame before its pixel loop
// (render.cpp:396-418): the disc constants, the camera tetrad, the star
// catalogue and the blackbody table.  The catalogue and table are built here
// with the reference's formulas and operand order on the host libm, so they
// are bit-identical to the reference's own (scene.h:62-107,
// spectrum.cpp:94-121); the GPU only reads them.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/bh_gpu.h"
#include "bh_frame.h"

namespace bhg {

struct HostSky {
    std::vector<double4> pos;        // x, y, z, irradiance, in bin order
    std::vector<double4> col;        // blackbody_xyz(T): x, z, 1/y, 0
    std::vector<int32_t> bin_start;  // kLat*kLon + 1
    double mw_x = 0, mw_z = 0, mw_inv = 0, diffuse_L = 0;
};

// ln X, ln Y, ln Z of the 4096-entry table (spectrum.cpp:101-121).
void build_blackbody_table(std::vector<double>& tab);
// Table lookup (spectrum.cpp:123-134).
void blackbody_xyz_host(const std::vector<double>& tab, double T, double out[3]);

// Star catalogue of `count` stars from `seed` in `sky_mode`, binned.
int build_sky(int count, uint64_t seed, int sky_mode, const std::vector<double>& tab, HostSky& out,
              std::string& err);

// The raw catalogue, six doubles per star in generation order.
int star_catalogue(int count, uint64_t seed, int sky_mode, double* out6);

// Validate a config and fill the frame constants.  Returns a bh_status.
int make_frame(const bh_render_config& c, FrameParams& F, std::string& err);

// The constants under which a mixed-precision frame's near-critical rays are
// traced in binary64: those of the binary64 path (the config's tolerances,
// the reference's step cap, no early capture, no mirrored hemisphere).
FrameParams binary64_treatment(const FrameParams& F);

// The reference defaults (render.h:15-53, scene.h:232-351, neutronstar.h:43-70,
// jet.h:96-146).
void default_config(bh_render_config& c);

// Jet::configure (jet.h:262-312) and the CLI's jet set-up (main.cpp:399-423).
void jet_configure(bh_jet& j, double spin, double mdot_c2, double r_g_m);
int setup_jet(bh_render_config& c);

}  // namespace bhg
