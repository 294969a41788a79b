// bh_display.h - Launch descriptor of the display transform (bh_display.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bh_gpu.h"

namespace bhg {

// Device state of the exposure meter's radix select.
struct ExposureState {
    unsigned long long count;        // positive finite luminances
    unsigned long long k[2];         // remaining rank of the 99.9th and 99.99th percentile
    unsigned long long prefix[2];    // their bits found so far
    unsigned long long mask;         // which bits are found
    unsigned long long hist[2][256];
};

struct DisplayLaunch {
    bh_xyz* pixels;                  // W x H, row-major (glare writes it in place)
    int width, height;
    // add_glare
    double glare, glare_radius;
    const double* k_near;            // normalised weights, 2 r + 1 each
    const double* k_far;
    int r_near, r_far;
    bh_xyz *tmp, *nearp, *farp;      // W x H scratch each
    // exposure: fixed when > 0, else metered with `key`
    double exposure, key;
    ExposureState* state;
    double* exposure_out;            // device double
    int reduce_blocks;
    // develop (skipped when rgb is null)
    int tonemap;
    double log_k, denom;             // 10^clamp(log_decades, 1, 20), log10(1 + log_k)
    uint8_t* rgb;                    // W x H x 3
};

cudaError_t launch_display(const DisplayLaunch& L, cudaStream_t stream);

}  // namespace bhg
