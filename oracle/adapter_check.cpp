// adapter_check.cpp - C entry points onto the drop-in adapter bh::render_gpu.
//
// TEST INFRASTRUCTURE.  Compiled by oracle/Makefile against the reference's
// own headers (render.h and what it includes) with the adapter source
// blackhole_b200/adapter/render_gpu.cpp, the reference's render.cpp,
// spectrum.cpp and image.cpp, and linked with libbh_gpu.so: the adapter is
// built exactly as a maintainer would build it into the reference, and the
// tests drive it from here.
//   - adc_roundtrip:  gpu_config(to_ref(in)): every field the reference has
//                     must come back unchanged (catches field drift);
//   - adc_render_gpu: bh::render_gpu of a config, pixels and stats out (the
//                     status of a GpuError otherwise);
//   - adc_render_ref: the reference's own bh::render of the same config.
#include <algorithm>
#include <cstring>
#include <string>

#include "render.h"
#include "render_gpu.h"
#include "../include/bh_gpu.h"
#include "ref_config.h"

namespace {

void stats_out(const bh::RenderStats& s, bh_render_stats* o) {
    if (!o) return;
    o->rays = s.rays;
    o->steps = s.steps;
    o->captured = s.captured;
    o->disc_hits = s.disc_hits;
    o->sun_hits = s.sun_hits;
    o->star_hits = s.star_hits;
    o->jet_rays = s.jet_rays;
    o->escaped = s.escaped;
    o->exhausted = s.exhausted;
    o->total_flux = s.total_flux;
    o->max_norm_error = s.max_norm_error;
    o->max_carter_drift = s.max_carter_drift;
    o->seconds = s.seconds;
}

}  // namespace

extern "C" {

int adc_roundtrip(const bh_render_config* in, bh_render_config* out, int precision) {
    if (!in || !out) return BH_ERR_INVALID_ARG;
    *out = bh::gpu_config(to_ref(*in, false), precision);
    return BH_OK;
}

int adc_render_gpu(const bh_render_config* c, bh_xyz* out, bh_render_stats* st, int precision) {
    if (!c || !out) return BH_ERR_INVALID_ARG;
    try {
        bh::RenderStats s;
        const img::Image im = bh::render_gpu(to_ref(*c), s, precision);
        std::memcpy(out, im.pixels.data(), im.pixels.size() * sizeof(spec::XYZ));
        stats_out(s, st);
        return BH_OK;
    } catch (const bh::GpuError& e) {
        return e.status;
    }
}

int adc_render_ref(const bh_render_config* c, bh_xyz* out, bh_render_stats* st) {
    if (!c || !out) return BH_ERR_INVALID_ARG;
    bh::RenderStats s;
    const img::Image im = bh::render(to_ref(*c), s);
    std::memcpy(out, im.pixels.data(), im.pixels.size() * sizeof(spec::XYZ));
    stats_out(s, st);
    return BH_OK;
}

void adc_release() { bh::release_gpu(); }

}  // extern "C"
