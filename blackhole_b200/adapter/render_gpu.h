// render_gpu.h - the `--gpu` drop-in for bh::render (render.h:72).
//
// Added to the reference's tree beside render.h (or compiled with -I to it and
// to this repository's include/), render_gpu.cpp turns a bh::RenderConfig into
// the C-ABI's bh_render_config and renders through libbh_gpu.so into an
// img::Image, so the caller's display chain (add_glare, auto_exposure,
// develop, write_png) runs unchanged.  The three call sites of bh::render in
// main.cpp (906 still, 941 exposure probe, 964 animation frames) become
// `use_gpu ? bh::render_gpu(cfg, st) : bh::render(cfg, st)`.
#pragma once

#include <stdexcept>
#include <string>

#include "bh_gpu.h"
#include "render.h"

namespace bh {

// A failed GPU call: `status` is the BH_ERR_* code (BH_ERR_NO_DEVICE when no
// sm_100 GPU is usable), what() the library's message.  The reference's
// render() has no error path; its GPU form reports one by exception.
struct GpuError : std::runtime_error {
    int status;
    GpuError(int st, const std::string& msg) : std::runtime_error(msg), status(st) {}
};

// bh::RenderConfig -> bh_render_config, field for field; the GPU extensions
// keep their defaults (binary64, the reference's sky and horizon stop) unless
// `precision` asks for BH_PRECISION_MIXED.
bh_render_config gpu_config(const RenderConfig& cfg, int precision = BH_PRECISION_FP64);

// Drop-in for render(cfg, stats) on this host thread's GPU context (device
// 0, created on the first call): the same pixels as an img::Image, stats
// added into `stats` as render() adds them (render.cpp:481-495), `seconds`
// overwritten.  Throws GpuError on failure.
img::Image render_gpu(const RenderConfig& cfg, RenderStats& stats, int precision = BH_PRECISION_FP64);

// Destroys this host thread's context (render_gpu makes a new one when
// called again).
void release_gpu();

}  // namespace bh
