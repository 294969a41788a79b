// bh_capi.cpp - The C-ABI of include/bh_gpu.h.
//
// A bh_ctx owns one CUDA stream on one device, the device copies of the
// blackbody table and of the star catalogue (rebuilt only when count, seed or
// sky mode change), and grow-only ray/pixel buffers.  A render call is: frame
// constants -> H2D, queue reset, the persistent trace kernel, the shade
// kernel, the stats reduction, D2H of pixels and stats.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/bh_gpu.h"
#include "bh_frame.h"
#include "bh_adjoint.h"
#include "bh_display.h"
#include "bh_launch.h"
#include "bh_scene.h"

using namespace bhg;

namespace {

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};

}  // namespace

struct bh_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t abort_stream = nullptr;
    cudaStream_t side_stream = nullptr;     // the binary32 kernel's, beside the near-critical binary64 one
    cudaEvent_t fork_event = nullptr, join_event = nullptr;
    std::string err;
    // Launch shapes of the FP64 [0] and mixed [1] trace kernels (measured
    // best on the 1024^2 edge-on frame: the tight register caps, blocks of
    // 128 for FP64 and 256 for mixed).
    bh_launch_params launch[2] = {{128, 1, 32, 0, 1}, {256, 1, 32, 0, 1}};
    unsigned long long budget = 0;
    std::atomic<int> abort_requested{0};
    int32_t* h_one = nullptr;          // pinned 1, source of the abort copy
    // Pinned read-back of a single-frame launch's queue state and stats,
    // copied on the stream before the call's one synchronisation.
    unsigned char* h_readback = nullptr;
    // bh_gpu_render's row-band pipeline: the driver's stream wait on a device
    // word (null where the driver does not offer it: no pipeline), the
    // streams the bands are shaded and copied on, the events that join them
    // back, and the per-band finished-ray counters.
    CUresult (*wait_value32)(CUstream, CUdeviceptr, cuuint32_t, unsigned int) = nullptr;
    cudaStream_t band_stream[8] = {};
    cudaEvent_t band_join[8] = {};

    std::vector<double> h_table;
    double* d_table = nullptr;

    bool sky_valid = false;
    int sky_count = -1;
    uint64_t sky_seed = 0;
    int sky_mode = -1;
    double4* d_star_pos = nullptr;
    double4* d_star_col = nullptr;
    int32_t* d_bin_start = nullptr;
    HostSky sky_meta;

    DevBuf hits, pixels, rays, lum, frames, ray_end, pix_end, partials, fstats, deferred, jet;
    DevBuf sel_flag, sel_list;         // near-critical classification of a mixed launch's rays
    // Adjoint: target image, per-ray gradients and luminances, checkpoint
    // slots, counters, sums and the edge pass's buffers.
    DevBuf adj_target, adj_grad, adj_Y, adj_ckpt, adj_counters, adj_sums, adj_xr, adj_cand, adj_edge, adj_high;
    DevBuf band_done;
    // Display transform: blur scratch, glare weights, meter state, 8-bit output.
    DevBuf disp_tmp, disp_near, disp_far, disp_k, disp_state, disp_rgb;
    // bh_gpu_eval: inputs and outputs.
    DevBuf eval_in, eval_out;
    QueueState* d_queue = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    long long h2d = 0, d2h = 0;          // bytes copied by the current call

    // Pinned staging of the per-launch constants, and the event after which
    // the last launch no longer reads it.
    unsigned char* stage = nullptr;
    size_t stage_cap = 0;
    cudaEvent_t stage_free = nullptr;

    // The captured CUDA graph of the last batch shape (bh_gpu_render_batch),
    // keyed by the launch descriptors it was captured from.
    cudaGraphExec_t batch_exec = nullptr;
    std::vector<unsigned char> batch_key;
};

namespace {

constexpr int kReduceBlocks = 512;
// Blocks of the near-critical binary64 kernel beside a mixed-precision launch.
constexpr int kSideBlocks = 32;
// Registers of one SM, and the registers a warp of threads using `per_thread`
// is allocated (in units of 256).
constexpr long long kSmRegs = 65536;
long long warp_regs(int per_thread) { return (static_cast<long long>(per_thread) * 32 + 255) / 256 * 256; }

int fail(bh_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(bh_ctx* ctx, cudaError_t e, const char* what) {
    return fail(ctx, e == cudaErrorMemoryAllocation ? BH_ERR_OUT_OF_MEMORY : BH_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                          \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

int ensure(bh_ctx* ctx, DevBuf& b, size_t bytes) {
    if (bytes <= b.cap) return BH_OK;
    if (b.p) {
        cudaFree(b.p);
        b.p = nullptr;
        b.cap = 0;
    }
    const size_t want = std::max<size_t>(bytes, 256);
    CK(cudaMalloc(&b.p, want));
    b.cap = want;
    return BH_OK;
}

int check_cfg_header(bh_ctx* ctx, const bh_render_config* cfg) {
    if (!cfg) return fail(ctx, BH_ERR_INVALID_ARG, "config is NULL");
    if (cfg->struct_size != sizeof(bh_render_config))
        return fail(ctx, BH_ERR_INVALID_ARG, "bh_render_config.struct_size does not match the library");
    if (cfg->abi_version != BH_GPU_ABI_VERSION)
        return fail(ctx, BH_ERR_INVALID_ARG, "bh_render_config.abi_version does not match the library");
    return BH_OK;
}

int ensure_table(bh_ctx* ctx) {
    if (ctx->d_table) return BH_OK;
    build_blackbody_table(ctx->h_table);
    CK(cudaMalloc(&ctx->d_table, ctx->h_table.size() * sizeof(double)));
    CK(cudaMemcpy(ctx->d_table, ctx->h_table.data(), ctx->h_table.size() * sizeof(double),
                  cudaMemcpyHostToDevice));
    return BH_OK;
}

int ensure_sky(bh_ctx* ctx, const bh_render_config& c) {
    int rc = ensure_table(ctx);
    if (rc != BH_OK) return rc;
    const int count = c.stars_enabled ? c.star_count : 0;
    if (ctx->sky_valid && ctx->sky_count == count && ctx->sky_seed == c.seed && ctx->sky_mode == c.sky_mode)
        return BH_OK;
    HostSky hs;
    std::string err;
    rc = build_sky(count, c.seed, c.sky_mode, ctx->h_table, hs, err);
    if (rc != BH_OK) return fail(ctx, rc, err);
    cudaFree(ctx->d_star_pos);
    cudaFree(ctx->d_star_col);
    cudaFree(ctx->d_bin_start);
    ctx->d_star_pos = nullptr;
    ctx->d_star_col = nullptr;
    ctx->d_bin_start = nullptr;
    ctx->sky_valid = false;
    const size_t n = std::max<size_t>(hs.pos.size(), 1);
    CK(cudaMalloc(&ctx->d_star_pos, n * sizeof(double4)));
    CK(cudaMalloc(&ctx->d_star_col, n * sizeof(double4)));
    CK(cudaMalloc(&ctx->d_bin_start, hs.bin_start.size() * sizeof(int32_t)));
    if (!hs.pos.empty()) {
        CK(cudaMemcpy(ctx->d_star_pos, hs.pos.data(), hs.pos.size() * sizeof(double4), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(ctx->d_star_col, hs.col.data(), hs.col.size() * sizeof(double4), cudaMemcpyHostToDevice));
    }
    CK(cudaMemcpy(ctx->d_bin_start, hs.bin_start.data(), hs.bin_start.size() * sizeof(int32_t),
                  cudaMemcpyHostToDevice));
    hs.pos.clear();
    hs.col.clear();
    ctx->sky_meta = std::move(hs);
    ctx->sky_count = count;
    ctx->sky_seed = c.seed;
    ctx->sky_mode = c.sky_mode;
    ctx->sky_valid = true;
    return BH_OK;
}

SkyData sky_data(const bh_ctx* ctx) {
    SkyData s;
    std::memset(&s, 0, sizeof s);
    s.star_pos = ctx->d_star_pos;
    s.star_col = ctx->d_star_col;
    s.bin_start = ctx->d_bin_start;
    s.table = ctx->d_table;
    s.mw_x = ctx->sky_meta.mw_x;
    s.mw_z = ctx->sky_meta.mw_z;
    s.mw_inv = ctx->sky_meta.mw_inv;
    s.diffuse_L = ctx->sky_meta.diffuse_L;
    s.n_stars = ctx->sky_count > 0 ? ctx->sky_count : 0;
    return s;
}

void stats_add(bh_render_stats* s, const FrameStats& f) {
    s->rays += (long long)f.rays;
    s->steps += (long long)f.steps;
    s->attempts += (long long)f.attempts;
    s->captured += (long long)f.captured;
    s->disc_hits += (long long)f.disc_hits;
    s->sun_hits += (long long)f.sun_hits;
    s->star_hits += (long long)f.star_hits;
    s->escaped += (long long)f.escaped;
    s->exhausted += (long long)f.exhausted;
    s->jet_rays += (long long)f.jet_rays;
    double mn, mq;
    std::memcpy(&mn, &f.max_norm_bits, sizeof mn);
    std::memcpy(&mq, &f.max_q_bits, sizeof mq);
    s->max_norm_error = std::max(s->max_norm_error, mn);
    s->max_carter_drift = std::max(s->max_carter_drift, mq);
    s->total_flux += f.total_flux;
}

// One launch of the pipeline, planned on the host.
struct Plan {
    int n = 0;
    int nf = 0;          // frames staged: n, or 2n with the binary64 treatment of mixed frames
    long long rays = 0, pix = 0;
    bool mixed = false;
    TraceLaunch tl;
    ShadeLaunch sl;
    ReduceLaunch rl;
    size_t stage_bytes = 0;
};

// Host half of a launch: size the device buffers (all allocation happens
// here) and write the frame constants, cumulative ends and the queue's
// initial state into the context's pinned staging buffer.
int plan_launch(bh_ctx* ctx, std::vector<FrameParams>& frames, bh_xyz* d_pixels, bh_ray_result* d_rays,
                bool timed, Plan& p) {
    const int n = static_cast<int>(frames.size());
    p.n = n;
    long long rays = 0, pix = 0;
    for (int i = 0; i < n; ++i) {
        frames[i].ray_begin = rays;
        frames[i].pixel_begin = pix;
        rays += frames[i].n_rays;
        pix += static_cast<long long>(frames[i].width) * frames[i].height;
    }
    p.rays = rays;
    p.pix = pix;
    int rc;
    if ((rc = ensure(ctx, ctx->hits, static_cast<size_t>(rays) * sizeof(HitRecord))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->lum, static_cast<size_t>(pix) * sizeof(double))) != BH_OK) return rc;
    p.mixed = frames[0].precision_tag == BH_PRECISION_MIXED;
    p.nf = p.mixed ? 2 * n : n;
    if ((rc = ensure(ctx, ctx->frames, p.nf * sizeof(FrameParams))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->ray_end, n * sizeof(long long))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->pix_end, n * sizeof(long long))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->partials, static_cast<size_t>(n) * kReduceBlocks * sizeof(FrameStats))) != BH_OK)
        return rc;
    if ((rc = ensure(ctx, ctx->fstats, n * sizeof(FrameStats))) != BH_OK) return rc;
    bool any_jet = false, any_surface = false, any_near_critical = false;
    for (int i = 0; i < n; ++i) {
        any_jet = any_jet || frames[i].jet_enabled;
        any_near_critical = any_near_critical || frames[i].fp64_near_critical;
        any_surface = any_surface || frames[i].sun_enabled || frames[i].ns_enabled;
    }
    if (any_jet && (rc = ensure(ctx, ctx->jet, static_cast<size_t>(rays) * sizeof(double))) != BH_OK) return rc;
    if (p.mixed && (rc = ensure(ctx, ctx->deferred, static_cast<size_t>(rays) * deferred_record_bytes())) != BH_OK)
        return rc;
    if (any_near_critical && (rc = ensure(ctx, ctx->sel_flag, static_cast<size_t>(rays))) != BH_OK) return rc;
    if (any_near_critical && (rc = ensure(ctx, ctx->sel_list, static_cast<size_t>(rays) * sizeof(int))) != BH_OK)
        return rc;

    // Pinned staging: [frames][binary64 treatment of mixed frames][ray ends]
    // [pixel ends][queue state].  The previous launch's copies out of it must
    // have completed.
    const size_t fbytes = static_cast<size_t>(p.nf) * sizeof(FrameParams);
    p.stage_bytes = fbytes + 2 * n * sizeof(long long) + sizeof(QueueState);
    CK(cudaEventSynchronize(ctx->stage_free));
    if (p.stage_bytes > ctx->stage_cap) {
        if (ctx->stage) CK(cudaFreeHost(ctx->stage));
        ctx->stage = nullptr;
        ctx->stage_cap = 0;
        CK(cudaHostAlloc(reinterpret_cast<void**>(&ctx->stage), p.stage_bytes, cudaHostAllocDefault));
        ctx->stage_cap = p.stage_bytes;
    }
    unsigned char* s = ctx->stage;
    std::memcpy(s, frames.data(), n * sizeof(FrameParams));
    for (int i = n; i < p.nf; ++i) {
        const FrameParams g = binary64_treatment(frames[i - n]);
        std::memcpy(s + i * sizeof(FrameParams), &g, sizeof g);
    }
    long long* ends = reinterpret_cast<long long*>(s + fbytes);
    for (int i = 0; i < n; ++i) {
        ends[i] = frames[i].ray_begin + frames[i].n_rays;
        ends[n + i] = frames[i].pixel_begin + static_cast<long long>(frames[i].width) * frames[i].height;
    }
    QueueState q;
    std::memset(&q, 0, sizeof q);
    q.budget = ctx->budget;
    q.abort = ctx->abort_requested.load() ? 1 : 0;
    std::memcpy(s + fbytes + 2 * n * sizeof(long long), &q, sizeof q);

    const int prec = frames[0].precision_tag;
    const bh_launch_params& lp = ctx->launch[prec == BH_PRECISION_MIXED ? 1 : 0];
    const bh_launch_params& lp64 = ctx->launch[0];
    int bps = lp.blocks_per_sm > 0 ? lp.blocks_per_sm : trace_blocks_per_sm(prec, lp.block_size, lp.reg_variant == 2);
    if (bps < 1) bps = 1;
    TraceLaunch& tl = p.tl;
    std::memset(&tl, 0, sizeof tl);
    tl.frames = static_cast<const FrameParams*>(ctx->frames.p);
    tl.frame_ray_end = static_cast<const long long*>(ctx->ray_end.p);
    tl.nframes = n;
    tl.total_rays = rays;
    tl.hits = static_cast<HitRecord*>(ctx->hits.p);
    tl.queue = ctx->d_queue;
    tl.precision = prec;
    tl.block_size = lp.block_size;
    tl.grid = ctx->sm_count * bps;
    tl.rays_per_thread = lp.rays_per_thread;
    tl.refill = lp.refill;
    tl.budget = ctx->budget;
    tl.deferred = p.mixed ? ctx->deferred.p : nullptr;
    tl.reg_variant = (lp.reg_variant == 2) ? 1 : 0;
    // The binary64 pass that finishes deferred mixed-precision rays: few rays
    // with long serial step chains, so it runs the spill-free (wide) register
    // variant in small blocks.
    tl.block_resume = 64;
    tl.reg_variant_resume = 1;
    {
        int bps64 = trace_blocks_per_sm(BH_PRECISION_FP64, tl.block_resume, true);
        tl.grid_resume = ctx->sm_count * (bps64 < 1 ? 1 : bps64);
    }
    tl.resume_event = timed ? ctx->ev[3] : nullptr;
    tl.jet = any_jet ? static_cast<double*>(ctx->jet.p) : nullptr;
    tl.surfaces = any_surface ? 1 : 0;
    if (p.mixed && any_near_critical) {
        // Near-critical rays in binary64 on kSideBlocks blocks beside the
        // binary32 kernel.  The binary32 grid gives up the slots those blocks
        // take, so that both are resident at once whichever is placed first;
        // as many binary32 blocks start in those slots after them.
        tl.near_critical = 1;
        tl.grid_side = std::min(kSideBlocks, ctx->sm_count);
        tl.frames_side = static_cast<const FrameParams*>(ctx->frames.p) + n;
        tl.side_stream = ctx->side_stream;
        tl.fork_event = ctx->fork_event;
        tl.join_event = ctx->join_event;
        tl.sel_flag = static_cast<unsigned char*>(ctx->sel_flag.p);
        tl.sel_list = static_cast<int*>(ctx->sel_list.p);
        tl.grid_list = ctx->sm_count * std::max(1, trace_blocks_per_sm(BH_PRECISION_FP64, 128, 0));
        if (lp.blocks_per_sm <= 0) {
            const long long side_regs = 4 * warp_regs(trace_registers(BH_PRECISION_FP64, 0));
            const long long block_regs = (lp.block_size / 32) * warp_regs(trace_registers(prec, tl.reg_variant));
            const int beside = block_regs > 0 ? static_cast<int>((kSmRegs - side_regs) / block_regs) : bps;
            const int lost = std::max(0, bps - std::max(0, beside));
            tl.grid_late = std::min(tl.grid - 1, tl.grid_side * lost);
            tl.grid -= tl.grid_late;
        }
    }

    ShadeLaunch& sl = p.sl;
    std::memset(&sl, 0, sizeof sl);
    sl.frames = tl.frames;
    sl.frame_pixel_end = static_cast<const long long*>(ctx->pix_end.p);
    sl.nframes = n;
    sl.total_pixels = pix;
    sl.hits = tl.hits;
    sl.sky = sky_data(ctx);
    sl.pixels = d_pixels;
    sl.rays = d_rays;
    sl.pixel_lum = static_cast<double*>(ctx->lum.p);
    sl.ray_class = nullptr;
    sl.jet = tl.jet;

    ReduceLaunch& rl = p.rl;
    std::memset(&rl, 0, sizeof rl);
    rl.frames = tl.frames;
    rl.nframes = n;
    rl.hits = tl.hits;
    rl.pixel_lum = sl.pixel_lum;
    rl.jet = tl.jet;
    rl.partials = static_cast<FrameStats*>(ctx->partials.p);
    rl.out = static_cast<FrameStats*>(ctx->fstats.p);
    rl.blocks_per_frame = kReduceBlocks;
    return BH_OK;
}

// Stream half: staging -> device copies, then the kernels.  No allocation and
// no host-synchronous call, so a CUDA graph can capture it.  Under capture the
// caller records `stage_free` after the graph launch instead (an event
// recorded during capture is not recorded again when the graph replays).
int record_launch(bh_ctx* ctx, const Plan& p, cudaStream_t stream, bool timed, bool captured = false) {
    const int n = p.n;
    const unsigned char* s = ctx->stage;
    const size_t fbytes = static_cast<size_t>(p.nf) * sizeof(FrameParams);
    CK(cudaMemcpyAsync(ctx->frames.p, s, fbytes, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(ctx->ray_end.p, s + fbytes, n * sizeof(long long), cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(ctx->pix_end.p, s + fbytes + n * sizeof(long long), n * sizeof(long long),
                       cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(ctx->d_queue, s + fbytes + 2 * n * sizeof(long long), sizeof(QueueState),
                       cudaMemcpyHostToDevice, stream));
    if (!captured) CK(cudaEventRecord(ctx->stage_free, stream));
    if (timed) CK(cudaEventRecord(ctx->ev[0], stream));
    if (p.rays > 0) CK(launch_trace(p.tl, stream));
    if (timed) CK(cudaEventRecord(ctx->ev[1], stream));
    CK(launch_shade(p.sl, stream));
    if (timed) CK(cudaEventRecord(ctx->ev[2], stream));
    CK(launch_reduce(p.rl, stream));
    return BH_OK;
}

// ---- bh_gpu_render's row-band pipeline -------------------------------------
// The frame's rays are handed out in pixel order, so its rows finish roughly
// in order while the trace runs.  The trace kernels count each band's
// finished rays; a stream waits (in the GPU's front end, not
// on an SM) for each band's count, shades that band and copies its rows to
// the host while the rest of the frame is still being traced.  The binary32
// trace grid may give up kBandReserveBlocks block slots for the shading
// (measured: none is best; the band streams have the trace's priority, a
// higher one, or slots left free, both slowed the trace more than they
// gained).  The bands go round kBandStreams
// streams, so a band whose rays finish late (the photon ring's) holds up only
// the bands that share its stream.
constexpr int kBandRows = 64;              // rows per band (a multiple of the 4-row pixel order)
constexpr int kBandReserveBlocks = 0;
constexpr int kBandStreams = 8;
static_assert(kBandStreams <= 8, "bh_ctx holds 8 band streams");

void setup_band_pipeline(bh_ctx* ctx) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuStreamWaitValue32", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
        cudaGetLastError();
        return;
    }
    for (int i = 0; i < kBandStreams; ++i)
        if (cudaStreamCreateWithFlags(&ctx->band_stream[i], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->band_join[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
    // The wait must work here: one on a word this stream has just zeroed
    // (the queue's first counter, zero anyway) returns at once.
    auto wait = reinterpret_cast<CUresult (*)(CUstream, CUdeviceptr, cuuint32_t, unsigned int)>(fn);
    if (cudaMemsetAsync(ctx->d_queue, 0, sizeof(unsigned int), ctx->band_stream[0]) != cudaSuccess ||
        wait(ctx->band_stream[0], reinterpret_cast<CUdeviceptr>(ctx->d_queue), 0u, CU_STREAM_WAIT_VALUE_GEQ) !=
            CUDA_SUCCESS ||
        cudaStreamSynchronize(ctx->band_stream[0]) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    ctx->wait_value32 = wait;
}

// The launch of plan `p` (one frame, d_pixels on the device) with its rows
// shaded and copied to `out_pixels` band by band as they finish.
int record_banded(bh_ctx* ctx, Plan& p, const bh_render_config* cfg, bh_xyz* out_pixels, cudaStream_t stream) {
    const int W = cfg->width, H = cfg->height;
    const int S = cfg->sqrt_spp > 1 ? cfg->sqrt_spp : 1;
    const int nb = (H + kBandRows - 1) / kBandRows;
    const long long px_band = static_cast<long long>(kBandRows) * W;
    int rc;
    if ((rc = ensure(ctx, ctx->band_done, static_cast<size_t>(nb) * sizeof(unsigned int))) != BH_OK) return rc;
    unsigned int* done = static_cast<unsigned int*>(ctx->band_done.p);
    p.tl.band_done = done;
    p.tl.rays_per_band = px_band * S * S;
    p.tl.nbands = nb;
    if (kBandReserveBlocks > 0 && p.tl.grid > 2 * kBandReserveBlocks) p.tl.grid -= kBandReserveBlocks;
    const unsigned char* st = ctx->stage;
    const size_t fbytes = static_cast<size_t>(p.nf) * sizeof(FrameParams);
    CK(cudaMemcpyAsync(ctx->frames.p, st, fbytes, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(ctx->ray_end.p, st + fbytes, sizeof(long long), cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(ctx->pix_end.p, st + fbytes + sizeof(long long), sizeof(long long), cudaMemcpyHostToDevice,
                       stream));
    CK(cudaMemcpyAsync(ctx->d_queue, st + fbytes + 2 * sizeof(long long), sizeof(QueueState), cudaMemcpyHostToDevice,
                       stream));
    CK(cudaEventRecord(ctx->stage_free, stream));
    CK(cudaMemsetAsync(done, 0, static_cast<size_t>(nb) * sizeof(unsigned int), stream));
    CK(cudaEventRecord(ctx->ev[0], stream));
    // The band streams start once the counters are cleared.
    const int ns = std::min(nb, kBandStreams);
    for (int i = 0; i < ns; ++i) CK(cudaStreamWaitEvent(ctx->band_stream[i], ctx->ev[0], 0));
    if (p.rays > 0) CK(launch_trace(p.tl, stream));
    CK(cudaEventRecord(ctx->ev[1], stream));
    const long long npx = static_cast<long long>(W) * H;
    for (int b = 0; b < nb; ++b) {
        cudaStream_t bs = ctx->band_stream[b % ns];
        const long long lo = b * px_band;
        const long long hi = std::min(npx, lo + px_band);
        const long long rays = (hi - lo) * S * S;
        if (ctx->wait_value32(bs, reinterpret_cast<CUdeviceptr>(done + b), static_cast<cuuint32_t>(rays),
                              CU_STREAM_WAIT_VALUE_GEQ) != CUDA_SUCCESS)
            return fail(ctx, BH_ERR_CUDA, "stream wait on a row band failed");
        ShadeLaunch sl = p.sl;
        sl.pixel_lo = lo;
        sl.total_pixels = hi;
        CK(launch_shade(sl, bs));
        CK(cudaMemcpyAsync(out_pixels + lo, static_cast<bh_xyz*>(ctx->pixels.p) + lo,
                           static_cast<size_t>(hi - lo) * sizeof(bh_xyz), cudaMemcpyDeviceToHost, bs));
    }
    for (int i = 0; i < ns; ++i) {
        CK(cudaEventRecord(ctx->band_join[i], ctx->band_stream[i]));
        CK(cudaStreamWaitEvent(stream, ctx->band_join[i], 0));
    }
    CK(cudaEventRecord(ctx->ev[2], stream));
    CK(launch_reduce(p.rl, stream));
    ctx->d2h += npx * static_cast<long long>(sizeof(bh_xyz));
    return BH_OK;
}

int enqueue(bh_ctx* ctx, std::vector<FrameParams>& frames, bh_xyz* d_pixels, bh_ray_result* d_rays,
            cudaStream_t stream, bool timed) {
    Plan p;
    int rc = plan_launch(ctx, frames, d_pixels, d_rays, timed, p);
    if (rc != BH_OK) return rc;
    ctx->h2d += static_cast<long long>(p.stage_bytes);
    return record_launch(ctx, p, stream, timed);
}

constexpr size_t kReadbackBytes = sizeof(QueueState) + sizeof(FrameStats);

// Enqueue the copies of a single-frame launch's queue state and stats into
// the pinned read-back buffer (read by finish(..., prefetched = true) once
// the stream has drained), so the call synchronises once.
int enqueue_readback(bh_ctx* ctx, cudaStream_t stream) {
    CK(cudaMemcpyAsync(ctx->h_readback, ctx->d_queue, sizeof(QueueState), cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(ctx->h_readback + sizeof(QueueState), ctx->fstats.p, sizeof(FrameStats),
                       cudaMemcpyDeviceToHost, stream));
    return BH_OK;
}

// Read back the queue state and per-frame stats after the stream drained
// (from the read-back buffer when enqueue_readback filled it).
int finish(bh_ctx* ctx, int n, bh_render_stats* per_frame, bh_render_stats* total, bool timed,
           double seconds, bool prefetched = false) {
    QueueState q;
    std::vector<FrameStats> fs(n);
    if (prefetched && n == 1) {
        std::memcpy(&q, ctx->h_readback, sizeof q);
        std::memcpy(fs.data(), ctx->h_readback + sizeof(QueueState), sizeof(FrameStats));
    } else {
        CK(cudaMemcpy(&q, ctx->d_queue, sizeof q, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(fs.data(), ctx->fstats.p, n * sizeof(FrameStats), cudaMemcpyDeviceToHost));
    }
    ctx->d2h += static_cast<long long>(sizeof q + n * sizeof(FrameStats));
    float t_trace = 0.f, t_shade = 0.f;
    if (timed) {
        CK(cudaEventElapsedTime(&t_trace, ctx->ev[0], ctx->ev[1]));
        CK(cudaEventElapsedTime(&t_shade, ctx->ev[1], ctx->ev[2]));
    }
    for (int i = 0; i < n; ++i) {
        if (per_frame) {
            stats_add(&per_frame[i], fs[i]);
            per_frame[i].seconds = seconds;
            per_frame[i].kernel_ms = t_trace;
            per_frame[i].shade_ms = t_shade;
            if (i == 0) {
                per_frame[i].h2d_bytes += ctx->h2d;
                per_frame[i].d2h_bytes += ctx->d2h;
            }
        }
        if (total) stats_add(total, fs[i]);
    }
    if (total) {
        total->h2d_bytes += ctx->h2d;
        total->d2h_bytes += ctx->d2h;
        total->seconds = seconds;
        total->kernel_ms = t_trace;
        total->shade_ms = t_shade;
    }
    if (q.abort == 1) return fail(ctx, BH_ERR_ABORTED, "launch aborted by bh_gpu_request_abort");
    if (q.abort == 2) return fail(ctx, BH_ERR_BUDGET, "step budget of the launch exhausted");
    return BH_OK;
}

int prepare_frames(bh_ctx* ctx, const bh_render_config* cfgs, int n, std::vector<FrameParams>& frames) {
    ctx->h2d = 0;
    ctx->d2h = 0;
    frames.resize(n);
    for (int i = 0; i < n; ++i) {
        int rc = check_cfg_header(ctx, &cfgs[i]);
        if (rc != BH_OK) return rc;
        std::string err;
        rc = make_frame(cfgs[i], frames[i], err);
        if (rc != BH_OK) return fail(ctx, rc, n > 1 ? "frame " + std::to_string(i) + ": " + err : err);
        frames[i].precision_tag = cfgs[i].precision;
        if (i > 0) {
            if (cfgs[i].precision != cfgs[0].precision)
                return fail(ctx, BH_ERR_INVALID_ARG, "all frames of a batch must share the precision");
            if ((cfgs[i].stars_enabled != 0) != (cfgs[0].stars_enabled != 0) ||
                (cfgs[i].stars_enabled && (cfgs[i].star_count != cfgs[0].star_count ||
                                           cfgs[i].seed != cfgs[0].seed ||
                                           cfgs[i].sky_mode != cfgs[0].sky_mode)))
                return fail(ctx, BH_ERR_INVALID_ARG, "all frames of a batch must share the star catalogue");
        }
    }
    return ensure_sky(ctx, cfgs[0]);
}

}  // namespace

extern "C" {

int bh_gpu_abi_version(void) { return BH_GPU_ABI_VERSION; }

void bh_render_config_default(bh_render_config* cfg) {
    if (cfg) default_config(*cfg);
}

int bh_gpu_create(int device, bh_ctx** out) {
    if (!out) return BH_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return BH_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return BH_ERR_INVALID_ARG;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return BH_ERR_NO_DEVICE;
    if (prop.major != 10) return BH_ERR_NO_DEVICE;   // built for sm_100a only
    bh_ctx* ctx = new bh_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    auto bail = [&](cudaError_t e) {
        bh_gpu_destroy(ctx);
        return e == cudaErrorMemoryAllocation ? BH_ERR_OUT_OF_MEMORY : BH_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return bail(e);
    if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e);
    if ((e = cudaStreamCreateWithFlags(&ctx->abort_stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e);
    if ((e = cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e);
    if ((e = cudaEventCreateWithFlags(&ctx->fork_event, cudaEventDisableTiming)) != cudaSuccess) return bail(e);
    if ((e = cudaEventCreateWithFlags(&ctx->join_event, cudaEventDisableTiming)) != cudaSuccess) return bail(e);
    if ((e = cudaMalloc(&ctx->d_queue, sizeof(QueueState))) != cudaSuccess) return bail(e);
    if ((e = cudaMemset(ctx->d_queue, 0, sizeof(QueueState))) != cudaSuccess) return bail(e);
    if ((e = cudaHostAlloc(&ctx->h_one, sizeof(int32_t), cudaHostAllocDefault)) != cudaSuccess) return bail(e);
    *ctx->h_one = 1;
    if ((e = cudaHostAlloc(reinterpret_cast<void**>(&ctx->h_readback), kReadbackBytes, cudaHostAllocDefault)) !=
        cudaSuccess)
        return bail(e);
    setup_band_pipeline(ctx);
    for (auto& ev : ctx->ev)
        if ((e = cudaEventCreate(&ev)) != cudaSuccess) return bail(e);
    if ((e = cudaEventCreateWithFlags(&ctx->stage_free, cudaEventDisableTiming)) != cudaSuccess) return bail(e);
    *out = ctx;
    return BH_OK;
}

void bh_gpu_destroy(bh_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (DevBuf* b : {&ctx->hits, &ctx->pixels, &ctx->rays, &ctx->lum, &ctx->frames, &ctx->ray_end, &ctx->deferred,
                      &ctx->pix_end, &ctx->partials, &ctx->fstats, &ctx->jet, &ctx->adj_target, &ctx->adj_grad, &ctx->adj_Y,
                      &ctx->adj_ckpt, &ctx->adj_counters, &ctx->adj_sums, &ctx->adj_xr, &ctx->adj_cand, &ctx->adj_edge,
                      &ctx->adj_high, &ctx->eval_in, &ctx->eval_out, &ctx->disp_tmp, &ctx->disp_near,
                      &ctx->disp_far, &ctx->disp_k, &ctx->disp_state, &ctx->disp_rgb, &ctx->sel_flag,
                      &ctx->sel_list, &ctx->band_done})
        if (b->p) cudaFree(b->p);
    cudaFree(ctx->d_table);
    cudaFree(ctx->d_star_pos);
    cudaFree(ctx->d_star_col);
    cudaFree(ctx->d_bin_start);
    cudaFree(ctx->d_queue);
    if (ctx->h_one) cudaFreeHost(ctx->h_one);
    if (ctx->h_readback) cudaFreeHost(ctx->h_readback);
    for (cudaStream_t st : ctx->band_stream)
        if (st) cudaStreamDestroy(st);
    for (cudaEvent_t ev : ctx->band_join)
        if (ev) cudaEventDestroy(ev);
    if (ctx->batch_exec) cudaGraphExecDestroy(ctx->batch_exec);
    if (ctx->stage) cudaFreeHost(ctx->stage);
    if (ctx->stage_free) cudaEventDestroy(ctx->stage_free);
    for (auto& ev : ctx->ev)
        if (ev) cudaEventDestroy(ev);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->abort_stream) cudaStreamDestroy(ctx->abort_stream);
    if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
    if (ctx->fork_event) cudaEventDestroy(ctx->fork_event);
    if (ctx->join_event) cudaEventDestroy(ctx->join_event);
    delete ctx;
}

const char* bh_gpu_last_error(const bh_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int bh_gpu_render(bh_ctx* ctx, const bh_render_config* cfg, bh_xyz* out_pixels, bh_render_stats* stats) {
    if (!ctx) return BH_ERR_INVALID_ARG;
    if (!out_pixels) return fail(ctx, BH_ERR_INVALID_ARG, "out_pixels is NULL");
    const auto t0 = std::chrono::steady_clock::now();
    CK(cudaSetDevice(ctx->device));
    std::vector<FrameParams> frames;
    int rc = prepare_frames(ctx, cfg, 1, frames);
    if (rc != BH_OK) return rc;
    const size_t npx = static_cast<size_t>(cfg->width) * cfg->height;
    if ((rc = ensure(ctx, ctx->pixels, npx * sizeof(bh_xyz))) != BH_OK) return rc;
    if (ctx->wait_value32 && cfg->height >= 2 * kBandRows) {
        // rows shaded and copied out band by band while the frame is traced
        Plan p;
        if ((rc = plan_launch(ctx, frames, static_cast<bh_xyz*>(ctx->pixels.p), nullptr, true, p)) != BH_OK)
            return rc;
        ctx->h2d += static_cast<long long>(p.stage_bytes);
        if ((rc = record_banded(ctx, p, cfg, out_pixels, ctx->stream)) != BH_OK) return rc;
    } else {
        rc = enqueue(ctx, frames, static_cast<bh_xyz*>(ctx->pixels.p), nullptr, ctx->stream, true);
        if (rc != BH_OK) return rc;
        CK(cudaMemcpyAsync(out_pixels, ctx->pixels.p, npx * sizeof(bh_xyz), cudaMemcpyDeviceToHost, ctx->stream));
        ctx->d2h += static_cast<long long>(npx * sizeof(bh_xyz));
    }
    if ((rc = enqueue_readback(ctx, ctx->stream)) != BH_OK) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    bh_render_stats local;
    std::memset(&local, 0, sizeof local);
    rc = finish(ctx, 1, nullptr, &local, true, secs, true);
    if (stats) {
        bh_render_stats s = local;
        stats->rays += s.rays; stats->steps += s.steps; stats->captured += s.captured;
        stats->disc_hits += s.disc_hits; stats->sun_hits += s.sun_hits; stats->star_hits += s.star_hits;
        stats->jet_rays += s.jet_rays; stats->escaped += s.escaped; stats->exhausted += s.exhausted;
        stats->total_flux += s.total_flux; stats->attempts += s.attempts;
        stats->max_norm_error = std::max(stats->max_norm_error, s.max_norm_error);
        stats->max_carter_drift = std::max(stats->max_carter_drift, s.max_carter_drift);
        stats->seconds = s.seconds;
        stats->kernel_ms = s.kernel_ms;
        stats->shade_ms = s.shade_ms;
        stats->h2d_bytes += s.h2d_bytes;
        stats->d2h_bytes += s.d2h_bytes;
    }
    return rc;
}

int bh_gpu_render_device(bh_ctx* ctx, const bh_render_config* cfg, bh_xyz* d_pixels, bh_render_stats* stats,
                         void* stream) {
    if (!ctx) return BH_ERR_INVALID_ARG;
    if (!d_pixels) return fail(ctx, BH_ERR_INVALID_ARG, "d_pixels is NULL");
    const auto t0 = std::chrono::steady_clock::now();
    CK(cudaSetDevice(ctx->device));
    std::vector<FrameParams> frames;
    int rc = prepare_frames(ctx, cfg, 1, frames);
    if (rc != BH_OK) return rc;
    // NULL is the legacy default stream, ordered with the caller's other
    // default-stream work (the context's own stream is non-blocking).
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
    rc = enqueue(ctx, frames, d_pixels, nullptr, s, stats != nullptr);
    if (rc != BH_OK || !stats) return rc;
    if ((rc = enqueue_readback(ctx, s)) != BH_OK) return rc;
    CK(cudaStreamSynchronize(s));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return finish(ctx, 1, stats, nullptr, true, secs, true);
}

int bh_gpu_trace_rays(bh_ctx* ctx, const bh_render_config* cfg, bh_ray_result* out, bh_render_stats* stats) {
    if (!ctx) return BH_ERR_INVALID_ARG;
    if (!out) return fail(ctx, BH_ERR_INVALID_ARG, "out is NULL");
    const auto t0 = std::chrono::steady_clock::now();
    CK(cudaSetDevice(ctx->device));
    std::vector<FrameParams> frames;
    int rc = prepare_frames(ctx, cfg, 1, frames);
    if (rc != BH_OK) return rc;
    const size_t npx = static_cast<size_t>(cfg->width) * cfg->height;
    const size_t nr = static_cast<size_t>(frames[0].n_rays);
    if ((rc = ensure(ctx, ctx->pixels, npx * sizeof(bh_xyz))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->rays, nr * sizeof(bh_ray_result))) != BH_OK) return rc;
    rc = enqueue(ctx, frames, static_cast<bh_xyz*>(ctx->pixels.p), static_cast<bh_ray_result*>(ctx->rays.p),
                 ctx->stream, true);
    if (rc != BH_OK) return rc;
    CK(cudaMemcpyAsync(out, ctx->rays.p, nr * sizeof(bh_ray_result), cudaMemcpyDeviceToHost, ctx->stream));
    ctx->d2h += static_cast<long long>(nr * sizeof(bh_ray_result));
    if ((rc = enqueue_readback(ctx, ctx->stream)) != BH_OK) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return finish(ctx, 1, stats, nullptr, true, secs, true);
}

int bh_gpu_render_batch(bh_ctx* ctx, const bh_render_config* cfgs, int n, bh_xyz* const* outs,
                        bh_render_stats* stats) {
    if (!ctx) return BH_ERR_INVALID_ARG;
    if (!cfgs || n <= 0 || !outs) return fail(ctx, BH_ERR_INVALID_ARG, "empty batch");
    for (int i = 0; i < n; ++i)
        if (!outs[i]) return fail(ctx, BH_ERR_INVALID_ARG, "outs[" + std::to_string(i) + "] is NULL");
    const auto t0 = std::chrono::steady_clock::now();
    CK(cudaSetDevice(ctx->device));
    std::vector<FrameParams> frames;
    int rc = prepare_frames(ctx, cfgs, n, frames);
    if (rc != BH_OK) return rc;
    size_t npx = 0;
    for (int i = 0; i < n; ++i) npx += static_cast<size_t>(cfgs[i].width) * cfgs[i].height;
    if ((rc = ensure(ctx, ctx->pixels, npx * sizeof(bh_xyz))) != BH_OK) return rc;
    // The whole batch is one CUDA graph: staging copies, the persistent trace
    // launch over every frame's rays (plus the binary64 pass), shading and the
    // stats.  It is captured once per batch shape and replayed while the shape
    // (frame count, sizes, buffers, launch shape) stays the same; the frame
    // constants change freely, they are read from the pinned staging buffer.
    Plan p;
    if ((rc = plan_launch(ctx, frames, static_cast<bh_xyz*>(ctx->pixels.p), nullptr, false, p)) != BH_OK)
        return rc;
    ctx->h2d += static_cast<long long>(p.stage_bytes);
    std::vector<unsigned char> key(sizeof p.tl + sizeof p.sl + sizeof p.rl + sizeof(void*) + sizeof(size_t));
    {
        unsigned char* k = key.data();
        std::memcpy(k, &p.tl, sizeof p.tl); k += sizeof p.tl;
        std::memcpy(k, &p.sl, sizeof p.sl); k += sizeof p.sl;
        std::memcpy(k, &p.rl, sizeof p.rl); k += sizeof p.rl;
        std::memcpy(k, &ctx->stage, sizeof(void*)); k += sizeof(void*);
        std::memcpy(k, &p.stage_bytes, sizeof(size_t));
    }
    if (!ctx->batch_exec || key != ctx->batch_key) {
        if (ctx->batch_exec) {
            cudaGraphExecDestroy(ctx->batch_exec);
            ctx->batch_exec = nullptr;
        }
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        const int rrc = record_launch(ctx, p, ctx->stream, false, true);
        const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
        if (rrc != BH_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rrc;
        }
        CK(ce);
        const cudaError_t ie = cudaGraphInstantiate(&ctx->batch_exec, graph, 0);
        cudaGraphDestroy(graph);
        CK(ie);
        ctx->batch_key = key;
    }
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    CK(cudaGraphLaunch(ctx->batch_exec, ctx->stream));
    CK(cudaEventRecord(ctx->stage_free, ctx->stream));
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    size_t off = 0;
    for (int i = 0; i < n; ++i) {
        const size_t m = static_cast<size_t>(cfgs[i].width) * cfgs[i].height;
        CK(cudaMemcpyAsync(outs[i], static_cast<bh_xyz*>(ctx->pixels.p) + off, m * sizeof(bh_xyz),
                           cudaMemcpyDeviceToHost, ctx->stream));
        off += m;
        ctx->d2h += static_cast<long long>(m * sizeof(bh_xyz));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return finish(ctx, n, stats, nullptr, true, secs);
}

// The binary64 render of `cfg` (its loss against `target`) and the discrete
// adjoint of that loss; per-ray gradients and luminances on request.
static int adjoint_impl(bh_ctx* ctx, const bh_render_config* cfg, const float* target, bh_grad4* out,
                        double* ray_grad, double* ray_Y) {
    if (!ctx) return BH_ERR_INVALID_ARG;
    if (!target || !out) return fail(ctx, BH_ERR_INVALID_ARG, "target and out must not be NULL");
    int rc = check_cfg_header(ctx, cfg);
    if (rc != BH_OK) return rc;
    const auto t0 = std::chrono::steady_clock::now();
    CK(cudaSetDevice(ctx->device));
    bh_render_config c = *cfg;
    c.precision = BH_PRECISION_FP64;       // the adjoint differentiates the binary64 path
    std::vector<FrameParams> frames;
    if ((rc = prepare_frames(ctx, &c, 1, frames)) != BH_OK) return rc;
    AdjointFrame X;
    {
        std::string err;
        if ((rc = make_adjoint_frame(c, frames[0], X, err)) != BH_OK) return fail(ctx, rc, err);
    }
    const int block = 128;
    int bps = adjoint_blocks_per_sm(block);
    if (bps < 1) bps = 1;
    const int grid = ctx->sm_count * bps;
    const size_t npx = static_cast<size_t>(c.width) * c.height;
    const long long n_rays = frames[0].n_rays;
    if ((rc = ensure(ctx, ctx->pixels, npx * sizeof(bh_xyz))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->adj_target, npx * sizeof(float))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->adj_grad, static_cast<size_t>(n_rays) * 4 * sizeof(double))) != BH_OK) return rc;
    if (ray_Y && (rc = ensure(ctx, ctx->adj_Y, static_cast<size_t>(n_rays) * sizeof(double))) != BH_OK) return rc;
    const size_t ck_bytes = static_cast<size_t>(grid) * block * X.checkpoint_slots * 8 * sizeof(double);
    if ((rc = ensure(ctx, ctx->adj_ckpt, ck_bytes)) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->adj_counters, kAdjCounters * sizeof(unsigned long long))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->adj_sums, kAdjSums * sizeof(double))) != BH_OK) return rc;
    const size_t n_slots = static_cast<size_t>(n_rays) * 2;     // two equatorial crossings per ray
    if ((rc = ensure(ctx, ctx->adj_xr, n_slots * sizeof(double))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->adj_cand, n_slots * sizeof(unsigned long long))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->adj_edge, n_slots * 3 * sizeof(double))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->adj_high, static_cast<size_t>(n_rays))) != BH_OK) return rc;

    CK(cudaMemcpyAsync(ctx->adj_target.p, target, npx * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    ctx->h2d += static_cast<long long>(npx * sizeof(float));
    CK(cudaMemsetAsync(ctx->adj_xr.p, 0, n_slots * sizeof(double), ctx->stream));
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    {
        // the render, recording each ray's first two equatorial crossings
        Plan p;
        if ((rc = plan_launch(ctx, frames, static_cast<bh_xyz*>(ctx->pixels.p), nullptr, false, p)) != BH_OK)
            return rc;
        p.tl.xing = static_cast<double*>(ctx->adj_xr.p);
        ctx->h2d += static_cast<long long>(p.stage_bytes);
        if ((rc = record_launch(ctx, p, ctx->stream, false)) != BH_OK) return rc;
    }
    CK(cudaMemsetAsync(ctx->adj_counters.p, 0, kAdjCounters * sizeof(unsigned long long), ctx->stream));
    CK(cudaMemsetAsync(ctx->adj_edge.p, 0, n_slots * 3 * sizeof(double), ctx->stream));
    AdjointLaunch L;
    std::memset(&L, 0, sizeof L);
    L.frame = frames[0];
    L.X = X;
    L.sky = sky_data(ctx);
    L.pixels = static_cast<const bh_xyz*>(ctx->pixels.p);
    L.target = static_cast<const float*>(ctx->adj_target.p);
    L.ray_grad = static_cast<double*>(ctx->adj_grad.p);
    L.ray_Y = ray_Y ? static_cast<double*>(ctx->adj_Y.p) : nullptr;
    L.ckpt = static_cast<double*>(ctx->adj_ckpt.p);
    L.xing_r = static_cast<double*>(ctx->adj_xr.p);
    L.cand = static_cast<unsigned long long*>(ctx->adj_cand.p);
    L.edge_out = static_cast<double*>(ctx->adj_edge.p);
    L.high_order = static_cast<unsigned char*>(ctx->adj_high.p);
    L.counters = static_cast<unsigned long long*>(ctx->adj_counters.p);
    L.sums = static_cast<double*>(ctx->adj_sums.p);
    L.n_rays = n_rays;
    L.grid = grid;
    L.block = block;
    CK(launch_adjoint(L, ctx->stream));
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    double sums[kAdjSums];
    unsigned long long cnt[kAdjCounters];
    CK(cudaMemcpyAsync(sums, ctx->adj_sums.p, sizeof sums, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(cnt, ctx->adj_counters.p, sizeof cnt, cudaMemcpyDeviceToHost, ctx->stream));
    if (ray_grad)
        CK(cudaMemcpyAsync(ray_grad, ctx->adj_grad.p, static_cast<size_t>(n_rays) * 4 * sizeof(double),
                           cudaMemcpyDeviceToHost, ctx->stream));
    if (ray_Y)
        CK(cudaMemcpyAsync(ray_Y, ctx->adj_Y.p, static_cast<size_t>(n_rays) * sizeof(double),
                           cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if ((rc = finish(ctx, 1, nullptr, nullptr, false, secs)) != BH_OK) return rc;
    std::memset(out, 0, sizeof *out);
    out->loss = sums[0];
    out->d_spin = sums[1] + sums[6];
    out->d_inclination = sums[2] + sums[7];
    out->d_eddington = sums[3];
    out->d_r_out = sums[4] + sums[5];
    out->edge_spin = sums[6];
    out->edge_inclination = sums[7];
    out->edge_candidates = static_cast<long long>(cnt[6]);
    out->edge_steps = static_cast<long long>(cnt[7]);
    out->edge_cells = static_cast<long long>(cnt[8]);
    out->held_spin = sums[8];
    out->held_inclination = sums[9];
    out->high_order_rays = static_cast<long long>(cnt[9]);
    out->kernel_ms = ms;
    out->rays = n_rays;
    out->steps = static_cast<long long>(cnt[1]);
    out->replayed_steps = static_cast<long long>(cnt[2]);
    out->disc_rays = static_cast<long long>(cnt[3]);
    out->sky_rays = static_cast<long long>(cnt[4]);
    out->max_checkpoint_interval = static_cast<int32_t>(cnt[5]);
    return BH_OK;
}

// The display transform of the W x H frame at d_pixels (device), on
// ctx->stream; copies the 8-bit image and the exposure back and synchronises.
static int display_impl(bh_ctx* ctx, const bh_display* d, bh_xyz* d_pixels, int width, int height,
                        uint8_t* out_rgb, double* exposure_used) {
    if (!(d->glare >= 0.0 && d->glare <= 1.0)) return fail(ctx, BH_ERR_INVALID_ARG, "glare must be in [0, 1]");
    if (d->tonemap < BH_TONEMAP_LINEAR || d->tonemap > BH_TONEMAP_HDR)
        return fail(ctx, BH_ERR_INVALID_ARG, "unknown tonemap");
    const size_t npx = static_cast<size_t>(width) * height;
    int rc;
    DisplayLaunch L;
    std::memset(&L, 0, sizeof L);
    L.pixels = d_pixels;
    L.width = width;
    L.height = height;
    L.glare = d->glare;
    L.glare_radius = d->glare_radius;
    if (d->glare > 0.0 && d->glare_radius > 0.0) {
        // img::add_glare's kernels (image.cpp:61-68), normalised on the host.
        std::vector<double> w;
        int r[2];
        for (int j = 0; j < 2; ++j) {
            const double sigma = (j == 0) ? d->glare_radius : d->glare_radius * 3.0;
            r[j] = std::max(1, static_cast<int>(std::ceil(3.0 * sigma)));
            std::vector<double> k(2 * r[j] + 1);
            double sum = 0.0;
            for (int i = -r[j]; i <= r[j]; ++i) {
                k[i + r[j]] = std::exp(-0.5 * (i * i) / (sigma * sigma));
                sum += k[i + r[j]];
            }
            for (double& v : k) v /= sum;
            w.insert(w.end(), k.begin(), k.end());
        }
        if ((rc = ensure(ctx, ctx->disp_k, w.size() * sizeof(double))) != BH_OK) return rc;
        for (DevBuf* b : {&ctx->disp_tmp, &ctx->disp_near, &ctx->disp_far})
            if ((rc = ensure(ctx, *b, npx * sizeof(bh_xyz))) != BH_OK) return rc;
        CK(cudaMemcpyAsync(ctx->disp_k.p, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice,
                           ctx->stream));
        ctx->h2d += static_cast<long long>(w.size() * sizeof(double));
        L.k_near = static_cast<const double*>(ctx->disp_k.p);
        L.k_far = L.k_near + (2 * r[0] + 1);
        L.r_near = r[0];
        L.r_far = r[1];
        L.tmp = static_cast<bh_xyz*>(ctx->disp_tmp.p);
        L.nearp = static_cast<bh_xyz*>(ctx->disp_near.p);
        L.farp = static_cast<bh_xyz*>(ctx->disp_far.p);
    }
    if ((rc = ensure(ctx, ctx->disp_state, sizeof(ExposureState) + 2 * sizeof(double))) != BH_OK) return rc;
    if (out_rgb && (rc = ensure(ctx, ctx->disp_rgb, npx * 3)) != BH_OK) return rc;
    L.exposure = d->exposure;
    L.key = d->key;
    L.state = static_cast<ExposureState*>(ctx->disp_state.p);
    L.exposure_out = reinterpret_cast<double*>(static_cast<unsigned char*>(ctx->disp_state.p) + sizeof(ExposureState));
    L.reduce_blocks = ctx->sm_count * 4;
    L.tonemap = d->tonemap;
    L.log_k = std::pow(10.0, std::min(std::max(d->log_decades, 1.0), 20.0));
    L.denom = std::log10(1.0 + L.log_k);
    L.rgb = out_rgb ? static_cast<uint8_t*>(ctx->disp_rgb.p) : nullptr;
    CK(launch_display(L, ctx->stream));
    double e = 0.0;
    CK(cudaMemcpyAsync(&e, L.exposure_out, sizeof e, cudaMemcpyDeviceToHost, ctx->stream));
    if (out_rgb) CK(cudaMemcpyAsync(out_rgb, ctx->disp_rgb.p, npx * 3, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->d2h += static_cast<long long>(sizeof e + (out_rgb ? npx * 3 : 0));
    if (exposure_used) *exposure_used = e;
    return BH_OK;
}

void bh_jet_configure(bh_jet* jet, double spin, double mdot_c2, double r_g_m) {
    if (jet) jet_configure(*jet, spin, mdot_c2, r_g_m);
}

int bh_render_config_setup_jet(bh_render_config* cfg) {
    if (!cfg) return BH_ERR_INVALID_ARG;
    return setup_jet(*cfg);
}

void bh_display_default(bh_display* d) {
    if (!d) return;
    std::memset(d, 0, sizeof *d);
    d->exposure = 0.0;
    d->key = 1.0;
    d->glare = 0.0;
    d->glare_radius = 3.0;
    d->log_decades = 16.0;
    d->tonemap = BH_TONEMAP_HDR;
}

int bh_gpu_develop(bh_ctx* ctx, const bh_xyz* pixels, int width, int height, const bh_display* d,
                   uint8_t* out_rgb, double* exposure_used) {
    if (!ctx) return BH_ERR_INVALID_ARG;
    if (!pixels || !d) return fail(ctx, BH_ERR_INVALID_ARG, "pixels and display settings must not be NULL");
    if (width <= 0 || height <= 0) return fail(ctx, BH_ERR_INVALID_ARG, "width and height must be positive");
    CK(cudaSetDevice(ctx->device));
    ctx->h2d = 0;
    ctx->d2h = 0;
    const size_t npx = static_cast<size_t>(width) * height;
    int rc;
    if ((rc = ensure(ctx, ctx->pixels, npx * sizeof(bh_xyz))) != BH_OK) return rc;
    CK(cudaMemcpyAsync(ctx->pixels.p, pixels, npx * sizeof(bh_xyz), cudaMemcpyHostToDevice, ctx->stream));
    ctx->h2d += static_cast<long long>(npx * sizeof(bh_xyz));
    return display_impl(ctx, d, static_cast<bh_xyz*>(ctx->pixels.p), width, height, out_rgb, exposure_used);
}

int bh_gpu_render_rgb(bh_ctx* ctx, const bh_render_config* cfg, const bh_display* d, uint8_t* out_rgb,
                      double* exposure_used, bh_render_stats* stats) {
    if (!ctx) return BH_ERR_INVALID_ARG;
    if (!d) return fail(ctx, BH_ERR_INVALID_ARG, "display settings must not be NULL");
    const auto t0 = std::chrono::steady_clock::now();
    CK(cudaSetDevice(ctx->device));
    std::vector<FrameParams> frames;
    int rc = prepare_frames(ctx, cfg, 1, frames);
    if (rc != BH_OK) return rc;
    const size_t npx = static_cast<size_t>(cfg->width) * cfg->height;
    if ((rc = ensure(ctx, ctx->pixels, npx * sizeof(bh_xyz))) != BH_OK) return rc;
    if ((rc = enqueue(ctx, frames, static_cast<bh_xyz*>(ctx->pixels.p), nullptr, ctx->stream, true)) != BH_OK)
        return rc;
    if ((rc = display_impl(ctx, d, static_cast<bh_xyz*>(ctx->pixels.p), cfg->width, cfg->height, out_rgb,
                           exposure_used)) != BH_OK)
        return rc;
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return finish(ctx, 1, stats, nullptr, true, secs);
}

int bh_gpu_render_batch_rgb(bh_ctx* ctx, const bh_render_config* cfgs, int n, const bh_display* d,
                            uint8_t* const* outs_rgb, double* exposure_used, bh_render_stats* stats) {
    if (!ctx) return BH_ERR_INVALID_ARG;
    if (!cfgs || n <= 0 || !outs_rgb || !d) return fail(ctx, BH_ERR_INVALID_ARG, "empty batch");
    const auto t0 = std::chrono::steady_clock::now();
    CK(cudaSetDevice(ctx->device));
    std::vector<FrameParams> frames;
    int rc = prepare_frames(ctx, cfgs, n, frames);
    if (rc != BH_OK) return rc;
    size_t npx = 0;
    for (int i = 0; i < n; ++i) npx += static_cast<size_t>(cfgs[i].width) * cfgs[i].height;
    if ((rc = ensure(ctx, ctx->pixels, npx * sizeof(bh_xyz))) != BH_OK) return rc;
    if ((rc = enqueue(ctx, frames, static_cast<bh_xyz*>(ctx->pixels.p), nullptr, ctx->stream, true)) != BH_OK)
        return rc;
    size_t off = 0;
    for (int i = 0; i < n; ++i) {
        double e = 0.0;
        rc = display_impl(ctx, d, static_cast<bh_xyz*>(ctx->pixels.p) + off, cfgs[i].width, cfgs[i].height,
                          outs_rgb[i], &e);
        if (rc != BH_OK) return rc;
        if (exposure_used) exposure_used[i] = e;
        off += static_cast<size_t>(cfgs[i].width) * cfgs[i].height;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return finish(ctx, n, stats, nullptr, true, secs);
}

int bh_gpu_eval(bh_ctx* ctx, const bh_render_config* cfg, int what, const double* in, long long n, double* out) {
    if (!ctx) return BH_ERR_INVALID_ARG;
    if (!out || n < 0 || (n > 0 && !in && what != BH_EVAL_FRAME))
        return fail(ctx, BH_ERR_INVALID_ARG, "in/out must not be NULL and n must be >= 0");
    if (what < BH_EVAL_RHS || what > BH_EVAL_FRAME) return fail(ctx, BH_ERR_INVALID_ARG, "unknown evaluation");
    CK(cudaSetDevice(ctx->device));
    std::vector<FrameParams> frames;
    int rc = prepare_frames(ctx, cfg, 1, frames);
    if (rc != BH_OK) return rc;
    const FrameParams& F = frames[0];
    if (what == BH_EVAL_FRAME) {
        out[0] = F.r_plus;
        out[1] = F.r_minus;
        out[2] = F.disc_enabled ? F.r_in : 0.0;
        out[3] = F.disc_enabled ? F.r_out : 0.0;
        out[4] = F.disc_enabled ? F.disc_eta : 0.0;
        out[5] = F.disc_enabled ? F.disc_mdot : 0.0;
        out[6] = F.r_stop;
        out[7] = F.r_escape;
        return BH_OK;
    }
    if (what == BH_EVAL_DISC_TEMPERATURE && !F.disc_enabled)
        return fail(ctx, BH_ERR_INVALID_ARG, "the config has no disc");
    if (n == 0) return BH_OK;
    const size_t n_in = static_cast<size_t>(n) * (what == BH_EVAL_RHS ? 8 : 1);
    const size_t n_out = static_cast<size_t>(n) * (what == BH_EVAL_RHS ? 8 : what == BH_EVAL_BLACKBODY ? 3 : 1);
    if ((rc = ensure(ctx, ctx->frames, sizeof(FrameParams))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->eval_in, n_in * sizeof(double))) != BH_OK) return rc;
    if ((rc = ensure(ctx, ctx->eval_out, n_out * sizeof(double))) != BH_OK) return rc;
    if (what == BH_EVAL_BLACKBODY && (rc = ensure_table(ctx)) != BH_OK) return rc;
    CK(cudaMemcpyAsync(ctx->frames.p, &F, sizeof(FrameParams), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->eval_in.p, in, n_in * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    const FrameParams* dF = static_cast<const FrameParams*>(ctx->frames.p);
    const double* din = static_cast<const double*>(ctx->eval_in.p);
    double* dout = static_cast<double*>(ctx->eval_out.p);
    if (what == BH_EVAL_RHS) CK(launch_eval_rhs(cfg->precision, dF, din, n, dout, ctx->stream));
    else CK(launch_eval_shade(what == BH_EVAL_DISC_TEMPERATURE ? 0 : 1, dF, ctx->d_table, din, n, dout, ctx->stream));
    CK(cudaMemcpyAsync(out, dout, n_out * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return BH_OK;
}

int bh_gpu_adjoint(bh_ctx* ctx, const bh_render_config* cfg, const float* target, bh_grad4* out) {
    return adjoint_impl(ctx, cfg, target, out, nullptr, nullptr);
}

int bh_gpu_adjoint_rays(bh_ctx* ctx, const bh_render_config* cfg, const float* target, bh_grad4* out,
                        double* ray_grad, double* ray_Y) {
    return adjoint_impl(ctx, cfg, target, out, ray_grad, ray_Y);
}

int bh_gpu_set_launch(bh_ctx* ctx, int precision, const bh_launch_params* p) {
    if (!ctx || !p) return BH_ERR_INVALID_ARG;
    if (precision == -1) {
        const int rc = bh_gpu_set_launch(ctx, BH_PRECISION_FP64, p);
        return rc != BH_OK ? rc : bh_gpu_set_launch(ctx, BH_PRECISION_MIXED, p);
    }
    if (precision != BH_PRECISION_FP64 && precision != BH_PRECISION_MIXED)
        return fail(ctx, BH_ERR_INVALID_ARG, "precision must be BH_PRECISION_FP64, _MIXED or -1");
    const int slot = precision == BH_PRECISION_MIXED ? 1 : 0;
    bh_launch_params n = ctx->launch[slot];
    if (p->block_size) {
        if (p->block_size < 32 || p->block_size > 1024 || p->block_size % 32)
            return fail(ctx, BH_ERR_INVALID_ARG, "block_size must be a multiple of 32 in [32, 1024]");
        n.block_size = p->block_size;
    }
    if (p->rays_per_thread) {
        if (p->rays_per_thread < 1 || p->rays_per_thread > 8)
            return fail(ctx, BH_ERR_INVALID_ARG, "rays_per_thread must be in [1, 8]");
        n.rays_per_thread = p->rays_per_thread;
    }
    if (p->refill) {
        if (p->refill < 1 || p->refill > 32) return fail(ctx, BH_ERR_INVALID_ARG, "refill must be in [1, 32]");
        n.refill = p->refill;
    }
    if (p->blocks_per_sm) {
        if (p->blocks_per_sm < 0 || p->blocks_per_sm > 64)
            return fail(ctx, BH_ERR_INVALID_ARG, "blocks_per_sm must be in [0, 64]");
        n.blocks_per_sm = p->blocks_per_sm;
    }
    if (p->reg_variant) {
        if (p->reg_variant != 1 && p->reg_variant != 2)
            return fail(ctx, BH_ERR_INVALID_ARG, "reg_variant must be 1 (tight) or 2 (wide)");
        n.reg_variant = p->reg_variant;
    }
    // Threads x registers of one block must fit in the SM's 64 K registers.
    if (n.block_size * trace_registers(precision, n.reg_variant == 2) > 65536)
        return fail(ctx, BH_ERR_INVALID_ARG, "block_size too large for the kernel's register count");
    ctx->launch[slot] = n;
    return BH_OK;
}

int bh_gpu_get_launch(const bh_ctx* ctx, int precision, bh_launch_params* p) {
    if (!ctx || !p || (precision != BH_PRECISION_FP64 && precision != BH_PRECISION_MIXED))
        return BH_ERR_INVALID_ARG;
    *p = ctx->launch[precision == BH_PRECISION_MIXED ? 1 : 0];
    return BH_OK;
}

// The launch-shape search of bh_gpu_autotune / bh_gpu_autotune_batch: every
// shape of the space renders the frame(s) twice, the shorter trace time
// counts, and the fastest shape is kept for cfgs[0].precision.
static int autotune_impl(bh_ctx* ctx, const bh_render_config* cfgs, int n, bh_launch_params* best,
                         double* best_ms) {
    if (!ctx) return BH_ERR_INVALID_ARG;
    if (!cfgs || n <= 0) return fail(ctx, BH_ERR_INVALID_ARG, "no frames to tune on");
    int rc = check_cfg_header(ctx, &cfgs[0]);
    if (rc != BH_OK) return rc;
    const int prec = cfgs[0].precision;
    if (prec != BH_PRECISION_FP64 && prec != BH_PRECISION_MIXED)
        return fail(ctx, BH_ERR_INVALID_ARG, "unknown precision");
    const int slot = prec == BH_PRECISION_MIXED ? 1 : 0;
    const bh_launch_params keep = ctx->launch[slot];
    std::vector<std::vector<bh_xyz>> px(n);
    std::vector<bh_xyz*> outs(n);
    for (int i = 0; i < n; ++i) {
        px[i].resize(static_cast<size_t>(std::max(cfgs[i].width, 1)) * std::max(cfgs[i].height, 1));
        outs[i] = px[i].data();
    }
    std::vector<bh_render_stats> st(n);
    bh_launch_params winner = keep;
    double winner_ms = 1e300;
    for (int rv = 1; rv <= 2; ++rv)
        for (int bs : {64, 128, 256, 512})
            for (int rpt : {1, 2, 4, 8})
                for (int refill : {8, 16, 24, 32}) {
                    if (bs * trace_registers(prec, rv == 2) > 65536) continue;
                    const bh_launch_params p{bs, rpt, refill, 0, rv};
                    ctx->launch[slot] = p;
                    double ms = 1e300;
                    for (int rep = 0; rep < 2; ++rep) {
                        std::memset(st.data(), 0, n * sizeof(bh_render_stats));
                        rc = (n == 1) ? bh_gpu_render(ctx, &cfgs[0], outs[0], st.data())
                                      : bh_gpu_render_batch(ctx, cfgs, n, outs.data(), st.data());
                        if (rc != BH_OK) {
                            ctx->launch[slot] = keep;
                            return rc;
                        }
                        ms = std::min(ms, st[0].kernel_ms);
                    }
                    if (ms < winner_ms) {
                        winner_ms = ms;
                        winner = p;
                    }
                }
    ctx->launch[slot] = winner;
    if (best) *best = winner;
    if (best_ms) *best_ms = winner_ms;
    return BH_OK;
}

int bh_gpu_autotune(bh_ctx* ctx, const bh_render_config* cfg, bh_launch_params* best, double* best_ms) {
    return autotune_impl(ctx, cfg, 1, best, best_ms);
}

int bh_gpu_autotune_batch(bh_ctx* ctx, const bh_render_config* cfgs, int n, bh_launch_params* best,
                          double* best_ms) {
    return autotune_impl(ctx, cfgs, n, best, best_ms);
}

int bh_gpu_set_step_budget(bh_ctx* ctx, long long budget) {
    if (!ctx || budget < 0) return BH_ERR_INVALID_ARG;
    ctx->budget = static_cast<unsigned long long>(budget);
    return BH_OK;
}

void bh_gpu_request_abort(bh_ctx* ctx) {
    if (!ctx) return;
    ctx->abort_requested.store(1);
    cudaSetDevice(ctx->device);
    // Lands in the queue state while a launch runs; the next launch starts
    // with the flag set anyway.
    cudaMemcpyAsync(&ctx->d_queue->abort, ctx->h_one, sizeof(int32_t), cudaMemcpyHostToDevice,
                    ctx->abort_stream);
}

int bh_star_catalogue(int count, uint64_t seed, int sky_mode, double* out6) {
    return star_catalogue(count, seed, sky_mode, out6);
}

int bh_blackbody_table(double* out) {
    if (!out) return BH_ERR_INVALID_ARG;
    std::vector<double> t;
    build_blackbody_table(t);
    std::memcpy(out, t.data(), t.size() * sizeof(double));
    return BH_OK;
}

void bh_gpu_clear_abort(bh_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->abort_stream);
    ctx->abort_requested.store(0);
}

}  // extern "C"
