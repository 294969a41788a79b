// bh_launch.h - Host-side launch wrappers of the trace, shade and stats kernels.
#pragma once

#include <cuda_runtime.h>

#include "bh_frame.h"

struct bh_xyz;
struct bh_ray_result;

namespace bhg {

struct TraceLaunch {
    const FrameParams* frames;       // device array
    const long long* frame_ray_end;  // device array: cumulative ray counts (exclusive end)
    int nframes;
    long long total_rays;
    HitRecord* hits;                 // device, total_rays entries
    QueueState* queue;               // device
    int precision;                   // BH_PRECISION_*
    int block_size;
    int grid;                        // blocks
    int rays_per_thread;
    int refill;
    unsigned long long budget;       // step-attempt budget of the launch, 0 = none
    int reg_variant;                 // 0: default register cap, 1: the wider one
    void* deferred;                  // mixed precision: total_rays deferred records
    int grid_resume;                 // blocks of the binary64 resume launch
    int block_resume;                // its threads per block
    int reg_variant_resume;          // its register cap (0 tight, 1 wide)
    cudaEvent_t resume_event;        // recorded between the two launches (optional)
    double* jet;                     // jet emission per ray (total_rays), or null when no
                                     // frame of the launch has a jet
    double* xing;                    // radii of each ray's first two equatorial crossings
                                     // (2 per ray, zeroed before; 0 = none), or null
    int surfaces;                    // 1 when a frame of the launch has the Sun or a neutron star
    // Mixed precision: near-critical rays (escaping rays that circle close to
    // the photon shell) traced by a binary64 kernel of grid_side blocks of 128
    // on `stream`, beside the binary32 kernel on side_stream (fork_event /
    // join_event order it against `stream`), or before it on `stream` when
    // side_stream is null.
    int near_critical;
    int grid_side;
    int grid_late;                   // binary32 blocks started on `stream` after the binary64 kernel
    int grid_list;                   // blocks of 128 of the binary64 pass over the listed rays left
                                     // after the binary32 kernels (beyond grid_side * 128 of them)
    const FrameParams* frames_side;  // device: the frames under binary64_treatment
    unsigned char* sel_flag;         // device, total_rays: near-critical flags (classification
                                     // pass), or null: then both kernels test each ray themselves
    int* sel_list;                   // device, total_rays: the near-critical rays' ids
    cudaStream_t side_stream;
    cudaEvent_t fork_event, join_event;
    // Row bands of a single-frame launch whose pixels are shaded and copied
    // out while the rest of the frame is traced: each finished ray adds one
    // to band_done[gid / rays_per_band]; after the last trace kernel every
    // counter is raised to its band's size (so a wait on it always ends).
    // Null: no counting.
    unsigned int* band_done;
    long long rays_per_band;
    int nbands;
};

// Bytes of one deferred-ray record.
size_t deferred_record_bytes();
constexpr size_t kDeferredRecordBytes = 96;   // checked against the record in bh_trace.cu

// Persistent trace kernel over all rays of all frames.
cudaError_t launch_trace(const TraceLaunch& L, cudaStream_t stream);

// Blocks per SM that fit for a precision and block size (occupancy query;
// the least over the plain, surface and jet kernels of that precision and cap).
int trace_blocks_per_sm(int precision, int block_size, int variant);
// Registers per thread of the trace kernels of a precision (the most over
// the plain, surface and jet kernels).
int trace_registers(int precision, int variant);

struct ShadeLaunch {
    const FrameParams* frames;
    const long long* frame_pixel_end;   // cumulative pixel counts
    int nframes;
    long long total_pixels;
    const HitRecord* hits;
    SkyData sky;
    bh_xyz* pixels;                  // device, total_pixels entries (frame-major, row-major)
    bh_ray_result* rays;             // optional device per-sample results (single frame)
    double* pixel_lum;               // device, total_pixels luminance for the flux sum
    unsigned char* ray_class;        // device, per-ray class after shading
    const double* jet;               // jet emission per ray (TraceLaunch::jet), or null
    long long pixel_lo;              // shade global pixels [pixel_lo, total_pixels) only
};

cudaError_t launch_shade(const ShadeLaunch& L, cudaStream_t stream);

struct ReduceLaunch {
    const FrameParams* frames;
    int nframes;
    const HitRecord* hits;
    const double* pixel_lum;
    const double* jet;               // jet emission per ray, or null
    FrameStats* partials;            // nframes * blocks_per_frame
    FrameStats* out;                 // nframes
    int blocks_per_frame;
};

cudaError_t launch_reduce(const ReduceLaunch& L, cudaStream_t stream);

// Known-answer evaluation of device functions (bh_gpu_eval): the trace
// kernels' right-hand side at n states of 8 doubles (8 derivatives each),
// and the shading's disc temperature (what 0: n radii -> n kelvin) or
// blackbody lookup (what 1: n kelvin -> 3n XYZ).
cudaError_t launch_eval_rhs(int precision, const FrameParams* d_frame, const double* d_in, long long n,
                            double* d_out, cudaStream_t stream);
cudaError_t launch_eval_shade(int what, const FrameParams* d_frame, const double* d_table, const double* d_in,
                              long long n, double* d_out, cudaStream_t stream);

}  // namespace bhg
