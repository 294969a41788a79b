// bh_noalloc.cu - bh_gpu_trace_noalloc: the trace kernel with no allocation.
//
// Some callers cannot call cudaMalloc: hosts whose GPU memory belongs to
// their own allocator or fixed budget, plug-in hosts that forbid device
// allocation inside the render callback, real-time loops that cannot take the
// implicit device synchronisation of cudaMalloc/cudaFree.  For them this entry
// point runs the same persistent trace kernels as the context API, but the
// kernels' scratch - the work-queue counters, the frame constants and, in
// mixed precision, the list of rays handed to the binary64 pass - lives in one
// file-scope __device__ array instead of context allocations.  The caller
// provides the output buffer; nothing is allocated on the device, and on the
// success path nothing on the host either.
//
// Limits and sharing: the array holds the deferred records of at most
// BH_NOALLOC_MAX_RAYS rays (6 MiB of its 6.3 MiB), so a call takes at most
// that many rays.  Every GPU that loads the library keeps the array until the
// process exits.  All calls share it and it keeps the last call's contents:
// each call clears the counters that must start at zero, and two calls whose
// work overlaps on the GPU race on the array, so callers serialise them.
//
// The frame constants reach the device as the arguments of a one-block
// staging kernel, which the launch copies when it is enqueued: no copy reads
// the host stack after the call returns.  The caller's current device is put
// back before every return.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/bh_gpu.h"
#include "bh_frame.h"
#include "bh_launch.h"
#include "bh_scene.h"

namespace bhg {
namespace {

constexpr size_t kQueueOff = 0;
constexpr size_t kFrameOff = 256;
constexpr size_t kFrameBytes = (sizeof(FrameParams) + 255) / 256 * 256;
constexpr size_t kFrameSideOff = kFrameOff + kFrameBytes;   // the frame under binary64_treatment
constexpr size_t kRayEndOff = kFrameSideOff + kFrameBytes;
constexpr size_t kDeferredOff = kRayEndOff + 256;
constexpr size_t kScratchBytes = kDeferredOff + (size_t)BH_NOALLOC_MAX_RAYS * kDeferredRecordBytes;

static_assert(sizeof(QueueState) <= 256, "queue slot too small");
static_assert(sizeof(bh_trace_record) == sizeof(HitRecord), "bh_trace_record must mirror HitRecord");
static_assert(offsetof(bh_trace_record, max_norm) == offsetof(HitRecord, max_norm), "layout");
static_assert(offsetof(bh_trace_record, what) == offsetof(HitRecord, what), "layout");
static_assert(offsetof(bh_trace_record, attempts) == offsetof(HitRecord, attempts), "layout");

// The scratch.  In host code `g_scratch` names a host-side stand-in, not the
// device array: its device address comes from cudaGetSymbolAddress, once per
// device, and only that address is handed to kernels and copies.
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// The frame constants of a call, the binary64 pass's version of them and the
// ray count, written with the work-queue counters cleared: one block, its
// threads copying the two frames a word at a time.
__global__ void noalloc_stage_kernel(const FrameParams F, const FrameParams G, long long n, QueueState* queue,
                                     FrameParams* frame, FrameParams* frame_side, long long* ray_end) {
    static_assert(sizeof(FrameParams) % sizeof(unsigned long long) == 0, "FrameParams is whole words");
    constexpr int kWords = (int)(sizeof(FrameParams) / sizeof(unsigned long long));
    const unsigned long long* f = reinterpret_cast<const unsigned long long*>(&F);
    const unsigned long long* g = reinterpret_cast<const unsigned long long*>(&G);
    unsigned long long* df = reinterpret_cast<unsigned long long*>(frame);
    unsigned long long* dg = reinterpret_cast<unsigned long long*>(frame_side);
    for (int i = threadIdx.x; i < kWords; i += blockDim.x) {
        df[i] = f[i];
        dg[i] = g[i];
    }
    constexpr int kQueueWords = (int)(sizeof(QueueState) / sizeof(unsigned long long));
    static_assert(sizeof(QueueState) % sizeof(unsigned long long) == 0, "QueueState is whole words");
    unsigned long long* dq = reinterpret_cast<unsigned long long*>(queue);
    for (int i = threadIdx.x; i < kQueueWords; i += blockDim.x) dq[i] = 0ull;
    if (threadIdx.x == 0) *ray_end = n;
}

// Puts the calling thread's current device back when the entry point returns.
struct DeviceRestore {
    int prev = -1;
    DeviceRestore() {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            cudaGetLastError();
            prev = -1;
        }
    }
    ~DeviceRestore() {
        int now = -1;
        if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
    }
};

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch on `device` (current); looked up on the
// first call for that device.
int scratch_address(int device, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) return BH_ERR_CUDA;
        g_scratch_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[device]);
    return BH_OK;
}

}  // namespace
}  // namespace bhg

extern "C" int bh_gpu_trace_noalloc(int device, const bh_render_config* cfg, bh_trace_record* d_out,
                                    void* stream) {
    using namespace bhg;
    if (!cfg || !d_out) return BH_ERR_INVALID_ARG;
    if (cfg->struct_size != sizeof(bh_render_config) || cfg->abi_version != BH_GPU_ABI_VERSION)
        return BH_ERR_INVALID_ARG;
    FrameParams F;
    std::string err;   // untouched (no allocation) unless the config is rejected
    int rc = make_frame(*cfg, F, err);
    if (rc != BH_OK) return rc;
    if (F.n_rays > BH_NOALLOC_MAX_RAYS) return BH_ERR_INVALID_ARG;
    if (F.jet_enabled) return BH_ERR_UNSUPPORTED;   // the jet's per-ray sum has no slot here
    F.precision_tag = cfg->precision;
    F.ray_begin = 0;
    F.pixel_begin = 0;

    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return BH_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count || device >= kMaxDevices) return BH_ERR_INVALID_ARG;
    const DeviceRestore restore;
    if (cudaSetDevice(device) != cudaSuccess) return BH_ERR_CUDA;
    unsigned char* base = nullptr;
    if ((rc = scratch_address(device, &base)) != BH_OK) return rc;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return BH_ERR_CUDA;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    QueueState* queue = reinterpret_cast<QueueState*>(base + kQueueOff);
    FrameParams* frame = reinterpret_cast<FrameParams*>(base + kFrameOff);
    long long* ray_end = reinterpret_cast<long long*>(base + kRayEndOff);
    const long long n = F.n_rays;
    // Counters start at zero on every call; the array keeps the last call's.
    FrameParams* frame_side = reinterpret_cast<FrameParams*>(base + kFrameSideOff);
    const FrameParams G = binary64_treatment(F);
    noalloc_stage_kernel<<<1, 128, 0, s>>>(F, G, n, queue, frame, frame_side, ray_end);
    if (cudaGetLastError() != cudaSuccess) return BH_ERR_CUDA;
    if (n == 0) return BH_OK;

    // The context API's default launch shapes: refill at 32 idle lanes, the
    // tight register caps, blocks of 128 for binary64 and 256 for binary32.
    const bool mixed = cfg->precision == BH_PRECISION_MIXED;
    TraceLaunch tl;
    std::memset(&tl, 0, sizeof tl);
    tl.frames = frame;
    tl.frame_ray_end = ray_end;
    tl.nframes = 1;
    tl.total_rays = n;
    tl.hits = reinterpret_cast<HitRecord*>(d_out);
    tl.queue = queue;
    tl.precision = cfg->precision;
    tl.block_size = mixed ? 256 : 128;
    tl.rays_per_thread = 1;
    tl.refill = 32;
    tl.budget = 0;
    tl.reg_variant = 0;
    const int bps = trace_blocks_per_sm(cfg->precision, tl.block_size, tl.reg_variant);
    tl.grid = sms * (bps < 1 ? 1 : bps);
    tl.deferred = mixed ? static_cast<void*>(base + kDeferredOff) : nullptr;
    tl.block_resume = 128;
    tl.reg_variant_resume = 0;
    const int bps64 = trace_blocks_per_sm(BH_PRECISION_FP64, 128, 0);
    tl.grid_resume = sms * (bps64 < 1 ? 1 : bps64);
    tl.resume_event = nullptr;
    tl.surfaces = (F.sun_enabled || F.ns_enabled) ? 1 : 0;
    // Near-critical rays in binary64 as the context API traces them, here
    // before the binary32 kernel on the caller's stream (no stream of our own).
    tl.near_critical = F.fp64_near_critical;
    tl.grid_side = sms;
    tl.frames_side = frame_side;
    tl.side_stream = nullptr;
    return launch_trace(tl, s) == cudaSuccess ? BH_OK : BH_ERR_CUDA;
}
