// bh_adjoint.cu - The discrete-adjoint kernel and its reductions (sm_100a).
//
// adjoint_kernel: one thread per ray at a time, rays handed out by a global
// atomic counter; each thread owns `checkpoint_slots` checkpoint states in
// global memory for the ray it is working on (bh_adjoint.cuh has the per-ray
// algorithm).  The ray's loss weight is 2 (Y_pixel - target) / S^2 for
// Loss = sum over pixels of (Y_pixel - target)^2, Y_pixel being the sample
// mean of the rendered frame (bh_gpu_render's output).
//
// adjoint_reduce_kernel: five blocks, each summing one quantity (the loss and
// the four gradient components) over a fixed thread-to-element assignment and
// a fixed tree, so the result does not depend on the order rays finished in.
#include <cuda_runtime.h>

#include "bh_adjoint.cuh"

namespace bhg {

namespace {

constexpr int kAdjBlock = 128;
constexpr int kReduceThreads = 1024;

__global__ void __launch_bounds__(kAdjBlock) adjoint_kernel(const AdjointLaunch L) {
    const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int slots = L.X.checkpoint_slots;
    double* ck = L.ckpt + slot * slots * 8;
    const int S = L.frame.S;
    const int SS = S * S;
    const int W = L.frame.width, H = L.frame.height;
    unsigned long long steps = 0, replay = 0, disc = 0, sky = 0, max_int = 0;
    for (;;) {
        const long long id = (long long)atomicAdd(&L.counters[0], 1ull);
        if (id >= L.n_rays) break;
        const long long pixel = id / SS;
        const int k = (int)(id - pixel * SS);
        int px, py;
        pixel_xy(W, H, pixel, &px, &py);
        const long long pix = (long long)py * W + px;
        const double w = 2.0 * (L.pixels[pix].y - (double)L.target[pix]) / (double)SS;
        adj::RayResult res;
        adj::adjoint_ray(L.frame, L.X, L.sky, id, w, ck, slots, false, &res);
        const long long o = pix * SS + k;
        #pragma unroll
        for (int q = 0; q < 4; ++q) L.ray_grad[o * 4 + q] = res.grad[q];
        if (L.ray_Y) L.ray_Y[o] = res.Y;
        steps += (unsigned long long)res.steps;
        replay += (unsigned long long)res.replay;
        disc += (res.what == BH_HIT_DISC) ? 1ull : 0ull;
        sky += (res.what == BH_HIT_SKY) ? 1ull : 0ull;
        if ((unsigned long long)res.interval > max_int) max_int = (unsigned long long)res.interval;
    }
    atomicAdd(&L.counters[1], steps);
    atomicAdd(&L.counters[2], replay);
    atomicAdd(&L.counters[3], disc);
    atomicAdd(&L.counters[4], sky);
    atomicMax(&L.counters[5], max_int);
}

__global__ void __launch_bounds__(kReduceThreads)
adjoint_reduce_kernel(const double* __restrict__ grad, long long n_rays, const bh_xyz* __restrict__ pixels,
                      const float* __restrict__ target, long long n_pix, double* out) {
    __shared__ double part[kReduceThreads];
    const int b = blockIdx.x;
    double acc = 0.0;
    if (b == 0) {
        for (long long p = threadIdx.x; p < n_pix; p += kReduceThreads) {
            const double d = pixels[p].y - (double)target[p];
            acc += d * d;
        }
    } else {
        for (long long i = threadIdx.x; i < n_rays; i += kReduceThreads) acc += grad[i * 4 + (b - 1)];
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kReduceThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[b] = part[0];
}

}  // namespace

int adjoint_blocks_per_sm(int block_size) {
    int n = 0;
    if (block_size != kAdjBlock) return 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, adjoint_kernel, block_size, 0);
    return n;
}

cudaError_t launch_adjoint(const AdjointLaunch& L, cudaStream_t stream) {
    if (L.block != kAdjBlock) return cudaErrorInvalidValue;
    if (L.n_rays > 0) adjoint_kernel<<<L.grid, L.block, 0, stream>>>(L);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const long long n_pix = (long long)L.frame.width * L.frame.height;
    adjoint_reduce_kernel<<<5, kReduceThreads, 0, stream>>>(L.ray_grad, L.n_rays, L.pixels, L.target, n_pix,
                                                           L.sums);
    return cudaGetLastError();
}

}  // namespace bhg
