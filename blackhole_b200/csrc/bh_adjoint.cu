// bh_adjoint.cu - The discrete-adjoint kernel and its reductions (sm_100a).
//
// adjoint_kernel: one thread per job at a time, jobs handed out by a global
// atomic counter; each thread owns `checkpoint_slots` checkpoint states in
// global memory for the job it is working on (bh_adjoint.cuh has the per-ray
// algorithm).  A ray's loss weight is 2 (Y_pixel - target) / S^2 for
// Loss = sum over pixels of (Y_pixel - target)^2, Y_pixel being the sample
// mean of the rendered frame (bh_gpu_render's output).
//
// The edge pass: a point-sampled frame has no derivative with respect to
// r_out, and its derivatives with respect to the spin and the inclination
// miss the motion of the disc's edges; the derivative of the frame averaged
// over each sample's cell has both.  edge_candidates_kernel picks each
// sample's first two equatorial crossings near an edge (adj::edge_mask,
// against the spread of the neighbouring samples' same crossing; the render
// records the crossings), and the adjoint kernel takes their edge terms
// (adj::edge_sample, weight 2 (Y_pixel - target)) as its first jobs, so the
// long ones overlap the per-ray work instead of forming a tail of their own.
//
// The edge pass covers the edges of the first two equatorial crossings (the
// direct image of the disc and its first lensed image).  Images of order
// three and higher are rings so thin that a sample's derivative holds over a
// small part of its cell, and their edges are not in the edge pass, so their
// per-ray spin and inclination terms are summed apart (the held-out sums)
// rather than into the frame gradient.
//
// adjoint_reduce_kernel: ten blocks, each summing one quantity (the loss,
// the four per-ray gradient components, the three edge components, the two
// held-out components) over a fixed thread-to-element assignment and a fixed
// tree, so the result does not depend on the order rays finished in.
#include <cuda_runtime.h>

#include "bh_adjoint.cuh"

namespace bhg {

namespace {

constexpr int kAdjBlock = 128;
constexpr int kReduceThreads = 1024;

// Candidate selection: one thread per sample (work order); each of its first
// two equatorial crossings, as the render recorded them, is compared with the
// same crossing of its four neighbours in the W S x H S sample grid
// (adj::edge_mask).
__global__ void __launch_bounds__(256) edge_candidates_kernel(const AdjointLaunch L) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= L.n_rays) return;
    const int S = L.frame.S;
    const int SS = S * S;
    const int W = L.frame.width, H = L.frame.height;
    const long long pixel = id / SS;
    const int k = (int)(id - pixel * SS);
    int px, py;
    pixel_xy(W, H, pixel, &px, &py);
    const int gx = px * S + k % S;
    const int gy = py * S + k / S;
    const int GW = W * S, GH = H * S;
    for (int j = 0; j < 2; ++j) {
        const double rc = L.xing_r[2 * id + j];
        if (rc == 0.0) break;
        double dmax = 0.0;
        #pragma unroll
        for (int n = 0; n < 4; ++n) {
            const int nx = gx + (n == 0) - (n == 1);
            const int ny = gy + (n == 2) - (n == 3);
            if (nx < 0 || nx >= GW || ny < 0 || ny >= GH) continue;
            const long long nid = pixel_index(W, H, nx / S, ny / S) * SS + (ny % S) * S + nx % S;
            const double rn = L.xing_r[2 * nid + j];
            if (rn == 0.0) continue;
            const double d = fabs(rc - rn);
            if (d > dmax) dmax = d;
        }
        const int m = adj::edge_mask(L.frame, rc, dmax);
        if (m) {
            const unsigned long long at = atomicAdd(&L.counters[6], 1ull);
            L.cand[at] = ((unsigned long long)(2 * id + j) << 2) | (unsigned long long)m;
        }
    }
}

// One queue of jobs: first the edge candidates (each a forward pass to its
// crossing, the continuation past it and a reverse sweep: the longest jobs),
// then the rays.  Each thread owns `checkpoint_slots` checkpoint states for
// the job it is working on; results go to per-ray and per-crossing slots, so
// the sums do not depend on which thread took which job.
__global__ void __launch_bounds__(kAdjBlock) adjoint_kernel(const AdjointLaunch L) {
    const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int slots = L.X.checkpoint_slots;
    double* ck = L.ckpt + slot * slots * 8;
    const int S = L.frame.S;
    const int SS = S * S;
    const int W = L.frame.width, H = L.frame.height;
    const unsigned long long n_cand = L.counters[6];
    unsigned long long steps = 0, replay = 0, disc = 0, sky = 0, max_int = 0, n_high = 0;
    unsigned long long edge_steps = 0, edge_cells = 0;
    for (;;) {
        const unsigned long long job = atomicAdd(&L.counters[0], 1ull);
        if (job < n_cand) {
            const unsigned long long c = L.cand[job];
            const long long xs = (long long)(c >> 2);     // 2 * ray + crossing
            const long long id = xs >> 1;
            const long long pixel = id / SS;
            const int k = (int)(id - pixel * SS);
            int px, py;
            pixel_xy(W, H, pixel, &px, &py);
            const long long pix = (long long)py * W + px;
            const double w = 2.0 * (L.pixels[pix].y - (double)L.target[pix]);
            double out[3];
            int n_cells = 0;
            edge_steps += (unsigned long long)adj::edge_sample(L.frame, L.X, L.sky, px, py, k, (int)(xs & 1) + 1,
                                                               (int)(c & 3ull), w, ck, slots, out, &n_cells);
            edge_cells += (unsigned long long)n_cells;
            L.edge_out[3 * xs] = out[0];
            L.edge_out[3 * xs + 1] = out[1];
            L.edge_out[3 * xs + 2] = out[2];
            continue;
        }
        const long long id = (long long)(job - n_cand);
        if (id >= L.n_rays) break;
        const long long pixel = id / SS;
        const int k = (int)(id - pixel * SS);
        int px, py;
        pixel_xy(W, H, pixel, &px, &py);
        const long long pix = (long long)py * W + px;
        const double w = 2.0 * (L.pixels[pix].y - (double)L.target[pix]) / (double)SS;
        adj::RayResult res;
        adj::Crossings xr;
        xr.n = 0;
        xr.count = 0;
        xr.r[0] = xr.r[1] = 0.0;
        xr.step[0] = xr.step[1] = 0;
        adj::adjoint_ray(L.frame, L.X, L.sky, id, w, ck, slots, false, &res, &xr);
        const long long o = pix * SS + k;
        const bool high = xr.count >= 3 && (res.what == BH_HIT_DISC || res.what == BH_HIT_SKY);
        L.high_order[o] = high ? 1 : 0;
        n_high += high ? 1ull : 0ull;
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
    atomicAdd(&L.counters[7], edge_steps);
    atomicAdd(&L.counters[8], edge_cells);
    atomicAdd(&L.counters[9], n_high);
}

__global__ void __launch_bounds__(kReduceThreads)
adjoint_reduce_kernel(const double* __restrict__ grad, const double* __restrict__ edge,
                      const unsigned char* __restrict__ high, long long n_rays, const bh_xyz* __restrict__ pixels,
                      const float* __restrict__ target, long long n_pix, double* out) {
    __shared__ double part[kReduceThreads];
    const int b = blockIdx.x;
    double acc = 0.0;
    if (b == 0) {
        for (long long p = threadIdx.x; p < n_pix; p += kReduceThreads) {
            const double d = pixels[p].y - (double)target[p];
            acc += d * d;
        }
    } else if (b <= 2) {           // spin, inclination: images of order one and two
        for (long long i = threadIdx.x; i < n_rays; i += kReduceThreads)
            if (!high[i]) acc += grad[i * 4 + (b - 1)];
    } else if (b <= 4) {           // Eddington ratio, r_out: every ray
        for (long long i = threadIdx.x; i < n_rays; i += kReduceThreads) acc += grad[i * 4 + (b - 1)];
    } else if (b <= 7) {
        for (long long i = threadIdx.x; i < 2 * n_rays; i += kReduceThreads) acc += edge[i * 3 + (b - 5)];
    } else {                       // spin, inclination: order three and higher
        for (long long i = threadIdx.x; i < n_rays; i += kReduceThreads)
            if (high[i]) acc += grad[i * 4 + (b - 8)];
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
    if (L.n_rays > 0) {
        edge_candidates_kernel<<<(unsigned)((L.n_rays + 255) / 256), 256, 0, stream>>>(L);
        adjoint_kernel<<<L.grid, L.block, 0, stream>>>(L);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const long long n_pix = (long long)L.frame.width * L.frame.height;
    adjoint_reduce_kernel<<<kAdjSums, kReduceThreads, 0, stream>>>(L.ray_grad, L.edge_out, L.high_order,
                                                                  L.n_rays, L.pixels, L.target, n_pix, L.sums);
    return cudaGetLastError();
}

}  // namespace bhg
