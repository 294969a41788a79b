// bh_peak.cu - Measured FMA throughput of this GPU, the roofline denominator
// of the ALU-bound trace kernel.
//
// Each thread runs 8 independent FMA chains for `iters` iterations; the grid
// covers every SM with enough warps to hide the FMA latency.  FLOPs = 2 per
// FMA.  Timed with CUDA events on the context's stream.
#include <cuda_runtime.h>

#include "../../include/bh_gpu.h"

namespace {

template <class T>
__global__ void fma_chains(T* out, int iters, T a, T b) {
    T x0 = (T)threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
    T x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
        #pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
            x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
        }
    }
    const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)-1.2345) out[blockIdx.x] = s;   // keeps the chains live
}

template <class T>
int run(int device, double* tflops) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return BH_ERR_CUDA;
    const int block = 256;
    const int grid = prop.multiProcessorCount * 8;
    const int iters = 2048;
    T* out = nullptr;
    if (cudaMalloc(&out, grid * sizeof(T)) != cudaSuccess) return BH_ERR_OUT_OF_MEMORY;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const T a = (T)0.999999, b = (T)1e-7;
    fma_chains<T><<<grid, block>>>(out, iters / 8, a, b);   // warm-up
    cudaEventRecord(e0);
    fma_chains<T><<<grid, block>>>(out, iters, a, b);
    cudaEventRecord(e1);
    const cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess || ms <= 0.f) return BH_ERR_CUDA;
    const double flops = 2.0 * 8.0 * 16.0 * (double)iters * block * (double)grid;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return BH_OK;
}

}  // namespace

extern "C" int bh_gpu_fma_peak(int device, int precision, double* tflops) {
    if (!tflops) return BH_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return BH_ERR_NO_DEVICE;
    return precision == BH_PRECISION_FP64 ? run<double>(device, tflops) : run<float>(device, tflops);
}
