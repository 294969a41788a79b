// bh_common.cuh - Helpers shared by the trace, shade and adjoint kernels (the
// arithmetic ones also compile for the host).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace bhg {

constexpr double kPi = 3.14159265358979323846;
constexpr unsigned kFull = 0xffffffffu;

// std::max / std::min / std::clamp semantics (NaN handling included).
__host__ __device__ __forceinline__ double dmaxr(double a, double b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ double dminr(double a, double b) { return (b < a) ? b : a; }
__host__ __device__ __forceinline__ double dclamp(double v, double lo, double hi) {
    return (v < lo) ? lo : (hi < v) ? hi : v;
}

// 1 / x in binary64 from the hardware's approximate reciprocal and two Newton
// steps e = 1 - x r, r += r e (the error squares each step, ending within an
// ulp): a handful of fused multiply-adds instead of the division sequence.
// x = 0 gives NaN where the division gives inf; both make the step
// non-finite, which the controller rejects.  Host code: the division.
__host__ __device__ __forceinline__ double rcp_nr(double x) {
#if defined(__CUDA_ARCH__)
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
#else
    return 1.0 / x;
#endif
}

// sin and cos of th0 + d from those of th0, |d| <= kMaxShift: angle addition
// with the Taylor series of sin d and cos d in Horner form (coefficients
// +-1/n!): to d^7 / d^6 in binary32, to d^13 / d^14 in binary64 (truncation
// below the format's rounding for |d| <= 1/4).
constexpr double kMaxShift = 0.25;
__host__ __device__ __forceinline__ void shift_sincos(float s0, float c0, float d, float* s, float* c) {
    const float d2 = d * d;
    const float ps = fmaf(d2, fmaf(d2, -1.f / 5040.f, 1.f / 120.f), -1.f / 6.f);
    const float pc = fmaf(d2, fmaf(d2, -1.f / 720.f, 1.f / 24.f), -0.5f);
    const float sd = fmaf(d * d2, ps, d);
    const float cd = fmaf(d2, pc, 1.f);
    *s = fmaf(s0, cd, c0 * sd);
    *c = fmaf(c0, cd, -(s0 * sd));
}
__host__ __device__ __forceinline__ void shift_sincos(double s0, double c0, double d, double* s, double* c) {
    const double d2 = d * d;
    const double ps = fma(d2, fma(d2, fma(d2, fma(d2, fma(d2, 1.0 / 6227020800.0, -1.0 / 39916800.0),
                                              1.0 / 362880.0), -1.0 / 5040.0), 1.0 / 120.0), -1.0 / 6.0);
    const double pc = fma(d2, fma(d2, fma(d2, fma(d2, fma(d2, fma(d2, -1.0 / 87178291200.0, 1.0 / 479001600.0),
                                                      -1.0 / 3628800.0), 1.0 / 40320.0), -1.0 / 720.0),
                              1.0 / 24.0), -0.5);
    const double sd = fma(d * d2, ps, d);
    const double cd = fma(d2, pc, 1.0);
    *s = fma(s0, cd, c0 * sd);
    *c = fma(c0, cd, -(s0 * sd));
}

// splitmix64 output of state z (scene.h:30-36) and its 53-bit uniform (scene.h:37).
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ double u53(uint64_t z) { return (double)(z >> 11) * 0x1.0p-53; }

// Pixel of a frame-local pixel index.  Pixels are enumerated in bands of four
// rows, column by column inside a band, so that 32 consecutive rays cover an
// 8 x 4 patch of the image (coherent paths) rather than 32 pixels of one row.
__host__ __device__ __forceinline__ void pixel_xy(int W, int H, long long p, int* x, int* y) {
    const long long band_px = 4LL * W;
    const int band = (int)(p / band_px);
    const int rel = (int)(p - (long long)band * band_px);
    const int y0 = 4 * band;
    const int bh = (H - y0 < 4) ? H - y0 : 4;
    *x = rel / bh;
    *y = y0 + rel % bh;
}

// The inverse of pixel_xy: the frame-local pixel index of pixel (x, y).
__host__ __device__ __forceinline__ long long pixel_index(int W, int H, int x, int y) {
    const int band = y >> 2;
    const int y0 = 4 * band;
    const int bh = (H - y0 < 4) ? H - y0 : 4;
    return (long long)band * 4 * W + (long long)x * bh + (y - y0);
}

// Index of the frame whose cumulative end exceeds `id` (ends ascending).
__device__ __forceinline__ int find_frame(const long long* __restrict__ ends, int n, long long id) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (id < __ldg(&ends[mid])) hi = mid; else lo = mid + 1;
    }
    return lo;
}

}  // namespace bhg
