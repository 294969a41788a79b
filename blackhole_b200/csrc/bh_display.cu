// bh_display.cu - The display transform on the GPU (image.cpp:22-191).
//
// A rendered frame stays on the device and leaves it as 8-bit sRGB (3 bytes
// per pixel instead of 24):
//
//   glare      add_glare (image.cpp:47-104): two separable Gaussian blurs with
//              clamped edges (sigma = radius and 3 radius), then
//              p core + near 0.7 s + far 0.3 s.  One thread per output pixel,
//              the taps summed in the reference's order without contraction,
//              with the reference's normalised weights computed on the host.
//   exposure   auto_exposure (image.cpp:22-45): the order statistics
//              k = (size_t)(q (n - 1)), q = 0.999 and 0.9999, of the n positive
//              finite luminances, found by an 8-pass most-significant-digit
//              radix select on the binary64 bit patterns (positive doubles
//              order like their bits): per pass one histogram kernel over the
//              frame (shared-memory bins, one global add per bin per block) and
//              one single-block kernel that picks the digit.  No host round
//              trip, so the whole transform can run inside a stream or graph.
//   develop    develop (image.cpp:117-191, spectrum.cpp:137-152): exposure,
//              XYZ -> linear sRGB, gamut clamp, tone curve, sRGB transfer,
//              rounding to 8 bits; one thread per pixel.
//
// The arithmetic is binary64 with the reference's operand order and no fused
// multiply-add, so the output equals the reference's byte for byte except
// where the device's pow/log10/tanh and the host libm's differ in the last
// bit at a rounding boundary of 255 v.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bh_gpu.h"
#include "bh_display.h"

namespace bhg {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }
__device__ __forceinline__ double clampd(double v, double lo, double hi) {
    return (v < lo) ? lo : (hi < v) ? hi : v;
}

// One pass of the separable blur: along x (dir 0) or y (dir 1).
__global__ void blur_pass(const bh_xyz* __restrict__ src, bh_xyz* __restrict__ dst, int w, int h,
                          const double* __restrict__ k, int r, int dir) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)w * h) return;
    const int y = (int)(p / w), x = (int)(p - (long long)y * w);
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int i = -r; i <= r; ++i) {
        const long long q = dir == 0 ? (long long)y * w + clampi(x + i, 0, w - 1)
                                     : (long long)clampi(y + i, 0, h - 1) * w + x;
        const double kk = __ldg(&k[i + r]);
        const bh_xyz s = src[q];
        ax = add(ax, mul(kk, s.x));
        ay = add(ay, mul(kk, s.y));
        az = add(az, mul(kk, s.z));
    }
    dst[p] = bh_xyz{ax, ay, az};
}

__global__ void glare_combine(bh_xyz* __restrict__ px, const bh_xyz* __restrict__ nearp,
                              const bh_xyz* __restrict__ farp, long long n, double core, double a, double b) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bh_xyz p = px[i];
    const bh_xyz q = nearp[i], f = farp[i];
    p.x = add(add(mul(p.x, core), mul(q.x, a)), mul(f.x, b));
    p.y = add(add(mul(p.y, core), mul(q.y, a)), mul(f.y, b));
    p.z = add(add(mul(p.z, core), mul(q.z, a)), mul(f.z, b));
    px[i] = p;
}

__device__ __forceinline__ bool metered(double y) { return y > 0.0 && isfinite(y); }

// Count of positive finite luminances; also resets the select state.
__global__ void exposure_count(const bh_xyz* __restrict__ px, long long n, ExposureState* st) {
    __shared__ unsigned long long part[kThreads];
    unsigned long long c = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        c += metered(px[i].y) ? 1ull : 0ull;
    part[threadIdx.x] = c;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0 && part[0]) atomicAdd(&st->count, part[0]);
}

// Histogram of the digit at `shift` of the keys that match each target's prefix.
__global__ void exposure_hist(const bh_xyz* __restrict__ px, long long n, ExposureState* st, int shift) {
    __shared__ unsigned int bins[2][256];
    for (int i = threadIdx.x; i < 512; i += blockDim.x) bins[i >> 8][i & 255] = 0u;
    __syncthreads();
    const unsigned long long mask = st->mask;
    const unsigned long long p0 = st->prefix[0], p1 = st->prefix[1];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double y = px[i].y;
        if (!metered(y)) continue;
        const unsigned long long key = (unsigned long long)__double_as_longlong(y);
        const unsigned d = (unsigned)((key >> shift) & 255ull);
        if ((key & mask) == p0) atomicAdd(&bins[0][d], 1u);
        if ((key & mask) == p1) atomicAdd(&bins[1][d], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 512; i += blockDim.x) {
        const unsigned v = bins[i >> 8][i & 255];
        if (v) atomicAdd(&st->hist[i >> 8][i & 255], (unsigned long long)v);
    }
}

// Pick the digit holding each target's order statistic: one thread per digit,
// a block-wide inclusive scan of the counts, and the thread whose range holds
// the rank extends the prefix.  After the last (least significant) digit,
// form the exposure.
constexpr int kPickThreads = 256;

__global__ void __launch_bounds__(kPickThreads)
exposure_pick(ExposureState* st, int shift, int first, int last, double key, double fixed, double* exposure) {
    __shared__ unsigned long long scan[2][kPickThreads];
    const int d = threadIdx.x;
    const unsigned long long m = st->count;
    if (first && m > 0 && d < 2) {
        const double q = (d == 0) ? 0.999 : 0.9999;
        const unsigned long long k = (unsigned long long)(q * (double)(m - 1));
        st->k[d] = (k > m - 1) ? m - 1 : k;
    }
    __syncthreads();
    const unsigned long long c0 = st->hist[0][d], c1 = st->hist[1][d];
    scan[0][d] = c0;
    scan[1][d] = c1;
    __syncthreads();
    for (int off = 1; off < kPickThreads; off <<= 1) {
        const unsigned long long a0 = (d >= off) ? scan[0][d - off] : 0ull;
        const unsigned long long a1 = (d >= off) ? scan[1][d - off] : 0ull;
        __syncthreads();
        scan[0][d] += a0;
        scan[1][d] += a1;
        __syncthreads();
    }
    const unsigned long long k0 = st->k[0], k1 = st->k[1];
    __syncthreads();
    if (m > 0) {
        const unsigned long long e0 = scan[0][d] - c0, e1 = scan[1][d] - c1;   // counts below digit d
        if (c0 && k0 >= e0 && k0 < e0 + c0) {
            st->prefix[0] |= (unsigned long long)d << shift;
            st->k[0] = k0 - e0;
        }
        if (c1 && k1 >= e1 && k1 < e1 + c1) {
            st->prefix[1] |= (unsigned long long)d << shift;
            st->k[1] = k1 - e1;
        }
        if (d == 0) st->mask |= 255ull << shift;
    }
    st->hist[0][d] = 0ull;
    st->hist[1][d] = 0ull;
    __syncthreads();
    if (last && d == 0) {
        double e = fixed;
        if (!(fixed > 0.0)) {
            e = 1.0;
            if (m > 0) {
                const double hi = __longlong_as_double((long long)st->prefix[0]);
                const double peak = __longlong_as_double((long long)st->prefix[1]);
                if (hi > 0.0) e = key / hi;
                if (peak > 0.0) {
                    const double c = 3.0 * key / peak;
                    if (c < e) e = c;
                }
            }
        }
        *exposure = e;
    }
}

__device__ __forceinline__ double aces_curve(double x) {
    const double a = 2.51, b = 0.03, c = 2.43, d = 0.59, e = 0.14;
    return clampd(mul(x, add(mul(a, x), b)) / add(mul(x, add(mul(c, x), d)), e), 0.0, 1.0);
}

__device__ __forceinline__ double srgb_encode(double v) {
    v = clampd(v, 0.0, 1.0);
    return (v <= 0.0031308) ? mul(12.92, v) : sub(mul(1.055, pow(v, 1.0 / 2.4)), 0.055);
}

__global__ void develop_kernel(const bh_xyz* __restrict__ px, long long n, const double* __restrict__ exposure,
                               int tonemap, double log_k, double denom, uint8_t* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double ex = *exposure;
    bh_xyz c = px[i];
    if (!isfinite(c.x) || !isfinite(c.y) || !isfinite(c.z)) c = bh_xyz{0.0, 0.0, 0.0};
    c.x = mul(c.x, ex);
    c.y = mul(c.y, ex);
    c.z = mul(c.z, ex);
    double v[3];
    v[0] = sub(sub(mul(3.2404542, c.x), mul(1.5371385, c.y)), mul(0.4985314, c.z));
    v[1] = add(add(mul(-0.9692660, c.x), mul(1.8760108, c.y)), mul(0.0415560, c.z));
    v[2] = add(sub(mul(0.0556434, c.x), mul(0.2040259, c.y)), mul(1.0572252, c.z));
    double m = v[0];
    if (v[1] < m) m = v[1];
    if (v[2] < m) m = v[2];
    if (!(m >= 0.0)) {
        v[0] = sub(v[0], m);
        v[1] = sub(v[1], m);
        v[2] = sub(v[2], m);
    }
    #pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        double x = (v[ch] < 0.0) ? 0.0 : v[ch];
        switch (tonemap) {
        case BH_TONEMAP_LINEAR: x = clampd(x, 0.0, 1.0); break;
        case BH_TONEMAP_REINHARD: x = x / add(1.0, x); break;
        case BH_TONEMAP_ACES: x = aces_curve(x); break;
        case BH_TONEMAP_LOG:
            x = clampd(log10(add(1.0, mul(log_k, (x < 0.0) ? 0.0 : x))) / denom, 0.0, 1.0);
            break;
        default: {
            const double cap = 0.12, wt = 0.5;
            const double f = aces_curve(x);
            const double l = clampd(log10(add(1.0, mul(log_k, (x < 0.0) ? 0.0 : x))) / denom, 0.0, 1.0);
            const double lift = mul(cap, tanh(mul(wt, l) / cap));
            x = clampd(add(f, mul(lift, sub(1.0, f))), 0.0, 1.0);
            break;
        }
        }
        out[i * 3 + ch] = (uint8_t)lround(mul(255.0, srgb_encode(x)));
    }
}

}  // namespace

cudaError_t launch_display(const DisplayLaunch& L, cudaStream_t s) {
    const long long n = (long long)L.width * L.height;
    if (n <= 0) return cudaSuccess;
    const int blocks = (int)((n + kThreads - 1) / kThreads);
    if (L.glare > 0.0 && L.glare_radius > 0.0) {
        blur_pass<<<blocks, kThreads, 0, s>>>(L.pixels, L.tmp, L.width, L.height, L.k_near, L.r_near, 0);
        blur_pass<<<blocks, kThreads, 0, s>>>(L.tmp, L.nearp, L.width, L.height, L.k_near, L.r_near, 1);
        blur_pass<<<blocks, kThreads, 0, s>>>(L.pixels, L.tmp, L.width, L.height, L.k_far, L.r_far, 0);
        blur_pass<<<blocks, kThreads, 0, s>>>(L.tmp, L.farp, L.width, L.height, L.k_far, L.r_far, 1);
        const double core = 1.0 - L.glare, a = 0.7 * L.glare, b = 0.3 * L.glare;
        glare_combine<<<blocks, kThreads, 0, s>>>(L.pixels, L.nearp, L.farp, n, core, a, b);
    }
    cudaError_t e = cudaMemsetAsync(L.state, 0, sizeof(ExposureState), s);
    if (e != cudaSuccess) return e;
    if (!(L.exposure > 0.0)) {
        const int grid = L.reduce_blocks;
        exposure_count<<<grid, kThreads, 0, s>>>(L.pixels, n, L.state);
        for (int pass = 0; pass < 8; ++pass) {
            const int shift = 56 - 8 * pass;
            exposure_hist<<<grid, kThreads, 0, s>>>(L.pixels, n, L.state, shift);
            exposure_pick<<<1, kPickThreads, 0, s>>>(L.state, shift, pass == 0, pass == 7, L.key, 0.0,
                                                     L.exposure_out);
        }
    } else {
        exposure_pick<<<1, kPickThreads, 0, s>>>(L.state, 0, 0, 1, L.key, L.exposure, L.exposure_out);
    }
    if (L.rgb)
        develop_kernel<<<blocks, kThreads, 0, s>>>(L.pixels, n, L.exposure_out, L.tonemap, L.log_k, L.denom, L.rgb);
    return cudaGetLastError();
}

}  // namespace bhg
