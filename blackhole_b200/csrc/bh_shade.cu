// bh_shade.cu - Shading and stats kernels of the render path.
//
//   shade_kernel      per-pixel shading of the terminated rays (render.cpp:265-393,
//                     disc.h:94-126, spectrum.cpp:123-134, scene.h:111-223) and the
//                     sample average of render.cpp:456-462.
//   reduce kernels    deterministic per-frame stats (render.cpp:481-494): fixed-shape
//                     block reductions, then a fixed-order sum of the block partials.
//
// Everything here is binary64: it runs once per ray, after the integration.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bh_gpu.h"
#include "bh_common.cuh"
#include "bh_frame.h"
#include "bh_launch.h"

namespace bhg {

namespace {

__device__ void blackbody(const double* __restrict__ tab, double T, double o[3]) {
    // spectrum.cpp:123-134
    const double kLogTMin = 1.6989700043360187, kLogTMax = 9.4771212547196626;
    const double lg = log10(dclamp(T, 50.0, 3.0e9));
    const double f = (lg - kLogTMin) / (kLogTMax - kLogTMin) * (kTableN - 1);
    int i = (int)f;
    i = (i < 0) ? 0 : (i > kTableN - 2 ? kTableN - 2 : i);
    const double u = f - i;
    o[0] = exp(__ldg(&tab[i]) * (1.0 - u) + __ldg(&tab[i + 1]) * u);
    o[1] = exp(__ldg(&tab[kTableN + i]) * (1.0 - u) + __ldg(&tab[kTableN + i + 1]) * u);
    o[2] = exp(__ldg(&tab[2 * kTableN + i]) * (1.0 - u) + __ldg(&tab[2 * kTableN + i + 1]) * u);
}

__device__ double circ_energy(double a, double r, int sigma) {
    const double sr = sqrt(r);
    const double num = r * r - 2.0 * r + sigma * a * sr;
    const double den = r * sqrt(r * r - 3.0 * r + 2.0 * sigma * a * sr);
    return num / den;
}
__device__ double circ_angmom(double a, double r, int sigma) {
    const double sr = sqrt(r);
    const double num = sigma * sr * (r * r - 2.0 * sigma * a * sr + a * a);
    const double den = r * sqrt(r * r - 3.0 * r + 2.0 * sigma * a * sr);
    return num / den;
}

// Novikov-Thorne effective temperature (disc.h:94-121, W from disc.h:46-64).
__device__ double disc_temperature(const FrameParams& F, double r) {
    if (r <= F.r_in || r > F.r_out) return 0.0;
    const double a = F.disc_a;
    const int sg = F.disc_sigma;
    const double x = sqrt(r);
    double W = x - F.x0 - 1.5 * a * log(x / F.x0);
    #pragma unroll
    for (int i = 0; i < 3; ++i)
        if (F.pt_c[i] != 0.0) W = W - F.pt_c[i] * log((x - F.pt_x[i]) / F.pt_den[i]);
    const double r32 = r * sqrt(r);
    const double Om = sg / (r32 + sg * a);
    const double dd = r32 + sg * a;
    const double dOm = -sg * 1.5 * sqrt(r) / (dd * dd);
    const double E = circ_energy(a, r, sg);
    const double L = circ_angmom(a, r, sg);
    const double den = E - Om * L;
    if (!(den > 0.0)) return 0.0;
    double Fd = (-dOm) / (4.0 * kPi * r * den * den) * W;
    if (!(Fd > 0.0 && isfinite(Fd))) Fd = 0.0;
    const double Fl = Fd * F.disc_mdot * 2.99792458e8 * 2.99792458e8 / F.disc_rg2;
    if (Fl <= 0.0) return 0.0;
    return pow(Fl / 5.670374419e-8, 0.25);
}

// Position derivatives dr, dth, dphi at a state (the RHS of geodesic.h:58-61).
__device__ void position_rates(const FrameParams& F, const double* y, double d[3]) {
    const double a = F.a, a2 = F.a2;
    const double r = y[1], th = y[2];
    double sn, cs;
    sincos(th, &sn, &cs);
    if (fabs(sn) < 1e-9) sn = (sn < 0.0) ? -1e-9 : 1e-9;
    const double sn2 = sn * sn, cs2 = cs * cs;
    const double Sig = r * r + a2 * cs2;
    const double Del = r * r - 2.0 * r + a2;
    const double SD = Sig * Del;
    const double gtp = -2.0 * a * r / SD;
    const double gpp = (Del - a2 * sn2) / (SD * sn2);
    d[0] = (Del / Sig) * y[5];
    d[1] = (1.0 / Sig) * y[6];
    d[2] = gtp * y[4] + gpp * y[7];
}

// render.cpp:15-26 (normalised at render.cpp:364-366).
__device__ bool sky_direction(const FrameParams& F, const double* y, double v[3]) {
    double dd[3];
    position_rates(F, y, dd);
    const double a = F.a;
    const double r = y[1], th = y[2], ph = y[3];
    const double R = sqrt(r * r + a * a);
    double sn, cs, sp, cp;
    sincos(th, &sn, &cs);
    sincos(ph, &sp, &cp);
    const double dr = dd[0], dth = dd[1], dph = dd[2];
    const double dR = (R > 0.0) ? r / R * dr : dr;
    v[0] = dR * sn * cp + R * cs * dth * cp - R * sn * sp * dph;
    v[1] = dR * sn * sp + R * cs * dth * sp + R * sn * cp * dph;
    v[2] = dr * cs - r * sn * dth;
    const double vn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (!(vn > 0.0)) return false;
    v[0] /= vn; v[1] /= vn; v[2] /= vn;
    return true;
}

// Star field + diffuse background along direction d (scene.h:111-158, 202-223).
__device__ void sky_radiance(const SkyData& sky, const FrameParams& F, const double d[3], double o[3]) {
    o[0] = o[1] = o[2] = 0.0;
    if (sky.n_stars > 0) {
        const double cutoff = F.cutoff, inv2s2 = F.inv2s2, norm = F.psf_norm;
        const double theta = acos(dclamp(d[2], -1.0, 1.0));
        const double phi = atan2(d[1], d[0]);
        const int it = (int)(theta / kPi * kLat);
        const double sn = dmaxr(sin(theta), 1e-6);
        const double dlon = 2.0 * kPi / kLon;
        int span_p = (int)ceil(cutoff / (sn * dlon));
        if (span_p < 1) span_p = 1;
        const int sp = (span_p * 2 + 1 >= kLon) ? kLon / 2 : span_p;
        const int pbase = (int)((phi + kPi) / (2.0 * kPi) * kLon);
        for (int a = -F.span_t; a <= F.span_t; ++a) {
            const int ti = it + a;
            if (ti < 0 || ti >= kLat) continue;
            for (int b = -sp; b <= sp; ++b) {
                int pi = pbase + b;
                pi = ((pi % kLon) + kLon) % kLon;
                const int bin = ti * kLon + pi;
                const int k0 = __ldg(&sky.bin_start[bin]), k1 = __ldg(&sky.bin_start[bin + 1]);
                for (int k = k0; k < k1; ++k) {
                    const double4 s = sky.star_pos[k];
                    const double dot = dclamp(d[0] * s.x + d[1] * s.y + d[2] * s.z, -1.0, 1.0);
                    if (dot < F.cut_dot) continue;   // outside the cutoff, without the acos
                    const double ang = (dot > 0.9999995) ? sqrt(dmaxr(0.0, 2.0 * (1.0 - dot))) : acos(dot);
                    if (ang > cutoff) continue;
                    const double w = norm * exp(-ang * ang * inv2s2) * s.w;
                    const double4 c = sky.star_col[k];
                    o[0] += w * c.x * c.z;
                    o[1] += w;
                    o[2] += w * c.y * c.z;
                }
            }
        }
    }
    if (F.milky_way) {
        double amp;
        if (F.sky_mode == BH_SKY_UNIFORM) {
            amp = sky.diffuse_L;
        } else {
            const double ca = 0.8660254037844387, sa = 0.5;
            const double g1 = ca * d[1] + sa * d[2];
            const double g2 = -sa * d[1] + ca * d[2];
            const double sin_b = dclamp(g2, -1.0, 1.0);
            const double band = exp(-fabs(sin_b) / 0.055);
            const double l = atan2(g1, d[0]);
            const double bulge = 0.55 + 0.45 * exp(-(l * l) / (2.0 * 0.45 * 0.45));
            const double lane = 0.65 + 0.35 * sin(l * 7.3 + sin_b * 41.0) * sin(l * 3.1 - sin_b * 17.0);
            amp = sky.diffuse_L * band * bulge * dmaxr(0.0, lane);
        }
        o[0] += amp * sky.mw_x * sky.mw_inv;
        o[1] += amp;
        o[2] += amp * sky.mw_z * sky.mw_inv;
    }
}

// render.cpp:265-375 for one terminated ray.  Returns g (disc/surface hits)
// and the sky direction (escaped rays) for the per-sample results.
__device__ void shade_one(const SkyData& sky, const FrameParams& F, const HitRecord& hr, double c[3],
                          double* g_out, double dir[3]) {
    c[0] = c[1] = c[2] = 0.0;
    *g_out = 0.0;
    dir[0] = dir[1] = dir[2] = 0.0;
    const double* y = hr.y;
    switch (hr.what) {
    case BH_HIT_DISC: {
        const double r = y[1];
        double T = disc_temperature(F, r);
        if (T <= 0.0) return;
        if (F.hs_enabled) {
            const double t_emit = F.observer_time + y[0];
            const double phi_s = F.hs_phi0 + F.hs_omega * t_emit;
            const double dx = r * cos(y[3]) - F.hs_r * cos(phi_s);
            const double dy = r * sin(y[3]) - F.hs_r * sin(phi_s);
            const double d2 = dx * dx + dy * dy;
            const double f = 1.0 + F.hs_contrast * exp(-0.5 * d2 / (F.hs_sigma * F.hs_sigma));
            T *= pow(f, 0.25);
        }
        // keplerian_four_velocity (kerr.h:260-266) and redshift_factor (render.cpp:31-34)
        const double a = F.disc_a;
        const int sg = F.disc_sigma;
        const double r32 = r * sqrt(r);
        const double Om = sg / (r32 + sg * a);
        const double dsc = r * r * r - 3.0 * r * r + 2.0 * sg * a * r32;
        const double ut = (r32 + sg * a) / sqrt(dmaxr(1e-300, dsc));
        const double ku = y[4] * ut + y[5] * 0.0 + y[6] * 0.0 + y[7] * (Om * ut);
        const double g = (ku > 1e-12) ? 1.0 / ku : 0.0;
        if (g <= 0.0) return;
        *g_out = g;
        blackbody(sky.table, g * T, c);
        return;
    }
    case BH_HIT_SUN: {
        const double a = F.a, r = y[1], th = y[2];
        double sn = sin(th);
        if (fabs(sn) < 1e-9) sn = (sn < 0.0) ? -1e-9 : 1e-9;
        const double cs = cos(th);
        const double Sig = r * r + F.a2 * cs * cs;
        const double mtt = -(1.0 - 2.0 * r / Sig);
        if (mtt >= 0.0) return;
        const double ut = 1.0 / sqrt(-mtt);
        const double ku = y[4] * ut;
        const double g = (ku > 1e-12) ? 1.0 / ku : 0.0;
        if (g <= 0.0) return;
        *g_out = g;
        // Viewing direction (normalised when non-zero, render.cpp:311-316) and
        // Eddington limb darkening (scene.h:266-276).
        double v[3];
        (void)sky_direction(F, y, v);
        const double rr = sqrt(r * r + a * a);
        const double p[3] = {rr * sin(th) * cos(y[3]), rr * sin(th) * sin(y[3]), r * cos(th)};
        double limb = 1.0;
        double nrm[3] = {p[0] - F.sun_c[0], p[1] - F.sun_c[1], p[2] - F.sun_c[2]};
        const double len = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        if (len > 0.0) {
            nrm[0] /= len; nrm[1] /= len; nrm[2] /= len;
            const double mu = dclamp(-(nrm[0] * v[0] + nrm[1] * v[1] + nrm[2] * v[2]), 0.0, 1.0);
            limb = (2.0 + 3.0 * mu) / 5.0;
        }
        blackbody(sky.table, g * F.sun_T_eff / F.sun_redshift_div, c);
        c[0] *= limb; c[1] *= limb; c[2] *= limb;
        return;
    }
    case BH_HIT_STAR: {
        const double r = y[1], th = y[2], ph = y[3];
        const double sn = sin(th);
        const double norm2 = 1.0 - 2.0 / F.ns_R - F.ns_Omega * F.ns_Omega * F.ns_R * F.ns_R * sn * sn;
        const double ut = (norm2 > 1e-12) ? 1.0 / sqrt(norm2) : 1.0;
        const double ku = y[4] * ut + y[7] * (F.ns_Omega * ut);
        if (!(ku > 1e-12)) return;
        const double g = 1.0 / ku;
        *g_out = g;
        double T = F.ns_T_eff;
        if (F.ns_caps) {
            const double t_emit = F.observer_time + y[0];
            const double phase = F.ns_cap_phase0 + F.ns_Omega * t_emit;
            const double m0 = sin(F.ns_cap_tilt) * cos(phase), m1 = sin(F.ns_cap_tilt) * sin(phase),
                         m2 = cos(F.ns_cap_tilt);
            const double n0 = sin(th) * cos(ph), n1 = sin(th) * sin(ph), n2 = cos(th);
            double ang = acos(dclamp(n0 * m0 + n1 * m1 + n2 * m2, -1.0, 1.0));
            if (F.ns_two_caps) ang = dminr(ang, kPi - ang);
            if (ang <= F.ns_cap_radius) {
                const double edge = 0.9 * F.ns_cap_radius;
                if (ang <= edge) {
                    T = F.ns_cap_T;
                } else {
                    const double u = (ang - edge) / (F.ns_cap_radius - edge);
                    const double w = 0.5 * (1.0 + cos(kPi * u));
                    T = F.ns_T_eff + (F.ns_cap_T - F.ns_T_eff) * w;
                }
            }
        }
        const double f = 1.0 - 2.0 / r;
        const double mu = (f > 0.0) ? dclamp(-y[5] * sqrt(f) / ku, 0.0, 1.0) : 1.0;
        const double limb = (2.0 + 3.0 * mu) / 5.0;
        blackbody(sky.table, g * T, c);
        c[0] *= limb; c[1] *= limb; c[2] *= limb;
        return;
    }
    case BH_HIT_SKY: {
        double v[3];
        if (!sky_direction(F, y, v)) return;
        dir[0] = v[0]; dir[1] = v[1]; dir[2] = v[2];
        if (!F.stars_enabled) return;
        sky_radiance(sky, F, v, c);
        return;
    }
    default:
        return;
    }
}

struct ShadeArgs {
    const FrameParams* frames;
    const long long* frame_pixel_end;
    int nframes;
    long long total_pixels;
    const HitRecord* hits;
    SkyData sky;
    bh_xyz* pixels;
    bh_ray_result* rays;
    double* pixel_lum;
    const double* jet;
    long long pixel_lo;
};

__global__ void shade_kernel(ShadeArgs A) {
    const long long gp = A.pixel_lo + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gp >= A.total_pixels) return;
    const int f = find_frame(A.frame_pixel_end, A.nframes, gp);
    const FrameParams& F = A.frames[f];
    const long long p = gp - F.pixel_begin;        // frame-local pixel, band order
    int px, py;
    pixel_xy(F.width, F.height, p, &px, &py);
    const int SS = F.S * F.S;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < SS; ++k) {
        const long long rid = F.ray_begin + p * SS + k;
        const HitRecord hr = A.hits[rid];
        double c[3], g, dir[3];
        shade_one(A.sky, F, hr, c, &g, dir);
        // Whatever the ray ended on, the jet light it collected on the way is
        // added in the jet's one colour (render.cpp:377-392).
        const double jet = (F.jet_enabled && A.jet) ? A.jet[rid] : 0.0;
        if (jet > 0.0) {
            c[0] += F.jet_col[0] * jet;
            c[1] += F.jet_col[1] * jet;
            c[2] += F.jet_col[2] * jet;
        }
        acc[0] += c[0]; acc[1] += c[1]; acc[2] += c[2];
        if (A.rays) {
            bh_ray_result& o = A.rays[((long long)py * F.width + px) * SS + k];
            o.what = hr.what;
            o.steps = hr.steps;
            #pragma unroll
            for (int i = 0; i < 8; ++i) o.y[i] = hr.y[i];
            o.g = g;
            o.dir[0] = dir[0]; o.dir[1] = dir[1]; o.dir[2] = dir[2];
            o.xyz.x = c[0]; o.xyz.y = c[1]; o.xyz.z = c[2];
            o.attempts = hr.attempts;
            o.reserved = 0;
            o.max_norm = hr.max_norm;
            o.max_q = hr.max_q;
            o.jet = jet;
        }
    }
    const double w = F.inv_SS;
    bh_xyz& out = A.pixels[F.pixel_begin + (long long)py * F.width + px];
    out.x = acc[0] * w;
    out.y = acc[1] * w;
    out.z = acc[2] * w;
    A.pixel_lum[gp] = acc[1] * w;
}

// ---- deterministic stats reduction ------------------------------------------

struct ReduceArgs {
    const FrameParams* frames;
    int nframes;
    const HitRecord* hits;
    const double* pixel_lum;
    const double* jet;
    FrameStats* partials;
    FrameStats* out;
    int bpf;
};

__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

constexpr int kRedThreads = 256;

__global__ void __launch_bounds__(kRedThreads) reduce_partial_kernel(ReduceArgs A) {
    const int f = blockIdx.y;
    const FrameParams& F = A.frames[f];
    __shared__ unsigned long long s_cnt[kRedThreads][10];
    __shared__ double s_max[kRedThreads][2];
    __shared__ double s_flux[kRedThreads];
    unsigned long long c[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double* jet = (F.jet_enabled && A.jet) ? A.jet + F.ray_begin : nullptr;
    double mn = 0.0, mq = 0.0, flux = 0.0;
    const long long stride = (long long)A.bpf * kRedThreads;
    for (long long i = (long long)blockIdx.x * kRedThreads + threadIdx.x; i < F.n_rays; i += stride) {
        const HitRecord& h = A.hits[F.ray_begin + i];
        c[0] += 1;
        c[1] += (unsigned long long)h.steps;
        c[2] += (unsigned long long)h.attempts;
        if (h.what >= 0 && h.what <= 5) c[3 + h.what] += 1;
        mn = dmaxr(mn, h.max_norm);
        mq = dmaxr(mq, h.max_q);
        if (jet && jet[i] > 0.0) c[9] += 1;
    }
    const long long npx = (long long)F.width * F.height;
    for (long long i = (long long)blockIdx.x * kRedThreads + threadIdx.x; i < npx; i += stride)
        flux += A.pixel_lum[F.pixel_begin + i];
    for (int k = 0; k < 10; ++k) s_cnt[threadIdx.x][k] = c[k];
    s_max[threadIdx.x][0] = mn;
    s_max[threadIdx.x][1] = mq;
    s_flux[threadIdx.x] = flux;
    __syncthreads();
    for (int off = kRedThreads / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            for (int k = 0; k < 10; ++k) s_cnt[threadIdx.x][k] += s_cnt[threadIdx.x + off][k];
            s_max[threadIdx.x][0] = dmaxr(s_max[threadIdx.x][0], s_max[threadIdx.x + off][0]);
            s_max[threadIdx.x][1] = dmaxr(s_max[threadIdx.x][1], s_max[threadIdx.x + off][1]);
            s_flux[threadIdx.x] += s_flux[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        FrameStats& o = A.partials[(long long)f * A.bpf + blockIdx.x];
        o.rays = s_cnt[0][0];
        o.steps = s_cnt[0][1];
        o.attempts = s_cnt[0][2];
        o.captured = s_cnt[0][3 + BH_HIT_HORIZON];
        o.disc_hits = s_cnt[0][3 + BH_HIT_DISC];
        o.sun_hits = s_cnt[0][3 + BH_HIT_SUN];
        o.star_hits = s_cnt[0][3 + BH_HIT_STAR];
        o.escaped = s_cnt[0][3 + BH_HIT_SKY];
        o.exhausted = s_cnt[0][3 + BH_HIT_EXHAUSTED];
        o.jet_rays = s_cnt[0][9];
        o.max_norm_bits = dbits(s_max[0][0]);
        o.max_q_bits = dbits(s_max[0][1]);
        o.total_flux = s_flux[0];
    }
}

// One block per frame: thread t sums the partials t, t + kRedThreads, ... in
// that order, then a fixed tree combines the threads: the same bits on every
// run.
__global__ void __launch_bounds__(kRedThreads) reduce_final_kernel(ReduceArgs A) {
    const int f = blockIdx.x;
    __shared__ unsigned long long s_cnt[kRedThreads][10];
    __shared__ double s_max[kRedThreads][2];
    __shared__ double s_flux[kRedThreads];
    unsigned long long c[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    double mn = 0.0, mq = 0.0, flux = 0.0;
    for (int b = threadIdx.x; b < A.bpf; b += kRedThreads) {
        const FrameStats& p = A.partials[(long long)f * A.bpf + b];
        c[0] += p.rays; c[1] += p.steps; c[2] += p.attempts;
        c[3] += p.captured; c[4] += p.disc_hits; c[5] += p.sun_hits;
        c[6] += p.star_hits; c[7] += p.escaped; c[8] += p.exhausted; c[9] += p.jet_rays;
        mn = dmaxr(mn, __longlong_as_double((long long)p.max_norm_bits));
        mq = dmaxr(mq, __longlong_as_double((long long)p.max_q_bits));
        flux += p.total_flux;
    }
    for (int k = 0; k < 10; ++k) s_cnt[threadIdx.x][k] = c[k];
    s_max[threadIdx.x][0] = mn;
    s_max[threadIdx.x][1] = mq;
    s_flux[threadIdx.x] = flux;
    __syncthreads();
    for (int off = kRedThreads / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            for (int k = 0; k < 10; ++k) s_cnt[threadIdx.x][k] += s_cnt[threadIdx.x + off][k];
            s_max[threadIdx.x][0] = dmaxr(s_max[threadIdx.x][0], s_max[threadIdx.x + off][0]);
            s_max[threadIdx.x][1] = dmaxr(s_max[threadIdx.x][1], s_max[threadIdx.x + off][1]);
            s_flux[threadIdx.x] += s_flux[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        FrameStats t = {};
        t.rays = s_cnt[0][0]; t.steps = s_cnt[0][1]; t.attempts = s_cnt[0][2];
        t.captured = s_cnt[0][3]; t.disc_hits = s_cnt[0][4]; t.sun_hits = s_cnt[0][5];
        t.star_hits = s_cnt[0][6]; t.escaped = s_cnt[0][7]; t.exhausted = s_cnt[0][8];
        t.jet_rays = s_cnt[0][9];
        t.max_norm_bits = dbits(s_max[0][0]);
        t.max_q_bits = dbits(s_max[0][1]);
        t.total_flux = s_flux[0];
        A.out[f] = t;
    }
}


// Device shading functions at given inputs (known-answer tests): what 0,
// the disc's effective temperature at radii in[i]; what 1, the blackbody
// XYZ of temperatures in[i] from the device table (3 per input).
__global__ void eval_shade_kernel(int what, const FrameParams* __restrict__ Fp, const double* __restrict__ tab,
                                  const double* __restrict__ in, long long n, double* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (what == 0) out[i] = disc_temperature(*Fp, in[i]);
    else blackbody(tab, in[i], out + 3 * i);
}

}  // namespace

cudaError_t launch_eval_shade(int what, const FrameParams* d_frame, const double* d_table, const double* d_in,
                              long long n, double* d_out, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    eval_shade_kernel<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(what, d_frame, d_table, d_in, n, d_out);
    return cudaGetLastError();
}

cudaError_t launch_shade(const ShadeLaunch& L, cudaStream_t stream) {
    if (L.total_pixels <= 0) return cudaSuccess;
    ShadeArgs A;
    A.frames = L.frames;
    A.frame_pixel_end = L.frame_pixel_end;
    A.nframes = L.nframes;
    A.total_pixels = L.total_pixels;
    A.hits = L.hits;
    A.sky = L.sky;
    A.pixels = L.pixels;
    A.rays = L.rays;
    A.pixel_lum = L.pixel_lum;
    A.jet = L.jet;
    A.pixel_lo = L.pixel_lo;
    const int bs = 128;
    const long long grid = (L.total_pixels - L.pixel_lo + bs - 1) / bs;
    if (grid <= 0) return cudaSuccess;
    shade_kernel<<<(unsigned)grid, bs, 0, stream>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_reduce(const ReduceLaunch& L, cudaStream_t stream) {
    ReduceArgs A;
    A.frames = L.frames;
    A.nframes = L.nframes;
    A.hits = L.hits;
    A.pixel_lum = L.pixel_lum;
    A.jet = L.jet;
    A.partials = L.partials;
    A.out = L.out;
    A.bpf = L.blocks_per_frame;
    reduce_partial_kernel<<<dim3(L.blocks_per_frame, L.nframes), kRedThreads, 0, stream>>>(A);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    reduce_final_kernel<<<L.nframes, kRedThreads, 0, stream>>>(A);
    return cudaGetLastError();
}

}  // namespace bhg
