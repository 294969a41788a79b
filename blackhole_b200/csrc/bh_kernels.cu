// bh_kernels.cu - sm_100a kernels of the geodesic render path.
//
//   trace_kernel<Fp64|Mixed>  persistent work-queue integrator: ray set-up
//                             (render.cpp:440-451, geodesic.h:215-231), the
//                             DP5(4) step loop with PI control and dense output
//                             (geodesic.h:123-204), per-step invariant
//                             diagnostics (render.cpp:139-145) and event
//                             location (render.cpp:158-251).
//   shade_kernel              per-pixel shading of the terminated rays
//                             (render.cpp:265-393, disc.h, spectrum.cpp:123-134,
//                             scene.h:111-223) and the sample average.
//   reduce kernels            deterministic per-frame stats (render.cpp:481-494).
//
// One thread owns one ray at a time.  A warp refills the lanes freed by rays
// that terminated early from a global atomic queue, with one atomicAdd per
// refill and ballot/popc compaction of the new ray ids, so that short rays
// (captured, direct disc hits) do not leave lanes idle behind long ones.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bh_gpu.h"
#include "bh_frame.h"
#include "bh_launch.h"

namespace bhg {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr unsigned kFull = 0xffffffffu;

// ---- Dormand-Prince 5(4) tableau (Hairer, Norsett & Wanner II.4) -----------
constexpr double A21 = 1.0 / 5.0;
constexpr double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
constexpr double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
constexpr double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0, A53 = 64448.0 / 6561.0,
                 A54 = -212.0 / 729.0;
constexpr double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0, A63 = 46732.0 / 5247.0,
                 A64 = 49.0 / 176.0, A65 = -5103.0 / 18656.0;
constexpr double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0,
                 B5 = -2187.0 / 6784.0, B6 = 11.0 / 84.0;
constexpr double E1 = 35.0 / 384.0 - 5179.0 / 57600.0;
constexpr double E3 = 500.0 / 1113.0 - 7571.0 / 16695.0;
constexpr double E4 = 125.0 / 192.0 - 393.0 / 640.0;
constexpr double E5 = -2187.0 / 6784.0 - (-92097.0 / 339200.0);
constexpr double E6 = 11.0 / 84.0 - 187.0 / 2100.0;
constexpr double E7 = 0.0 - 1.0 / 40.0;
constexpr double D1 = -12715105075.0 / 11282082432.0, D3 = 87487479700.0 / 32700410799.0,
                 D4 = -10690763975.0 / 1880347072.0, D5 = 701980252875.0 / 199316789632.0,
                 D6 = -1453857185.0 / 822651844.0, D7 = 69997945.0 / 29380423.0;
// PI controller (geodesic.h:170-173): alpha = 0.7/5, beta = 0.4/5, safety 0.9.
constexpr double kAlpha = 0.7 / 5.0, kBeta = 0.4 / 5.0;

// ---- precision policies ------------------------------------------------------
struct Fp64 {
    using R = double;
    static constexpr bool kMixed = false;
    __device__ static __forceinline__ void sc(double x, double* s, double* c) { sincos(x, s, c); }
    __device__ static __forceinline__ double rcp(double x) { return 1.0 / x; }
};

struct Mixed {
    using R = float;
    static constexpr bool kMixed = true;
    __device__ static __forceinline__ void sc(float x, float* s, float* c) { sincosf(x, s, c); }
    __device__ static __forceinline__ float rcp(float x) {
        float r;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
        return r;
    }
};

// Exact (non-contracted) double arithmetic, so that ray set-up reproduces the
// host computation bit for bit.
__device__ __forceinline__ double xm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xa(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xs(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ double dmaxr(double a, double b) { return (a < b) ? b : a; }  // std::max
__device__ __forceinline__ double dminr(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dclamp(double v, double lo, double hi) {
    return (v < lo) ? lo : (hi < v) ? hi : v;
}

// splitmix64 output for state s (scene.h:30-36).
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double u53(uint64_t z) { return (double)(z >> 11) * 0x1.0p-53; }

// Pixel of a frame-local pixel index.  Pixels are enumerated in bands of four
// rows, column by column inside a band, so that the 32 rays of a warp cover an
// 8 x 4 patch of the image (coherent paths) rather than 32 pixels of one row.
__device__ __forceinline__ void pixel_xy(int W, int H, long long p, int* x, int* y) {
    const long long band_px = 4LL * W;
    const int band = (int)(p / band_px);
    const int rel = (int)(p - (long long)band * band_px);
    const int y0 = 4 * band;
    const int bh = min(4, H - y0);
    *x = rel / bh;
    *y = y0 + rel % bh;
}

__device__ __forceinline__ int find_frame(const long long* __restrict__ ends, int n, long long id) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (id < __ldg(&ends[mid])) hi = mid; else lo = mid + 1;
    }
    return lo;
}

// Initial photon state of a ray (render.cpp:440-451, scene.h:356-384,
// geodesic.h:215-231) and its Carter constant Q0 (kerr.h:342-348).
__device__ void ray_setup(const FrameParams& F, long long local_id, double y[8], double* Q0) {
    const int S = F.S;
    const long long pixel = local_id / (S * S);
    const int k = (int)(local_id - pixel * (S * S));
    const int sy = k / S, sx = k - (k / S) * S;
    int px, py;
    pixel_xy(F.width, F.height, pixel, &px, &py);
    const uint64_t s0 = F.seed ^ ((uint64_t)py << 32) ^ ((uint64_t)px * 0x9E3779B97F4A7C15ull);
    const uint64_t g = 0x9E3779B97F4A7C15ull;
    const double u1 = u53(mix64(s0 + (uint64_t)(2 * k + 1) * g));
    const double u2 = u53(mix64(s0 + (uint64_t)(2 * k + 2) * g));
    const double jx = xm(xa((double)sx, u1), F.inv_S);
    const double jy = xm(xa((double)sy, u2), F.inv_S);
    const double su = xs(__ddiv_rn(xm(2.0, xa((double)px, jx)), (double)F.width), 1.0);
    const double sv = xs(1.0, __ddiv_rn(xm(2.0, xa((double)py, jy)), (double)F.height));
    // Camera::ray_direction
    double x = xm(su, F.tanf);
    double yy = __ddiv_rn(xm(sv, F.tanf), F.aspect);
    const double z = 1.0;
    if (F.has_roll) {
        const double xr = xs(xm(F.cr, x), xm(F.sr, yy));
        const double yr = xa(xm(F.sr, x), xm(F.cr, yy));
        x = xr; yy = yr;
    }
    const double y2 = xs(xm(F.cp, yy), xm(F.sp, z));
    const double z2 = xa(xm(F.sp, yy), xm(F.cp, z));
    const double x2 = xa(xm(F.cy, x), xm(F.sy, z2));
    const double z3 = xa(xm(-F.sy, x), xm(F.cy, z2));
    const double v0 = -z3, v1 = -y2, v2 = x2;
    const double n = __dsqrt_rn(xa(xa(xm(v0, v0), xm(v1, v1)), xm(v2, v2)));
    const double d0 = __ddiv_rn(v0, n), d1 = __ddiv_rn(v1, n), d2 = __ddiv_rn(v2, n);
    // make_photon, past directed: p^mu = -(e0 - d^i e_i), then lowered.
    const double zero = 0.0;
    const double p0 = -xa(F.tet00, xm(-1.0, xa(xa(xm(d0, zero), xm(d1, zero)), xm(d2, zero))));
    const double p1 = -xa(zero, xm(-1.0, xa(xa(xm(d0, F.tet11), xm(d1, zero)), xm(d2, zero))));
    const double p2 = -xa(zero, xm(-1.0, xa(xa(xm(d0, zero), xm(d1, F.tet22)), xm(d2, zero))));
    const double p3 = -xa(F.tet03, xm(-1.0, xa(xa(xm(d0, zero), xm(d1, zero)), xm(d2, F.tet33))));
    y[0] = 0.0;
    y[1] = F.cam_r;
    y[2] = F.cam_th;
    y[3] = F.cam_ph;
    y[4] = xa(xm(F.ml_tt, p0), xm(F.ml_tp, p3));
    y[5] = xm(F.ml_rr, p1);
    y[6] = xm(F.ml_thth, p2);
    y[7] = xa(xm(F.ml_tp, p0), xm(F.ml_pp, p3));
    // invariants(y).Q with m2 = 0 (carter_constant at the camera).
    const double E = -y[4], Lz = y[7], pth = y[6];
    *Q0 = xa(xm(pth, pth), xm(F.cam_cs2, xa(xm(xm(F.a, F.a), xs(0.0, xm(E, E))),
                                              __ddiv_rn(xm(Lz, Lz), F.cam_sn2))));
}

// ---- the geodesic right-hand side -------------------------------------------
//
// Hamilton's equations for H = 1/2 g^{mu nu} p_mu p_nu (geodesic.h:50-71).
// The same function of (r, theta, p) is evaluated here in Carter's separated
// form of the Kerr inverse metric,
//   2 Sigma H = Delta p_r^2 + p_th^2 + (L_z - a E sin^2)^2 / sin^2
//               - ((r^2 + a^2) E - a L_z)^2 / Delta,
// with E = -p_t and L_z = p_phi constant (dp_t = dp_phi = 0 exactly), which
// needs three reciprocals instead of fifteen divisions.  The constraint H = 0
// is not imposed: B below is the full bracket.
template <class P>
struct Lane {
    using R = typename P::R;
    R y[6];                 // t, r, th, phi, p_r, p_th
    R k1[6];
    R E, Lz, aR, a2R, aE, aLz, a2E2, Lz2;
    double pt, pph;         // exact p_t, p_phi
    double a, a2, rp, rm;
    double h, err_prev, errp_pow;
    double Q0, inv_Q0;
    double max_norm, max_q;
    R c0;                   // cos(th) at y
    int factored;
    int steps, tries, attempts;
    int have_k1;
    int bad_sc;             // atol + rtol |p_t| or |p_phi| is zero: error norm is NaN
    long long gid;
    int frame;
};

template <class P>
struct Aux {
    typename P::R cs, sn2, cs2;
    double Sig, Del;
};

template <class P>
__device__ __forceinline__ void rhs(const Lane<P>& L, typename P::R r, typename P::R th,
                                    typename P::R pr, typename P::R pth, typename P::R* d,
                                    Aux<P>* aux) {
    using R = typename P::R;
    R sn, cs;
    P::sc(th, &sn, &cs);
    if (fabs(sn) < R(1e-9)) sn = (sn < R(0)) ? R(-1e-9) : R(1e-9);   // kerr.h:51
    const R sn2 = sn * sn, cs2 = cs * cs;
    // Sigma and Delta in binary64 in both precisions (Delta cancels near r_+).
    const double rd = (double)r;
    const double Sig = rd * rd + L.a2 * (double)cs2;
    const double Del = L.factored ? (rd - L.rp) * (rd - L.rm) : (rd * rd - 2.0 * rd + L.a2);
    const R S = (R)Sig, D = (R)Del;
    const R iS = P::rcp(S), iD = P::rcp(D), isn2 = P::rcp(sn2);
    const R r2a2 = r * r + L.a2R;
    const R K = r2a2 * L.E - L.aLz;
    const R Lp = L.Lz - L.aE * sn2;
    const R KiD = K * iD;
    const R B = D * pr * pr + pth * pth + Lp * Lp * isn2 - K * KiD;
    const R Dr = R(2) * r - R(2);
    d[0] = iS * (L.aR * Lp + r2a2 * KiD);
    d[1] = D * pr * iS;
    d[2] = pth * iS;
    d[3] = iS * (Lp * isn2 + L.aR * KiD);
    d[4] = R(-0.5) * iS * (Dr * pr * pr - R(4) * r * L.E * KiD + Dr * KiD * KiD - R(2) * r * B * iS);
    d[5] = -sn * cs * iS * (L.a2E2 - L.Lz2 * isn2 * isn2 + L.a2R * B * iS);
    if (aux) {
        aux->cs = cs;
        aux->sn2 = sn2;
        aux->cs2 = cs2;
        aux->Sig = Sig;
        aux->Del = Del;
    }
}

// Dense-output coefficients of one component (geodesic.h:176-185).
struct DenseC { double r1, r2, r3, r4, r5; };

__device__ __forceinline__ DenseC dense_coef(double h, double y, double yn, double k1, double k3,
                                             double k4, double k5, double k6, double k7) {
    DenseC c;
    c.r1 = y;
    c.r2 = yn - y;
    c.r3 = h * k1 - c.r2;
    c.r4 = c.r2 - h * k7 - c.r3;
    c.r5 = h * (D1 * k1 + D3 * k3 + D4 * k4 + D5 * k5 + D6 * k6 + D7 * k7);
    return c;
}
__device__ __forceinline__ double dense_eval(const DenseC& c, double s) {
    const double s1 = 1.0 - s;
    return c.r1 + s * (c.r2 + s1 * (c.r3 + s * (c.r4 + s1 * c.r5)));
}

struct TraceArgs {
    const FrameParams* frames;
    const long long* frame_ray_end;
    int nframes;
    long long total_rays;
    HitRecord* hits;
    QueueState* queue;
    int rays_per_thread;
    int refill;
    unsigned long long budget;
};

template <class P>
__device__ __forceinline__ void write_hit(const TraceArgs& A, const Lane<P>& L, int what,
                                          const double y8[8]) {
    HitRecord* o = &A.hits[L.gid];
    #pragma unroll
    for (int i = 0; i < 8; ++i) o->y[i] = y8[i];
    o->max_norm = L.max_norm;
    o->max_q = L.max_q;
    o->what = what;
    o->steps = L.steps;
    o->attempts = L.attempts;
}

template <class P>
__device__ __forceinline__ void lane_state8(const Lane<P>& L, double y8[8]) {
    y8[0] = (double)L.y[0];
    y8[1] = (double)L.y[1];
    y8[2] = (double)L.y[2];
    y8[3] = (double)L.y[3];
    y8[4] = L.pt;
    y8[5] = (double)L.y[4];
    y8[6] = (double)L.y[5];
    y8[7] = L.pph;
}

// Start ray `gid`; returns false when it terminates at once (max_steps <= 0).
template <class P>
__device__ bool start_ray(const TraceArgs& A, Lane<P>& L, long long gid) {
    using R = typename P::R;
    L.gid = gid;
    L.frame = find_frame(A.frame_ray_end, A.nframes, gid);
    const FrameParams& F = A.frames[L.frame];
    double y8[8], Q0;
    ray_setup(F, gid - F.ray_begin, y8, &Q0);
    L.y[0] = (R)y8[0]; L.y[1] = (R)y8[1]; L.y[2] = (R)y8[2]; L.y[3] = (R)y8[3];
    L.y[4] = (R)y8[5]; L.y[5] = (R)y8[6];
    L.pt = y8[4];
    L.pph = y8[7];
    L.a = F.a;
    L.a2 = F.a2;
    L.rp = F.r_plus;
    L.rm = F.r_minus;
    L.factored = F.factored_delta;
    const double E = -y8[4], Lz = y8[7];
    L.E = (R)E;
    L.Lz = (R)Lz;
    L.aR = (R)F.a;
    L.a2R = (R)F.a2;
    L.aE = (R)(F.a * E);
    L.aLz = (R)(F.a * Lz);
    L.a2E2 = (R)(F.a2 * E * E);
    L.Lz2 = (R)(Lz * Lz);
    L.h = F.h0;
    L.err_prev = 1e-4;
    L.errp_pow = pow(1e-4, kBeta);
    L.Q0 = Q0;
    L.inv_Q0 = 1.0 / (fabs(Q0) + 1e-12);
    L.max_norm = 0.0;
    L.max_q = 0.0;
    L.steps = 0;
    L.tries = 0;
    L.attempts = 0;
    L.have_k1 = 0;
    L.bad_sc = (F.atol + F.rtol * fabs(L.pt) == 0.0) || (F.atol + F.rtol * fabs(L.pph) == 0.0);
    if (F.max_steps <= 0) {
        write_hit(A, L, BH_HIT_EXHAUSTED, y8);
        return false;
    }
    return true;
}

// One step attempt.  Returns true when the ray terminated (hit written).
template <class P>
__device__ bool attempt(const TraceArgs& A, Lane<P>& L) {
    using R = typename P::R;
    const FrameParams& F = A.frames[L.frame];
    if (L.tries == 0) {
        // render.cpp:130-131: keep the step resolved near the hole and unable
        // to skip over the disc plane.
        const double hmax = 0.05 * dmaxr(1.0, (double)L.y[1] - F.r_h) + 0.01;
        if (L.h > hmax) L.h = hmax;
    }
    if (!L.have_k1) {
        Aux<P> ax;
        rhs<P>(L, L.y[1], L.y[2], L.y[4], L.y[5], L.k1, &ax);
        L.c0 = ax.cs;
        L.have_k1 = 1;
    }
    const R h = (R)L.h;
    R t[6], k2[6], k3[6], k4[6], k5[6], k6[6], k7[6], yn[6];
    #pragma unroll
    for (int i = 0; i < 6; ++i) t[i] = L.y[i] + h * R(A21) * L.k1[i];
    rhs<P>(L, t[1], t[2], t[4], t[5], k2, nullptr);
    #pragma unroll
    for (int i = 0; i < 6; ++i) t[i] = L.y[i] + h * (R(A31) * L.k1[i] + R(A32) * k2[i]);
    rhs<P>(L, t[1], t[2], t[4], t[5], k3, nullptr);
    #pragma unroll
    for (int i = 0; i < 6; ++i)
        t[i] = L.y[i] + h * (R(A41) * L.k1[i] + R(A42) * k2[i] + R(A43) * k3[i]);
    rhs<P>(L, t[1], t[2], t[4], t[5], k4, nullptr);
    #pragma unroll
    for (int i = 0; i < 6; ++i)
        t[i] = L.y[i] + h * (R(A51) * L.k1[i] + R(A52) * k2[i] + R(A53) * k3[i] + R(A54) * k4[i]);
    rhs<P>(L, t[1], t[2], t[4], t[5], k5, nullptr);
    #pragma unroll
    for (int i = 0; i < 6; ++i)
        t[i] = L.y[i] + h * (R(A61) * L.k1[i] + R(A62) * k2[i] + R(A63) * k3[i] +
                             R(A64) * k4[i] + R(A65) * k5[i]);
    rhs<P>(L, t[1], t[2], t[4], t[5], k6, nullptr);
    #pragma unroll
    for (int i = 0; i < 6; ++i)
        yn[i] = L.y[i] + h * (R(B1) * L.k1[i] + R(B3) * k3[i] + R(B4) * k4[i] + R(B5) * k5[i] +
                              R(B6) * k6[i]);
    Aux<P> ax7;
    rhs<P>(L, yn[1], yn[2], yn[4], yn[5], k7, &ax7);

    // Scaled RMS error over all eight components (geodesic.h:157-166); the
    // p_t and p_phi terms are exactly zero.  Accumulated in binary64.
    double err2 = 0.0;
    #pragma unroll
    for (int i = 0; i < 6; ++i) {
        const R e = h * (R(E1) * L.k1[i] + R(E3) * k3[i] + R(E4) * k4[i] + R(E5) * k5[i] +
                         R(E6) * k6[i] + R(E7) * k7[i]);
        const double sc = F.atol + F.rtol * dmaxr(fabs((double)L.y[i]), fabs((double)yn[i]));
        const double q = (double)e / sc;
        err2 += q * q;
    }
    double err = sqrt(err2 / 8.0);
    if (L.bad_sc || !isfinite(err)) err = 1e10;
    ++L.attempts;

    double fac;
    if (P::kMixed) {
        const float ef = (float)dmaxr(err, 1e-16);
        fac = (double)(0.9f * __powf(ef, (float)-kAlpha)) * L.errp_pow;
    } else {
        fac = 0.9 * pow(dmaxr(err, 1e-16), -kAlpha) * L.errp_pow;
    }
    fac = dclamp(fac, 0.2, 5.0);

    if (!(err <= 1.0)) {
        L.h *= dminr(fac, 1.0);
        if (++L.tries > 40 || fabs(L.h) < 1e-14) {
            // render.cpp:133-136: a step that cannot be made is a capture; the
            // reported state is the ray's initial one.
            double y8[8], Q0;
            ray_setup(F, L.gid - F.ray_begin, y8, &Q0);
            write_hit(A, L, BH_HIT_HORIZON, y8);
            return true;
        }
        return false;
    }

    // ---- accepted ---------------------------------------------------------
    L.tries = 0;
    ++L.steps;
    const double rn = (double)yn[1];
    {
        // Invariant diagnostics at y_new (render.cpp:139-145) in binary64:
        // the relative null norm uses the five terms of g^{ab} p_a p_b
        // (kerr.h:301-321), all scaled by Sigma Delta sin^2 > 0.
        const double sn2 = (double)ax7.sn2, cs2 = (double)ax7.cs2, Del = ax7.Del;
        const double pr = (double)yn[4], pth = (double)yn[5];
        const double rpa = rn * rn + L.a2;
        const double Ak = rpa * rpa - L.a2 * Del * sn2;
        const double T1 = -Ak * L.pt * L.pt * sn2;
        const double T2 = -4.0 * L.a * rn * L.pt * L.pph * sn2;
        const double T3 = Del * Del * sn2 * pr * pr;
        const double T4 = Del * sn2 * pth * pth;
        const double T5 = (Del - L.a2 * sn2) * L.pph * L.pph;
        const double nrm = T1 + T2 + T3 + T4 + T5;
        const double scl = fabs(T1) + fabs(T2) + fabs(T3) + fabs(T4) + fabs(T5);
        const double nrel = (scl > 0.0) ? fabs(nrm) / scl : fabs(nrm);
        L.max_norm = dmaxr(L.max_norm, nrel);
        const double E = -L.pt, Lz = L.pph;
        const double Q = pth * pth + cs2 * (L.a2 * (0.0 - E * E) + Lz * Lz / sn2);
        L.max_q = dmaxr(L.max_q, fabs(Q - L.Q0) * L.inv_Q0);
    }

    const double hd = L.h;
    // ---- events (render.cpp:158-251) --------------------------------------
    int what = -1;
    double yh[8];
    if (F.ns_enabled && rn <= F.ns_R) {
        // neutron-star surface: bisect r on the dense polynomial
        const DenseC cr = dense_coef(hd, L.y[1], yn[1], L.k1[1], k3[1], k4[1], k5[1], k6[1], k7[1]);
        double lo = 0.0, hi = 1.0;
        for (int it = 0; it < 60; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (dense_eval(cr, mid) <= F.ns_R) hi = mid; else lo = mid;
        }
        const double s_end = 0.5 * (lo + hi);
        what = BH_HIT_STAR;
        #pragma unroll
        for (int i = 0; i < 6; ++i) {
            const DenseC c = dense_coef(hd, L.y[i], yn[i], L.k1[i], k3[i], k4[i], k5[i], k6[i], k7[i]);
            yh[i < 4 ? i : i + 1] = dense_eval(c, s_end);
        }
        yh[4] = L.pt;
        yh[7] = L.pph;
    } else if (rn <= F.r_stop) {
        what = BH_HIT_HORIZON;
    } else if (F.disc_enabled && (double)L.c0 * (double)ax7.cs < 0.0) {
        // equatorial crossing: bisect cos(theta) on the dense polynomial
        const DenseC cth = dense_coef(hd, L.y[2], yn[2], L.k1[2], k3[2], k4[2], k5[2], k6[2], k7[2]);
        const double c0 = (double)L.c0;
        double lo = 0.0, hi = 1.0;
        for (int it = 0; it < 60; ++it) {
            const double mid = 0.5 * (lo + hi);
            const double cm = cos(dense_eval(cth, mid));
            if (cm * c0 <= 0.0) hi = mid; else lo = mid;
        }
        const double s_end = 0.5 * (lo + hi);
        const DenseC crr = dense_coef(hd, L.y[1], yn[1], L.k1[1], k3[1], k4[1], k5[1], k6[1], k7[1]);
        const double rc = dense_eval(crr, s_end);
        if (rc >= F.r_in && rc <= F.r_out) {
            what = BH_HIT_DISC;
            #pragma unroll
            for (int i = 0; i < 6; ++i) {
                const DenseC c = dense_coef(hd, L.y[i], yn[i], L.k1[i], k3[i], k4[i], k5[i], k6[i], k7[i]);
                yh[i < 4 ? i : i + 1] = dense_eval(c, s_end);
            }
            yh[4] = L.pt;
            yh[7] = L.pph;
        }
    }
    if (what < 0 && F.sun_enabled) {
        // The Sun (render.cpp:201-241): probe the dense geodesic, then bisect.
        const double a = L.a;
        auto cart = [&](double r, double th, double ph, double q[3]) {
            const double rr = sqrt(r * r + a * a);
            const double sn = sin(th);
            q[0] = rr * sn * cos(ph);
            q[1] = rr * sn * sin(ph);
            q[2] = r * cos(th);
        };
        double p0[3], p1[3];
        cart((double)L.y[1], (double)L.y[2], (double)L.y[3], p0);
        cart(rn, (double)yn[2], (double)yn[3], p1);
        const double sg0 = p1[0] - p0[0], sg1 = p1[1] - p0[1], sg2 = p1[2] - p0[2];
        const double seg_len = sqrt(sg0 * sg0 + sg1 * sg1 + sg2 * sg2);
        const double dc = sqrt((p0[0] - F.sun_c[0]) * (p0[0] - F.sun_c[0]) +
                               (p0[1] - F.sun_c[1]) * (p0[1] - F.sun_c[1]) +
                               (p0[2] - F.sun_c[2]) * (p0[2] - F.sun_c[2]));
        if (dc <= seg_len + F.sun_R * 1.5) {
            const DenseC cr = dense_coef(hd, L.y[1], yn[1], L.k1[1], k3[1], k4[1], k5[1], k6[1], k7[1]);
            const DenseC ct = dense_coef(hd, L.y[2], yn[2], L.k1[2], k3[2], k4[2], k5[2], k6[2], k7[2]);
            const DenseC cp = dense_coef(hd, L.y[3], yn[3], L.k1[3], k3[3], k4[3], k5[3], k6[3], k7[3]);
            auto f = [&](double s) {
                double q[3];
                cart(dense_eval(cr, s), dense_eval(ct, s), dense_eval(cp, s), q);
                const double dx = q[0] - F.sun_c[0], dy = q[1] - F.sun_c[1], dz = q[2] - F.sun_c[2];
                return dx * dx + dy * dy + dz * dz - F.sun_R2;
            };
            double s_end = -1.0;
            bool inside0 = false;
            if (f(0.0) <= 0.0) {
                inside0 = true;
            } else {
                double prev_s = 0.0;
                for (int k = 1; k <= 12; ++k) {
                    const double s = (double)k / 12;
                    if (f(s) <= 0.0) {
                        double lo = prev_s, hi = s;
                        for (int b = 0; b < 50; ++b) {
                            const double mid = 0.5 * (lo + hi);
                            if (f(mid) <= 0.0) hi = mid; else lo = mid;
                        }
                        s_end = 0.5 * (lo + hi);
                        break;
                    }
                    prev_s = s;
                }
            }
            if (inside0) {
                // the start of the step is already inside: report that state
                what = BH_HIT_SUN;
                lane_state8(L, yh);
            } else if (s_end >= 0.0) {
                what = BH_HIT_SUN;
                #pragma unroll
                for (int i = 0; i < 6; ++i) {
                    const DenseC c = dense_coef(hd, L.y[i], yn[i], L.k1[i], k3[i], k4[i], k5[i], k6[i], k7[i]);
                    yh[i < 4 ? i : i + 1] = dense_eval(c, s_end);
                }
                yh[4] = L.pt;
                yh[7] = L.pph;
            }
        }
    }
    if (what < 0 && rn > F.r_escape) what = BH_HIT_SKY;

    // Advance (FSAL: k7 becomes the next k1).
    #pragma unroll
    for (int i = 0; i < 6; ++i) {
        L.y[i] = yn[i];
        L.k1[i] = k7[i];
    }
    L.err_prev = dmaxr(err, 1e-4);
    L.errp_pow = P::kMixed ? (double)__powf((float)L.err_prev, (float)kBeta) : pow(L.err_prev, kBeta);
    L.h = hd * fac;
    L.c0 = ax7.cs;

    if (what == BH_HIT_HORIZON || what == BH_HIT_SKY) {
        lane_state8(L, yh);
    } else if (what < 0 && L.steps >= F.max_steps) {
        what = BH_HIT_EXHAUSTED;
        lane_state8(L, yh);
    }
    if (what >= 0) {
        write_hit(A, L, what, yh);
        return true;
    }
    return false;
}

template <class P>
__global__ void trace_kernel(TraceArgs A) {
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    Lane<P> L;
    bool active = false, done = false;
    long long q_next = 0;
    int q_left = 0, q_stride = 0;
    while (true) {
        // Lanes with ids left in their own mini-queue start the next ray.
        while (!active && !done && q_left > 0) {
            if (q_next >= A.total_rays) { q_left = 0; done = true; break; }
            const long long id = q_next;
            q_next += q_stride;
            --q_left;
            active = start_ray<P>(A, L, id);
        }
        const unsigned want = __ballot_sync(kFull, !active && !done);
        if (want) {
            const unsigned live = __ballot_sync(kFull, active);
            const int n = __popc(want);
            if (n >= A.refill || live == 0) {
                const int leader = __ffs(want) - 1;
                unsigned long long base = 0;
                int stop = 0;
                if (lane == leader) {
                    stop = *(volatile int*)&A.queue->abort;
                    if (!stop) base = atomicAdd(&A.queue->next, (unsigned long long)n * A.rays_per_thread);
                }
                base = __shfl_sync(kFull, base, leader);
                stop = __shfl_sync(kFull, stop, leader);
                if (want & (1u << lane)) {
                    if (stop) {
                        done = true;
                    } else {
                        q_next = (long long)base + __popc(want & lt_mask);
                        q_stride = n;
                        q_left = A.rays_per_thread;
                        while (!active && q_left > 0) {
                            if (q_next >= A.total_rays) { q_left = 0; break; }
                            const long long id = q_next;
                            q_next += q_stride;
                            --q_left;
                            active = start_ray<P>(A, L, id);
                        }
                        if (!active && q_left == 0) done = true;
                    }
                }
            }
        }
        if (__ballot_sync(kFull, active) == 0) {
            if (__ballot_sync(kFull, !done) == 0) break;
            continue;
        }
        if (active) {
            if (attempt<P>(A, L)) {
                active = false;
                if (A.budget) atomicAdd(&A.queue->attempts, (unsigned long long)L.attempts);
            }
        }
        if (A.budget && lane == 0) {
            if (*(volatile unsigned long long*)&A.queue->attempts > A.budget &&
                *(volatile int*)&A.queue->abort == 0) {
                atomicCAS(&A.queue->abort, 0, 2);
            }
        }
    }
}

// ---- shading (FP64) ----------------------------------------------------------

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
};

__global__ void shade_kernel(ShadeArgs A) {
    const long long gp = (long long)blockIdx.x * blockDim.x + threadIdx.x;
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
    FrameStats* partials;
    FrameStats* out;
    int bpf;
};

__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

constexpr int kRedThreads = 256;

__global__ void __launch_bounds__(kRedThreads) reduce_partial_kernel(ReduceArgs A) {
    const int f = blockIdx.y;
    const FrameParams& F = A.frames[f];
    __shared__ unsigned long long s_cnt[kRedThreads][9];
    __shared__ double s_max[kRedThreads][2];
    __shared__ double s_flux[kRedThreads];
    unsigned long long c[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
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
    }
    const long long npx = (long long)F.width * F.height;
    for (long long i = (long long)blockIdx.x * kRedThreads + threadIdx.x; i < npx; i += stride)
        flux += A.pixel_lum[F.pixel_begin + i];
    for (int k = 0; k < 9; ++k) s_cnt[threadIdx.x][k] = c[k];
    s_max[threadIdx.x][0] = mn;
    s_max[threadIdx.x][1] = mq;
    s_flux[threadIdx.x] = flux;
    __syncthreads();
    for (int off = kRedThreads / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            for (int k = 0; k < 9; ++k) s_cnt[threadIdx.x][k] += s_cnt[threadIdx.x + off][k];
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
        o.max_norm_bits = dbits(s_max[0][0]);
        o.max_q_bits = dbits(s_max[0][1]);
        o.total_flux = s_flux[0];
    }
}

__global__ void reduce_final_kernel(ReduceArgs A) {
    const int f = blockIdx.x;
    if (threadIdx.x != 0) return;
    FrameStats t = {};
    double mn = 0.0, mq = 0.0;
    for (int b = 0; b < A.bpf; ++b) {
        const FrameStats& p = A.partials[(long long)f * A.bpf + b];
        t.rays += p.rays; t.steps += p.steps; t.attempts += p.attempts;
        t.captured += p.captured; t.disc_hits += p.disc_hits; t.sun_hits += p.sun_hits;
        t.star_hits += p.star_hits; t.escaped += p.escaped; t.exhausted += p.exhausted;
        mn = dmaxr(mn, __longlong_as_double((long long)p.max_norm_bits));
        mq = dmaxr(mq, __longlong_as_double((long long)p.max_q_bits));
        t.total_flux += p.total_flux;
    }
    t.max_norm_bits = dbits(mn);
    t.max_q_bits = dbits(mq);
    A.out[f] = t;
}

template <class P>
cudaError_t launch_trace_t(const TraceLaunch& L, cudaStream_t s) {
    TraceArgs A;
    A.frames = L.frames;
    A.frame_ray_end = L.frame_ray_end;
    A.nframes = L.nframes;
    A.total_rays = L.total_rays;
    A.hits = L.hits;
    A.queue = L.queue;
    A.rays_per_thread = L.rays_per_thread < 1 ? 1 : L.rays_per_thread;
    A.refill = L.refill < 1 ? 1 : (L.refill > 32 ? 32 : L.refill);
    A.budget = L.budget;
    trace_kernel<P><<<L.grid, L.block_size, 0, s>>>(A);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_trace(const TraceLaunch& L, cudaStream_t stream) {
    if (L.precision == BH_PRECISION_MIXED) return launch_trace_t<Mixed>(L, stream);
    return launch_trace_t<Fp64>(L, stream);
}

int trace_blocks_per_sm(int precision, int block_size) {
    int n = 0;
    if (precision == BH_PRECISION_MIXED)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, trace_kernel<Mixed>, block_size, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, trace_kernel<Fp64>, block_size, 0);
    return n;
}

int trace_registers(int precision) {
    cudaFuncAttributes at;
    if (precision == BH_PRECISION_MIXED)
        cudaFuncGetAttributes(&at, trace_kernel<Mixed>);
    else
        cudaFuncGetAttributes(&at, trace_kernel<Fp64>);
    return at.numRegs;
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
    const int bs = 128;
    const long long grid = (L.total_pixels + bs - 1) / bs;
    shade_kernel<<<(unsigned)grid, bs, 0, stream>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_reduce(const ReduceLaunch& L, cudaStream_t stream) {
    ReduceArgs A;
    A.frames = L.frames;
    A.nframes = L.nframes;
    A.hits = L.hits;
    A.pixel_lum = L.pixel_lum;
    A.partials = L.partials;
    A.out = L.out;
    A.bpf = L.blocks_per_frame;
    reduce_partial_kernel<<<dim3(L.blocks_per_frame, L.nframes), kRedThreads, 0, stream>>>(A);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    reduce_final_kernel<<<L.nframes, 32, 0, stream>>>(A);
    return cudaGetLastError();
}

}  // namespace bhg
