// bh_trace.cu - The persistent trace kernels of the render path (sm_100a).
//
//   trace_kernel<Fp64>   every operation in binary64.
//   trace_kernel<Mixed>  binary32 ray state, stages and right-hand side;
//                        binary64 for the step size, the error-norm sum and
//                        the accept/reject test, event root refinement and the
//                        invariant diagnostics.  A ray that is provably falling
//                        into the hole (moving inwards inside the innermost
//                        photon orbit) is handed to binary64 for the plunge,
//                        where Delta -> 0 makes the binary32 Hamiltonian lose
//                        all its digits: its state goes to a deferred list and
//                        trace_kernel<Fp64> resumes it in a second launch.
//
// Each lane integrates one ray: ray set-up (render.cpp:440-451,
// geodesic.h:215-231), DP5(4) attempts with PI step control
// (geodesic.h:123-204) under the hmax limiter (render.cpp:130-131), the
// invariant diagnostics (render.cpp:139-145) and the events (render.cpp:158-251).
// A warp refills lanes freed by terminated rays from a global atomic queue:
// one atomicAdd per refill, new ids compacted over the idle lanes with
// ballot/popc, so a refill hands out a contiguous (image-coherent) run of rays.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bh_gpu.h"
#include "bh_common.cuh"
#include "bh_dp5.cuh"
#include "bh_frame.h"
#include "bh_jet.cuh"
#include "bh_launch.h"

namespace bhg {

namespace {

// Binary32 rays closer to a pole than sin(th) = 0.01 go to binary64.
constexpr double kPoleSin2 = 1e-4;

// ---- precision policies -------------------------------------------------------
struct Fp64 {
    using R = double;
    static constexpr bool kMixed = false;
    __device__ static __forceinline__ void sc(double x, double* s, double* c) { sincos(x, s, c); }
    __device__ static __forceinline__ double rcp(double x) { return rcp_nr(x); }
    __device__ static __forceinline__ double powd(double x, double y) { return pow(x, y); }
};

constexpr float kLog2ErrFloor = -13.287712379549449f;   // log2 1e-4, the floor of err_prev

struct Mixed {
    using R = float;
    static constexpr bool kMixed = true;
    __device__ static __forceinline__ void sc(float x, float* s, float* c) { sincosf(x, s, c); }
    __device__ static __forceinline__ float rcp(float x) {
        float r;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
        return r;
    }
    __device__ static __forceinline__ double powd(double x, double y) {
        return (double)__powf((float)x, (float)y);
    }
    // base-2 logarithm and power of the special-function unit (__powf's parts)
    __device__ static __forceinline__ float lg2(float x) {
        float r;
        asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
        return r;
    }
    __device__ static __forceinline__ float ex2(float x) {
        float r;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
        return r;
    }
};

// Exact (non-contracted) binary64 arithmetic for the ray set-up, so that the
// initial photon reproduces the host (reference) computation bit for bit.
__device__ __forceinline__ double xm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xa(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xs(double a, double b) { return __dsub_rn(a, b); }

// Initial photon state of frame-local ray `local_id` (render.cpp:440-451,
// scene.h:356-384, geodesic.h:215-231) and its Carter constant
// (kerr.h:342-348, with the camera's sin^2/cos^2 precomputed on the host).
// Out of line: it runs once per ray, and inlined it would push the step loop
// apart in the instruction cache.
__device__ __noinline__ void ray_setup(const FrameParams& F, long long local_id, double y[8], double* Q0) {
    const int S = F.S;
    const long long pixel = local_id / (S * S);
    const int k = (int)(local_id - pixel * (S * S));
    const int sy = k / S, sx = k - (k / S) * S;
    int px, py;
    pixel_xy(F.width, F.height, pixel, &px, &py);
    // Rng(seed ^ y<<32 ^ x*phi64), draws 2k+1 and 2k+2 of its splitmix64 stream.
    const uint64_t s0 = F.seed ^ ((uint64_t)py << 32) ^ ((uint64_t)px * 0x9E3779B97F4A7C15ull);
    const uint64_t g = 0x9E3779B97F4A7C15ull;
    const double u1 = u53(mix64(s0 + (uint64_t)(2 * k + 1) * g));
    const double u2 = u53(mix64(s0 + (uint64_t)(2 * k + 2) * g));
    const double jx = xm(xa((double)sx, u1), F.inv_S);
    const double jy = xm(xa((double)sy, u2), F.inv_S);
    const double su = xs(__ddiv_rn(xm(2.0, xa((double)px, jx)), (double)F.width), 1.0);
    const double sv = xs(1.0, __ddiv_rn(xm(2.0, xa((double)py, jy)), (double)F.height));
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
    // p^mu = -(e_0 - d^i e_i) with the ZAMO legs, then lowered with g_{mu nu}.
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
    const double E = -y[4], Lz = y[7], pth = y[6];
    *Q0 = xa(xm(pth, pth), xm(F.cam_cs2, xa(xm(xm(F.a, F.a), xs(0.0, xm(E, E))),
                                              __ddiv_rn(xm(Lz, Lz), F.cam_sn2))));
}

// ---- lane state -------------------------------------------------------------
template <class P>
struct Lane {
    using R = typename P::R;
    R y[6];                  // t, r, th, phi, p_r, p_th
    R k1[6];                 // FSAL stage
    R E, Lz, aR, a2R, aE, aLz, a2E2, Lz2;
    R rp_hi, rp_lo, rm_hi, rm_lo;   // r_+ and r_- as exact two-term sums
    R c0;                    // cos(th) at y (disc-plane test, stage angles)
    R sn0;                   // sin(th) at y as the metric clamps it (stage angles)
    R h;
    R err_prev;              // PI-controller memory: the last accepted error norm
                             // (binary32 lanes: only at set-up and hand-over)
    R errp_mem;              // its factor in logarithms: beta log2 err_prev (binary32
                             // lanes), beta ln err_prev (binary64 lanes)
    R Q0;
    float inv_Q0, max_norm, max_q;
    float err_w;             // weight of the squared error norm (kTightErrWeight: tolerances / 4)
    int steps, tries, attempts;
    int att0;                // attempts already counted against the budget
    double jet;              // jet emission picked up so far (jet kernels only)
    int gid, frame;
    int mirror;              // mixed: the state holds pi - th and -p_th
    int factored;
    int bad_sc;
};

template <class P>
struct Aux {
    typename P::R sn, cs, sn2, cs2, D;
};


// ---- packed binary32 pairs ----------------------------------------------------
// sm_100's f32x2 arithmetic: one instruction does the same binary32 operation,
// rounded to nearest, on the two halves of a 64-bit register pair.  The stage
// sums of the mixed kernel run on the six components as three pairs, in the
// order and with the roundings of the scalar form (product, then fused
// multiply-adds, then the fused y + h * sum).  (Pairing the independent
// products of the right-hand side the same way was measured slower: 4.10
// against 3.98 ms on the 1024^2 edge-on frame, the pairs' register moves and
// spills outweighing the instructions saved.)
using u64 = unsigned long long;
__device__ __forceinline__ u64 pk2(float lo, float hi) {
    u64 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void up2(u64 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c) {
    u64 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ u64 mul2(u64 a, u64 b) {
    u64 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Hamilton's equations for H = 1/2 g^{mu nu} p_mu p_nu (geodesic.h:50-71),
// with the Kerr inverse metric in Carter's separated form
//   2 Sigma H = Delta p_r^2 + p_th^2 + (L_z - a E sin^2)^2 / sin^2
//               - ((r^2 + a^2) E - a L_z)^2 / Delta,
// E = -p_t and L_z = p_phi constant (their derivatives vanish exactly).  The
// same function of (r, th, p) as the reference's quotient-rule form, with one
// reciprocal (of Sigma Delta sin^2) instead of fifteen divisions.  H = 0 is
// not imposed (B is the full bracket).  Delta = (r - r_+)(r - r_-) with each
// factor formed against a two-term r_+-, so the factor that vanishes at the
// horizon is exact.  sn, cs: sin and cos of th.
template <class P>
__device__ __forceinline__ void rhs_sc(const Lane<P>& L, typename P::R r, typename P::R sn,
                                       typename P::R cs, typename P::R pr, typename P::R pth,
                                       typename P::R* d, Aux<P>* aux) {
    using R = typename P::R;
    if (fabs(sn) < R(1e-9)) sn = (sn < R(0)) ? R(-1e-9) : R(1e-9);   // kerr.h:51
    const R sn2 = sn * sn, cs2 = cs * cs;
    const R r2 = r * r;
    const R S = r2 + L.a2R * cs2;
    const R D = L.factored ? ((r - L.rp_hi) - L.rp_lo) * ((r - L.rm_hi) - L.rm_lo)
                           : (r2 - R(2) * r + L.a2R);
    const R SD = S * D;
    const R inv = P::rcp(SD * sn2);
    const R iS = inv * D * sn2, iD = inv * S * sn2, isn2 = inv * SD;
    const R r2a2 = r2 + L.a2R;
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
        aux->sn = sn;
        aux->cs = cs;
        aux->sn2 = sn2;
        aux->cs2 = cs2;
        aux->D = D;
    }
}

// The full sin/cos of an angle that angle addition from the step's base angle
// does not reach: a stage whose angle moved more than kMaxShift (and, in
// binary64, a ray's first angle or a step's end that moved that far).  Rare,
// so out of line: inlined in five stages it kept the step loop from staying
// in the instruction cache (-2% per frame in both precisions).
template <class P>
__device__ __noinline__ void stage_sincos_far(typename P::R th, typename P::R* sn, typename P::R* cs) {
    P::sc(th, sn, cs);
}

// The RHS at a fresh angle (full sincos).
template <class P>
__device__ __forceinline__ void rhs(const Lane<P>& L, typename P::R r, typename P::R th,
                                    typename P::R pr, typename P::R pth, typename P::R* d,
                                    Aux<P>* aux) {
    typename P::R sn, cs;
    P::sc(th, &sn, &cs);
    rhs_sc<P>(L, r, sn, cs, pr, pth, d, aux);
}

// The RHS at a stage angle th, from the sin/cos of the step's base angle
// L.y[2] by angle addition (full sincos when the stage moved th by more
// than kMaxShift).
template <class P>
__device__ __forceinline__ void rhs_stage(const Lane<P>& L, typename P::R r, typename P::R th,
                                          typename P::R pr, typename P::R pth, typename P::R* d) {
    using R = typename P::R;
    const R dth = th - L.y[2];
    R sn, cs;
    if (fabs(dth) <= R(kMaxShift)) shift_sincos(L.sn0, L.c0, dth, &sn, &cs);
    else stage_sincos_far<P>(th, &sn, &cs);
    rhs_sc<P>(L, r, sn, cs, pr, pth, d, nullptr);
}


// sum_s c[s] k_s[i] for the component pair (2j, 2j+1).
template <int N>
__device__ __forceinline__ u64 stage_sum_f2(int j, const float (&c)[N], const float* const (&k)[N]) {
    u64 m = mul2(pk2(c[0], c[0]), pk2(k[0][2 * j], k[0][2 * j + 1]));
    #pragma unroll
    for (int s = 1; s < N; ++s) m = fma2(pk2(c[s], c[s]), pk2(k[s][2 * j], k[s][2 * j + 1]), m);
    return m;
}
// out[i] = y[i] + h * sum_s c[s] k_s[i], i = 0..5.
template <int N>
__device__ __forceinline__ void stage_f2(const float* y, float h, const float (&c)[N],
                                         const float* const (&k)[N], float* out) {
    const u64 H = pk2(h, h);
    #pragma unroll
    for (int j = 0; j < 3; ++j)
        up2(fma2(H, stage_sum_f2<N>(j, c, k), pk2(y[2 * j], y[2 * j + 1])), out[2 * j], out[2 * j + 1]);
}
// out[i] = h * sum_s c[s] k_s[i], i = 0..5 (the embedded error estimate).
template <int N>
__device__ __forceinline__ void scaled_sum_f2(float h, const float (&c)[N], const float* const (&k)[N],
                                              float* out) {
    const u64 H = pk2(h, h);
    #pragma unroll
    for (int j = 0; j < 3; ++j) up2(mul2(H, stage_sum_f2<N>(j, c, k)), out[2 * j], out[2 * j + 1]);
}

// One accepted step's ends and stages (k1, k3..k7) for the dense output.
template <class R>
struct StepData {
    R y0[6], y1[6];
    R k[6][6];
};

// The state at fraction s of the step on the dense polynomial
// (geodesic.h:109-121), as the 8-component (t, r, th, phi, p_t, p_r, p_th,
// p_phi) vector.  Not inlined: it runs once per ray, and inlined into the step
// loop its code would take instruction-cache room from every step.
template <class R>
__device__ __noinline__ void dense_state_at(const StepData<R>* d, double h, double s, double pt, double pph,
                                            double yh[8]) {
    #pragma unroll
    for (int i = 0; i < 6; ++i) {
        const DenseC c = dense_coef(h, d->y0[i], d->y1[i], d->k[0][i], d->k[1][i], d->k[2][i], d->k[3][i],
                                    d->k[4][i], d->k[5][i]);
        yh[i < 4 ? i : i + 1] = dense_eval(c, s);
    }
    yh[4] = pt;
    yh[7] = pph;
}

// Deferred ray: a mixed-precision ray handed to the binary64 kernel.
struct Deferred {
    double y[6];
    double h;
    double Q0;
    float err_prev, max_norm, max_q;
    int gid, frame, steps, attempts;
    int tight;               // the ray runs at a quarter of the tolerances (kRayTight)
};
static_assert(sizeof(Deferred) == kDeferredRecordBytes, "kDeferredRecordBytes is stale");

struct TraceArgs {
    const FrameParams* frames;
    const long long* frame_ray_end;
    int nframes;
    long long total_rays;
    HitRecord* hits;
    QueueState* queue;
    Deferred* deferred;      // mixed: append target; resume: source
    int resume;              // 1: take rays from the deferred list
    int rays_per_thread;
    int refill;
    unsigned long long budget;
    double* jet;             // jet emission per ray (jet kernels only)
    double* xing;            // first two equatorial crossing radii per ray, or null
    int select;              // 0: every ray; 1: near-critical rays only; 2: all others
    const unsigned char* sel_flag;   // per ray: kRay* class from the classification pass, or null
    const int* sel_list;     // the near-critical rays' global ids, or null (then select 1 scans)
    long long list_cap;      // select 1 with a list: the rays [0, list_cap) beside the binary32
                             // kernel (phase 0), the rest [list_cap, ..) after it (phase 1)
    int phase;
    unsigned int* band_done; // finished rays per row band, or null
    long long rays_per_band;
};

template <class P>
__device__ __forceinline__ void state8(const Lane<P>& L, const double ptph[2], double y8[8]) {
    y8[0] = (double)L.y[0];
    y8[1] = (double)L.y[1];
    y8[2] = (double)L.y[2];
    y8[3] = (double)L.y[3];
    y8[4] = ptph[0];
    y8[5] = (double)L.y[4];
    y8[6] = (double)L.y[5];
    y8[7] = ptph[1];
}

template <class P, bool JET>
__device__ __forceinline__ void write_hit(const TraceArgs& A, const Lane<P>& L, int what, const double y8[8]) {
    if (JET) A.jet[L.gid] = L.jet;
    // y[4] = p_t and y[7] = p_phi were stored exactly when the ray started.
    HitRecord* o = &A.hits[L.gid];
    o->y[0] = y8[0];
    o->y[1] = y8[1];
    o->y[2] = y8[2];
    o->y[3] = y8[3];
    o->y[5] = y8[5];
    o->y[6] = y8[6];
    o->max_norm = (double)L.max_norm;
    o->max_q = (double)L.max_q;
    o->what = what;
    o->steps = L.steps;
    o->attempts = L.attempts;
    if (A.band_done) {
        // the record is visible device-wide before its band's count moves
        __threadfence();
        atomicAdd(&A.band_done[L.gid / A.rays_per_band], 1u);
    }
}

// pi in two binary32 parts: pi - th as (kPiHi - th) + kPiLo, the first
// difference exact for pi/2 <= th <= pi.
constexpr float kPiHi = 3.14159274f;
constexpr float kPiLo = -8.74227766e-8f;

// Reflect a binary32 lane through the equatorial plane: th -> pi - th,
// p_th -> -p_th (and the stage and the cosine that go with them).  Kerr
// geodesics map to Kerr geodesics under this reflection, and DP5 commutes
// with it, so integrating the mirror image and reflecting the result back
// gives the same ray; near the south pole the mirrored angle is small and
// resolved to binary32's relative precision.
template <class P>
__device__ __forceinline__ void mirror_lane(Lane<P>& L) {
    L.y[2] = (typename P::R)((kPiHi - (float)L.y[2]) + kPiLo);
    L.y[5] = -L.y[5];
    L.k1[2] = -L.k1[2];
    L.k1[5] = -L.k1[5];
    L.c0 = -L.c0;
    L.mirror ^= 1;
}

// Bounds on |R_min| / r*^4 (below): under kNearCritical a ray is traced in
// binary64; under kNearCriticalTight a binary32 ray runs at a quarter of the
// frame's tolerances (its error norm weighted by kTightErrWeight = 4^2).
constexpr double kNearCritical = 0.1;
constexpr double kNearCriticalTight = 0.2;
constexpr float kTightErrWeight = 16.f;
enum { kRayPlain = 0, kRayBinary64 = 1, kRayTight = 2 };

// Whether a photon from the camera passes close to the photon shell on its way
// out: its radial potential per E^2 (kerr.h carter form, b = L_z/E, q = Q/E^2)
//   R(r) = (r^2 + a^2 - a b)^2 - Delta (q + (b - a)^2)
//        = r^4 + (a^2 - b^2 - q) r^2 + 2 (q + (b - a)^2) r - a^2 q
// has its local minimum R_min at the largest root r* of R'; R_min < 0 is a
// turning point (the ray escapes), and the closer R_min is to 0 the more
// times the ray circles near r* and the more a small change of its state is
// amplified (about e^(2 pi) per orbit).  Such rays (ingoing from outside r*,
// -kNearCritical < R_min / r*^4 < 0) go to binary64: no binary32 state
// resolves their final direction.  The next band (down to -kNearCriticalTight)
// stays in binary32 at a quarter of the tolerances: measured on the CPU
// restatement over 120 random scenes (1.47 M rays, cameras beyond 100 M),
// the rays beyond 1e-4 rad against the binary64 path went from 30 to 0 for
// 0.6% more attempts, where sending the band to binary64 made the frame 50%
// slower.  Returns kRayPlain, kRayBinary64 or kRayTight.  Out of line and in
// explicitly rounded binary64, so that every kernel that calls it decides
// the same for a ray.
__device__ __noinline__ int near_critical(const FrameParams& F, const double y8[8], double Q0) {
    if (!F.fp64_near_critical) return kRayPlain;
    // The traced photon runs backwards in time (E = -p_t < 0 for the camera's
    // rays); b and q are the same for it as for the photon it reverses.
    const double E = -y8[4];
    if (!(E != 0.0) || !(y8[5] < 0.0)) return kRayPlain;      // ingoing photons only
    const double b = __ddiv_rn(y8[7], E);
    const double q = __ddiv_rn(Q0, __dmul_rn(E, E));
    const double bma = __dsub_rn(b, F.a);
    const double c2 = __dsub_rn(__dsub_rn(F.a2, __dmul_rn(b, b)), q);
    const double c1 = __dmul_rn(2.0, __dadd_rn(q, __dmul_rn(bma, bma)));
    const double c0 = -__dmul_rn(F.a2, q);
    if (!(c2 < 0.0)) return kRayPlain;                         // R' > 0 for r > 0: no minimum
    // Newton on R'(r) = 4 r^3 + 2 c2 r + c1 from sqrt(-c2), right of its
    // largest root (there 2 r (2 r^2 + c2) > 0 and c1 >= 0): monotone.
    double r = __dsqrt_rn(-c2);
    for (int it = 0; it < 60; ++it) {
        const double r2 = __dmul_rn(r, r);
        const double d1 = __dadd_rn(__dmul_rn(__dmul_rn(4.0, r2), r), __dadd_rn(__dmul_rn(__dmul_rn(2.0, c2), r), c1));
        const double d2 = __dadd_rn(__dmul_rn(12.0, r2), __dmul_rn(2.0, c2));
        if (!(d2 > 0.0)) return kRayPlain;
        const double step = __ddiv_rn(d1, d2);
        r = __dsub_rn(r, step);
        if (!(fabs(step) > 1e-13 * r)) break;
    }
    if (!(r > F.r_plus) || !(y8[1] > r)) return kRayPlain;
    const double r2 = __dmul_rn(r, r);
    const double R = __dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn(__dadd_rn(r2, c2), r), c1), r), c0);
    const double Rn = __ddiv_rn(R, __dmul_rn(r2, r2));
    if (!(Rn < 0.0)) return kRayPlain;
    return Rn > -kNearCritical ? kRayBinary64 : (Rn > -kNearCriticalTight ? kRayTight : kRayPlain);
}

// Lane set-up from an initial photon (fresh ray) or a deferred state.
template <class P, bool JET>
__device__ bool start_ray(const TraceArgs& A, Lane<P>& L, long long id) {
    using R = typename P::R;
    const Deferred* dr = nullptr;
    if (A.resume) {
        dr = &A.deferred[id];
        L.gid = dr->gid;
        L.frame = dr->frame;
    } else {
        L.gid = (A.select == 1 && A.sel_list) ? A.sel_list[id + (A.phase ? A.list_cap : 0)] : (int)id;
        // the binary32 kernel leaves the listed rays to the binary64 one
        if (A.select == 2 && A.sel_flag && A.sel_flag[L.gid] == kRayBinary64) return false;
        L.frame = find_frame(A.frame_ray_end, A.nframes, L.gid);
    }
    const FrameParams& F = A.frames[L.frame];
    double y8[8], Q0;
    ray_setup(F, (long long)L.gid - F.ray_begin, y8, &Q0);
    // Near-critical rays of a mixed-precision launch are traced by the
    // binary64 kernel that runs beside the binary32 one: each of the two
    // skips the other's rays (no hit record written here).
    int ray_class = kRayPlain;
    if (!dr && A.select) {
        ray_class = A.sel_flag ? (int)A.sel_flag[L.gid] : near_critical(F, y8, Q0);
        if (!A.sel_flag && (ray_class == kRayBinary64) != (A.select == 1)) return false;
    }
    L.err_w = dr ? (dr->tight ? kTightErrWeight : 1.f) : (ray_class == kRayTight ? kTightErrWeight : 1.f);
    const double E = -y8[4], Lz = y8[7];
    L.E = (R)E;
    L.Lz = (R)Lz;
    L.aR = (R)F.a;
    L.a2R = (R)F.a2;
    L.aE = (R)(F.a * E);
    L.aLz = (R)(F.a * Lz);
    L.a2E2 = (R)(F.a2 * E * E);
    L.Lz2 = (R)(Lz * Lz);
    L.rp_hi = (R)F.r_plus;
    L.rp_lo = (R)(F.r_plus - (double)L.rp_hi);
    L.rm_hi = (R)F.r_minus;
    L.rm_lo = (R)(F.r_minus - (double)L.rm_hi);
    L.factored = F.factored_delta;
    L.bad_sc = (F.atol + F.rtol * fabs(y8[4]) == 0.0) || (F.atol + F.rtol * fabs(y8[7]) == 0.0);
    L.tries = 0;
    if (JET) L.jet = A.resume ? A.jet[L.gid] : 0.0;
    // p_t and p_phi never change: store them now, the rest at termination.
    A.hits[L.gid].y[4] = y8[4];
    A.hits[L.gid].y[7] = y8[7];
    if (dr) {
        #pragma unroll
        for (int i = 0; i < 6; ++i) L.y[i] = (R)dr->y[i];
        L.h = dr->h;
        L.err_prev = (R)dr->err_prev;
        L.Q0 = dr->Q0;
        L.max_norm = dr->max_norm;
        L.max_q = dr->max_q;
        L.steps = dr->steps;
        L.attempts = dr->attempts;
        L.att0 = dr->attempts;
    } else {
        L.y[0] = (R)y8[0]; L.y[1] = (R)y8[1]; L.y[2] = (R)y8[2]; L.y[3] = (R)y8[3];
        L.y[4] = (R)y8[5]; L.y[5] = (R)y8[6];
        L.h = F.h0;
        L.err_prev = R(1e-4);
        if (P::kMixed) {
            // Carter constant of the binary32 initial state, the reference for
            // the drift of the binary32 integration.
            const double cs2 = F.cam_cs2, sn2 = F.cam_sn2;
            const double Ef = (double)L.E, Lf = (double)L.Lz, pf = (double)L.y[5];
            L.Q0 = pf * pf + cs2 * (F.a2 * (0.0 - Ef * Ef) + Lf * Lf / sn2);
        } else {
            L.Q0 = Q0;
        }
        L.max_norm = 0.f;
        L.max_q = 0.f;
        L.steps = 0;
        L.attempts = 0;
        L.att0 = 0;
    }
    if constexpr (P::kMixed) L.errp_mem = (float)kBeta * Mixed::lg2(fmaxf(L.err_prev, 1e-4f));
    else L.errp_mem = kBeta * log(dmaxr((double)L.err_prev, 1e-4));   // binary64: beta ln err_prev
    L.inv_Q0 = (float)(1.0 / (fabs(L.Q0) + 1e-12));
    L.mirror = 0;
    if (P::kMixed && F.mirror_ok && !dr && (double)L.y[2] > 0.5 * kPi) {
        // a camera below the equator: start in the mirror image (k1 and
        // cos(th) are evaluated there, below)
        L.y[2] = (R)((kPiHi - (float)L.y[2]) + kPiLo);
        L.y[5] = -L.y[5];
        L.mirror = 1;
    }
    if (!dr && F.max_steps <= 0) {
        write_hit<P, JET>(A, L, BH_HIT_EXHAUSTED, y8);
        return false;
    }
    // The first stage (FSAL: every later step starts from the last one's
    // stage 7) and the base angle's sin/cos, here rather than behind a branch
    // in the step loop (-2.3% per mixed frame, -1.4% per FP64 frame).
    Aux<P> ax;
    if constexpr (P::kMixed) {
        rhs<P>(L, L.y[1], L.y[2], L.y[4], L.y[5], L.k1, &ax);
    } else {
        double sn, cs;
        stage_sincos_far<P>(L.y[2], &sn, &cs);
        rhs_sc<P>(L, L.y[1], sn, cs, L.y[4], L.y[5], L.k1, &ax);
    }
    L.c0 = ax.cs;
    L.sn0 = ax.sn;
    return true;
}

// What a trace kernel is compiled with beyond the integration and the
// horizon, disc and escape events: nothing; the Sun's and the neutron star's
// surface tests and the record of equatorial crossings; the crossing record
// alone (the discrete adjoint's render).
enum { kSurfNone = 0, kSurfAll = 1, kSurfCrossings = 2 };
constexpr int kFamily = 4;   // trace kernels of a precision and register cap

// One step attempt.  Returns true when the lane's ray is finished here
// (terminated, or deferred to the binary64 kernel).  SURF (kSurf*): what the
// kernel is compiled with besides the horizon, disc and escape events;
// launches run the kernel with no more than they need (code taken by no lane
// still costs instruction-cache room and registers).
template <class P, bool JET, int SURF>
__device__ bool attempt(const TraceArgs& A, Lane<P>& L) {
    using R = typename P::R;
    const FrameParams& F = A.frames[L.frame];
    if (L.tries == 0) {
        if constexpr (P::kMixed) {
            const float hmax = fmaf(F.f_hmax_a, fmaxf(1.f, L.y[1] - F.f_r_h), F.f_hmax_b);
            if (L.h > hmax) L.h = hmax;
        } else {
            const double hmax = F.hmax_a * dmaxr(1.0, L.y[1] - F.r_h) + F.hmax_b;
            if (L.h > hmax) L.h = hmax;
        }
    }
    if (L.tries == 0 && F.land_escape && L.k1[1] > typename P::R(0) &&
        (float)L.y[1] + (float)L.h * (float)L.k1[1] > F.f_land_limit && (double)L.y[1] < F.r_escape) {
        // An escaping step lands within the reference's cap of r_escape: a
        // step predicted (to first order) to end beyond land_limit ends near
        // land_target instead, as it would under the reference's step cap.
        const double hl = (F.land_target - (double)L.y[1]) / (double)L.k1[1];
        if (hl > 0.0 && hl < (double)L.h) L.h = (R)hl;
    }
    const R h = (R)L.h;
    R t[6], k2[6], k3[6], k4[6], k5[6], k6[6], k7[6], yn[6];
    if constexpr (P::kMixed) {
        {
            const float c[1] = {float(A21)};
            const float* const k[1] = {L.k1};
            stage_f2<1>(L.y, h, c, k, t);
        }
        rhs_stage<P>(L, t[1], t[2], t[4], t[5], k2);
        {
            const float c[2] = {float(A31), float(A32)};
            const float* const k[2] = {L.k1, k2};
            stage_f2<2>(L.y, h, c, k, t);
        }
        rhs_stage<P>(L, t[1], t[2], t[4], t[5], k3);
        {
            const float c[3] = {float(A41), float(A42), float(A43)};
            const float* const k[3] = {L.k1, k2, k3};
            stage_f2<3>(L.y, h, c, k, t);
        }
        rhs_stage<P>(L, t[1], t[2], t[4], t[5], k4);
        {
            const float c[4] = {float(A51), float(A52), float(A53), float(A54)};
            const float* const k[4] = {L.k1, k2, k3, k4};
            stage_f2<4>(L.y, h, c, k, t);
        }
        rhs_stage<P>(L, t[1], t[2], t[4], t[5], k5);
        {
            const float c[5] = {float(A61), float(A62), float(A63), float(A64), float(A65)};
            const float* const k[5] = {L.k1, k2, k3, k4, k5};
            stage_f2<5>(L.y, h, c, k, t);
        }
        rhs_stage<P>(L, t[1], t[2], t[4], t[5], k6);
        {
            const float c[5] = {float(B1), float(B3), float(B4), float(B5), float(B6)};
            const float* const k[5] = {L.k1, k3, k4, k5, k6};
            stage_f2<5>(L.y, h, c, k, yn);
        }
    } else {
        #pragma unroll
        for (int i = 0; i < 6; ++i) t[i] = L.y[i] + h * R(A21) * L.k1[i];
        rhs_stage<P>(L, t[1], t[2], t[4], t[5], k2);
        #pragma unroll
        for (int i = 0; i < 6; ++i) t[i] = L.y[i] + h * (R(A31) * L.k1[i] + R(A32) * k2[i]);
        rhs_stage<P>(L, t[1], t[2], t[4], t[5], k3);
        #pragma unroll
        for (int i = 0; i < 6; ++i)
            t[i] = L.y[i] + h * (R(A41) * L.k1[i] + R(A42) * k2[i] + R(A43) * k3[i]);
        rhs_stage<P>(L, t[1], t[2], t[4], t[5], k4);
        #pragma unroll
        for (int i = 0; i < 6; ++i)
            t[i] = L.y[i] + h * (R(A51) * L.k1[i] + R(A52) * k2[i] + R(A53) * k3[i] + R(A54) * k4[i]);
        rhs_stage<P>(L, t[1], t[2], t[4], t[5], k5);
        #pragma unroll
        for (int i = 0; i < 6; ++i)
            t[i] = L.y[i] + h * (R(A61) * L.k1[i] + R(A62) * k2[i] + R(A63) * k3[i] +
                                 R(A64) * k4[i] + R(A65) * k5[i]);
        rhs_stage<P>(L, t[1], t[2], t[4], t[5], k6);
        #pragma unroll
        for (int i = 0; i < 6; ++i)
            yn[i] = L.y[i] + h * (R(B1) * L.k1[i] + R(B3) * k3[i] + R(B4) * k4[i] + R(B5) * k5[i] +
                                  R(B6) * k6[i]);
    }
    // The last stage is the next step's first (FSAL) and its angle the next
    // base angle.  binary32: full sincos, so angle-addition errors never
    // chain.  binary64: by angle addition from the step's base angle like the
    // stages (a chain of ulp-sized roundings, ~1e-15 after a thousand steps),
    // which keeps the full sin/cos out of the step loop (-1.7% per frame).
    Aux<P> ax7;
    if constexpr (P::kMixed) {
        rhs<P>(L, yn[1], yn[2], yn[4], yn[5], k7, &ax7);
    } else {
        const double dth = yn[2] - L.y[2];
        double sn, cs;
        if (fabs(dth) <= kMaxShift) shift_sincos(L.sn0, L.c0, dth, &sn, &cs);
        else stage_sincos_far<P>(yn[2], &sn, &cs);
        rhs_sc<P>(L, yn[1], sn, cs, yn[4], yn[5], k7, &ax7);
    }

    // RMS error over the eight components (geodesic.h:157-166): the p_t and
    // p_phi terms are exactly zero.  binary64: squares summed in binary64;
    // mixed: the scaled errors, the norm, the accept/reject test and the step
    // control in binary32 (a binary64 step control converted between the
    // formats about twenty times per attempt: 3.38 against 3.16 ms per 1024^2
    // frame).
    double err2 = 0.0;
    float err2f = 0.f;
    R ev[6];
    if constexpr (P::kMixed) {
        const float c[6] = {float(E1), float(E3), float(E4), float(E5), float(E6), float(E7)};
        const float* const k[6] = {L.k1, k3, k4, k5, k6, k7};
        scaled_sum_f2<6>(h, c, k, ev);
    }
    #pragma unroll
    for (int i = 0; i < 6; ++i) {
        const R e = P::kMixed ? ev[i]
                              : h * (R(E1) * L.k1[i] + R(E3) * k3[i] + R(E4) * k4[i] + R(E5) * k5[i] +
                                     R(E6) * k6[i] + R(E7) * k7[i]);
        if (P::kMixed) {
            // the scale of the true angle where the lane holds its mirror;
            // the azimuth's scale is atol + rtol, whatever its value: an
            // angle's error does not grow with the distance from phi = 0
            // (under the reference's |phi| scale a camera at phi = 0 takes
            // more steps than the same scene turned about the axis)
            const float y0 = (i == 2 && L.mirror) ? kPiHi - (float)L.y[i] : (float)L.y[i];
            const float y1 = (i == 2 && L.mirror) ? kPiHi - (float)yn[i] : (float)yn[i];
            const float sc = (i == 3) ? F.f_atol + F.f_rtol : F.f_atol + F.f_rtol * fmaxf(fabsf(y0), fabsf(y1));
            const float q = (float)e * Mixed::rcp(sc);
            err2f += q * q;
        } else {
            const double sc = F.atol + F.rtol * dmaxr(fabs((double)L.y[i]), fabs((double)yn[i]));
            const double q = (double)e * rcp_nr(sc);
            err2 += q * q;
        }
    }
    // err holds the square of the RMS norm sqrt(err2 / 8): the accept test
    // err^2 <= 1 and the controller's powers of err^2 need no square root.
    // The step control runs in the lane's precision.
    R err;
    if constexpr (P::kMixed) {
        err = err2f * L.err_w * 0.125f;
    } else {
        if (L.err_w != 1.f) err2 *= (double)L.err_w;
        err = err2 * 0.125;
    }
    if (L.bad_sc || !isfinite(err)) err = R(1e10);
    if (P::kMixed && L.Lz != R(0) && (ax7.sn < R(0)) != (L.sn0 < R(0))) {
        // A ray with L_z != 0 never reaches the axis (Theta(th) < 0 near it:
        // it turns at th_min ~ |L_z| / sqrt(Q + a^2 E^2)).  A binary32 step
        // that ends across the axis has jumped over that turn, where the
        // L_z^2 / sin^3 force changes over th_min / p_th of affine parameter
        // and atol alone bounds the error in th: rejected, so the steps
        // shrink until they resolve the turn.
        err = R(1e10);
    }
    ++L.attempts;
    // The PI step factor 0.9 err^-alpha err_prev^beta (geodesic.h:171-173)
    // as one power of beta log err_prev - alpha log err, the logarithm of
    // this attempt's norm kept for the next step (no root of the squared
    // norm, no second power): binary32 lanes in base 2 on the special-
    // function unit (2.2% per frame against two powers and a root), binary64
    // lanes in base e (binary64 pow is a long extended-precision sequence,
    // and the factor only sets the next step's size).
    R fac, lq = R(0);
    if constexpr (P::kMixed) {
        lq = Mixed::lg2(fmaxf(err, 1e-32f));
        fac = 0.9f * Mixed::ex2(fmaf((float)(-0.5 * kAlpha), lq, L.errp_mem));
    } else {
        lq = log(dmaxr(err, 1e-32));
        fac = 0.9 * exp(fma(-0.5 * kAlpha, lq, L.errp_mem));
    }
    fac = (fac < R(0.2)) ? R(0.2) : (R(5) < fac) ? R(5) : fac;   // std::clamp(fac, 0.2, 5)

    if (!(err <= R(1))) {
        L.h *= (R(1) < fac) ? R(1) : fac;
        if (++L.tries > 40 || fabs(L.h) < R(1e-14)) {
            // render.cpp:133-136: no acceptable step is a capture, reported
            // with the ray's initial state.
            double y8[8], Q0;
            ray_setup(F, (long long)L.gid - F.ray_begin, y8, &Q0);
            write_hit<P, JET>(A, L, BH_HIT_HORIZON, y8);
            return true;
        }
        return false;
    }

    // ---- accepted -----------------------------------------------------------
    L.tries = 0;
    ++L.steps;
    const double rn = (double)yn[1];
    const double pt = -(double)L.E, pph = (double)L.Lz;
    const double hd = L.h;
    // the mixed kernel's stop radii in binary32 (the binary64 one reads F's)
    float r_stop_f = 0.f, r_escape_f = 0.f, r_promote_f = 0.f;
    if constexpr (P::kMixed) {
        r_stop_f = F.f_r_stop;
        r_escape_f = F.f_r_escape;
        r_promote_f = F.f_r_promote;
    }
    const double ptph[2] = {pt, pph};
    int what = -1;
    double yh[8];
    auto dense_state = [&](double s_end) {
        // Out of line (taken once per ray, at its event): the step's data go
        // through a stack copy, so the stage arrays stay in registers.
        StepData<R> d;
        #pragma unroll
        for (int i = 0; i < 6; ++i) {
            d.y0[i] = L.y[i];
            d.y1[i] = yn[i];
            d.k[0][i] = L.k1[i];
            d.k[1][i] = k3[i];
            d.k[2][i] = k4[i];
            d.k[3][i] = k5[i];
            d.k[4][i] = k6[i];
            d.k[5][i] = k7[i];
        }
        dense_state_at<R>(&d, hd, s_end, pt, pph, yh);
    };
    // Fraction of the step the jet integral covers: up to an occluding
    // event, all of it otherwise; < 0: none (render.cpp:107-122, 165-244).
    double s_jet = 1.0;
    if (SURF == kSurfAll && F.ns_enabled && rn <= F.ns_R) {
        // neutron-star surface (render.cpp:158-169)
        const DenseC cr = dense_coef(hd, L.y[1], yn[1], L.k1[1], k3[1], k4[1], k5[1], k6[1], k7[1]);
        what = BH_HIT_STAR;
        s_jet = dense_crossing(cr, F.ns_R);
        dense_state(s_jet);
    } else if (P::kMixed ? yn[1] <= r_stop_f : rn <= F.r_stop) {
        what = BH_HIT_HORIZON;             // render.cpp:172-177
    } else if (F.disc_enabled && (P::kMixed ? ((L.c0 < R(0)) && (ax7.cs > R(0))) || ((L.c0 > R(0)) && (ax7.cs < R(0)))
                                            : (double)L.c0 * (double)ax7.cs < 0.0)) {
        // equatorial crossing (render.cpp:180-199): cos(th) changes sign at
        // th* = pi/2 + m pi between th(0) and th(1)
        const DenseC cth = dense_coef(hd, L.y[2], yn[2], L.k1[2], k3[2], k4[2], k5[2], k6[2], k7[2]);
        const double th0 = cth.r1, th1 = cth.r1 + cth.r2;
        const double m = (th1 > th0) ? ceil((th0 - 0.5 * kPi) / kPi) : floor((th0 - 0.5 * kPi) / kPi);
        const double s_end = dense_crossing(cth, 0.5 * kPi + m * kPi);
        const DenseC crr = dense_coef(hd, L.y[1], yn[1], L.k1[1], k3[1], k4[1], k5[1], k6[1], k7[1]);
        const double rc = dense_eval(crr, s_end);
        if (SURF && A.xing) {
            // the crossings the discrete adjoint's edge pass starts from
            double* x = A.xing + 2 * L.gid;
            if (x[0] == 0.0) x[0] = rc;
            else if (x[1] == 0.0) x[1] = rc;
        }
        if (rc >= F.r_in && rc <= F.r_out) {
            what = BH_HIT_DISC;
            s_jet = s_end;
            dense_state(s_end);
        }
    }
    if (SURF == kSurfAll && what < 0 && F.sun_enabled) {
        // The Sun (render.cpp:201-241): probe the dense geodesic, then bisect.
        const double a = F.a;
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
            if (f(0.0) <= 0.0) {
                what = BH_HIT_SUN;
                s_jet = -1.0;
                state8(L, ptph, yh);       // already inside at the start of the step
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
                        what = BH_HIT_SUN;
                        s_jet = 0.5 * (lo + hi);
                        dense_state(s_jet);
                        break;
                    }
                    prev_s = s;
                }
            }
        }
    }
    if (JET && s_jet > 0.0) {
        // Optically thin jet emission along the step (render.cpp:150-152,
        // 107-122): skipped unless the chord passes within r_bound of the hole.
        double q0[3], q1[3];
        bl_cartesian(F.a, (double)L.y[1], (double)L.y[2], (double)L.y[3], q0);
        bl_cartesian(F.a, rn, (double)yn[2], (double)yn[3], q1);
        if (segment_distance_to_origin(q0, q1) < F.jet_r_bound) {
            const DenseC cr = dense_coef(hd, L.y[1], yn[1], L.k1[1], k3[1], k4[1], k5[1], k6[1], k7[1]);
            const DenseC ct = dense_coef(hd, L.y[2], yn[2], L.k1[2], k3[2], k4[2], k5[2], k6[2], k7[2]);
            const DenseC cpr = dense_coef(hd, L.y[4], yn[4], L.k1[4], k3[4], k4[4], k5[4], k6[4], k7[4]);
            const DenseC cpt = dense_coef(hd, L.y[5], yn[5], L.k1[5], k3[5], k4[5], k5[5], k6[5], k7[5]);
            L.jet += jet_step_integral(F, cr, ct, cpr, cpt, (double)L.E, (double)L.Lz, hd, s_jet);
        }
    }
    if (what < 0 && (P::kMixed ? yn[1] > r_escape_f : rn > F.r_escape)) what = BH_HIT_SKY;   // render.cpp:247-251

    // Advance; FSAL: k7 becomes the next k1.
    #pragma unroll
    for (int i = 0; i < 6; ++i) {
        L.y[i] = yn[i];
        L.k1[i] = k7[i];
    }
    if constexpr (P::kMixed) {
        L.errp_mem = (float)kBeta * fmaxf(0.5f * lq, kLog2ErrFloor);   // err_prev >= 1e-4
    } else {
        L.errp_mem = kBeta * dmaxr(0.5 * lq, kLnErrFloor);   // err_prev >= 1e-4
    }
    L.h = P::kMixed ? L.h * fac : (R)(hd * fac);
    L.c0 = ax7.cs;
    L.sn0 = ax7.sn;

    // Invariant diagnostics at the new state (render.cpp:139-145), after
    // the events so the stage values are no longer live.  The five terms of
    // g^{ab} p_a p_b (kerr.h:301-321) are all scaled by Sigma Delta sin^2 > 0
    // and Carter's Q by sin^2, which leaves both ratios unchanged; a division
    // only when a maximum grows.  Binary64 frames evaluate them in binary64;
    // mixed ones in binary32, from the binary32 state they measure: each term
    // to a few ulp, so the reported ratios carry up to about 1e-6 of their
    // own rounding.
    if constexpr (P::kMixed) {
        const float sn2 = ax7.sn2, cs2 = ax7.cs2, Del = ax7.D;
        const float rf = yn[1], pr = L.y[4], pth = L.y[5];
        const float a2 = L.a2R;
        const float pt2 = L.E * L.E, pph2 = L.Lz2, pth2 = pth * pth;
        const float Ds = Del * sn2, Dpr = Del * pr;
        const float rpa = fmaf(rf, rf, a2);
        const float T1 = fmaf(a2, Ds, -(rpa * rpa)) * (pt2 * sn2);
        const float T2 = (4.f * L.aE * L.Lz) * (rf * sn2);
        const float T3 = (Ds * pr) * Dpr;
        const float T4 = Ds * pth2;
        const float T5 = fmaf(-a2, sn2, Del) * pph2;
        const float nrm = fabsf(T1 + T2 + T3 + T4 + T5);
        const float scl = fabsf(T1) + fabsf(T2) + fabsf(T3) + fabsf(T4) + fabsf(T5);
        if (nrm > L.max_norm * scl) L.max_norm = (scl > 0.f) ? nrm / scl : nrm;
        const float Qs = fmaf(pth2, sn2, cs2 * fmaf(-L.a2E2, sn2, pph2));
        const float dev = fabsf(fmaf(-L.Q0, sn2, Qs)) * L.inv_Q0;
        if (dev > L.max_q * sn2) L.max_q = dev / sn2;
    } else {
        const double sn2 = (double)ax7.sn2, cs2 = (double)ax7.cs2, Del = (double)ax7.D;
        const double pr = (double)L.y[4], pth = (double)L.y[5];
        const double a2 = F.a2;
        const double pt2 = pt * pt, pph2 = pph * pph, pth2 = pth * pth;
        const double Ds = Del * sn2, Dpr = Del * pr;
        const double rpa = rn * rn + a2;
        const double T1 = (a2 * Ds - rpa * rpa) * (pt2 * sn2);
        const double T2 = (-4.0 * F.a * pt * pph) * (rn * sn2);
        const double T3 = (Ds * pr) * Dpr;
        const double T4 = Ds * pth2;
        const double T5 = (Del - a2 * sn2) * pph2;
        const double nrm = fabs(T1 + T2 + T3 + T4 + T5);
        const double scl = fabs(T1) + fabs(T2) + fabs(T3) + fabs(T4) + fabs(T5);
        if (nrm > (double)L.max_norm * scl) L.max_norm = (float)((scl > 0.0) ? nrm / scl : nrm);
        const double Qs = pth2 * sn2 + cs2 * (pph2 - a2 * pt2 * sn2);
        const double dev = fabs(Qs - L.Q0 * sn2) * (double)L.inv_Q0;
        if (dev > (double)L.max_q * sn2) L.max_q = (float)(dev / sn2);
    }

    if (what == BH_HIT_HORIZON || what == BH_HIT_SKY) {
        state8(L, ptph, yh);
    } else if (what < 0 && L.steps >= F.max_steps) {
        what = BH_HIT_EXHAUSTED;
        state8(L, ptph, yh);
    }
    if (what < 0 && F.early_capture && (P::kMixed ? yn[1] < r_promote_f : rn < F.r_promote) && k7[1] < R(0)) {
        // Moving inwards inside the innermost photon orbit: no radial turning
        // point is left, the ray falls into the hole, and nothing lies on
        // its way (no neutron star, no jet; the disc is outside the ISCO).
        // Mixed-precision frames only (early_capture is 0 for binary64 ones):
        // here, or in the binary64 pass over the rays handed over near a pole.
        what = BH_HIT_HORIZON;
        state8(L, ptph, yh);
    }
    if (what >= 0) {
        if (P::kMixed && L.mirror) {          // back to the true angle
            yh[2] = kPi - yh[2];
            yh[6] = -yh[6];
        }
        write_hit<P, JET>(A, L, what, yh);
        return true;
    }
    if (P::kMixed && A.deferred &&
        (((P::kMixed ? yn[1] < r_promote_f : rn < F.r_promote) && k7[1] < R(0)) ||
         (!F.mirror_ok && ax7.sn2 < R(kPoleSin2)))) {
        // Two places where binary32 state cannot carry the geodesic, handed
        // to the binary64 kernel for the rest of the ray:
        //  - moving inwards inside the innermost photon orbit: the ray is
        //    falling in, and Delta -> 0 cancels every digit of the
        //    Hamiltonian's radial terms;
        //  - within 0.01 of a pole: sin(th) carries the L_z^2 / sin^4 term,
        //    and th = pi - 1e-5 is only resolved to 2.4e-7 in binary32 (not
        //    where the lane integrates the mirror image: the angle from the
        //    nearer pole is then small and resolved).
        const unsigned long long slot = atomicAdd(&A.queue->deferred, 1ull);
        Deferred* dd = &A.deferred[slot];
        #pragma unroll
        for (int i = 0; i < 6; ++i) dd->y[i] = (double)L.y[i];
        if (L.mirror) {
            dd->y[2] = kPi - dd->y[2];
            dd->y[5] = -dd->y[5];
        }
        dd->h = L.h;
        dd->Q0 = L.Q0;
        dd->err_prev = exp2f(L.errp_mem / (float)kBeta);
        dd->max_norm = L.max_norm;
        dd->max_q = L.max_q;
        dd->gid = L.gid;
        dd->frame = L.frame;
        dd->steps = L.steps;
        dd->attempts = L.attempts;
        dd->tight = L.err_w != 1.f;
        if (JET) A.jet[L.gid] = L.jet;   // the binary64 pass continues the sum
        return true;
    }
    // Crossed the equatorial plane in the integrated frame: continue in the
    // other one, so the lane's angle stays within pi/2 of the nearer pole.
    if (P::kMixed && F.mirror_ok && L.c0 < R(0)) mirror_lane(L);
    return false;
}

template <class P, int MAXREG, bool JET, int SURF>
__global__ void __maxnreg__(MAXREG) trace_kernel(TraceArgs A) {
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    long long total = A.resume ? (long long)*(volatile unsigned long long*)&A.queue->deferred : A.total_rays;
    unsigned long long* counter = A.resume ? &A.queue->resume_next
                                           : (A.select == 1 ? &A.queue->select_next : &A.queue->next);
    if (!A.resume && A.select == 1 && A.sel_list) {
        const long long listed = (long long)*(volatile unsigned long long*)&A.queue->selected;
        if (A.phase == 0) {
            total = listed < A.list_cap ? listed : A.list_cap;
        } else {
            total = listed > A.list_cap ? listed - A.list_cap : 0;
            counter = &A.queue->select_next2;
        }
    }
    Lane<P> L;
    bool active = false, done = false;
    long long q_next = 0;
    int q_left = 0, q_stride = 0;
    while (true) {
        const unsigned want = __ballot_sync(kFull, !active && !done && q_left == 0);
        if (want) {
            const unsigned live = __ballot_sync(kFull, active);
            const int n = __popc(want);
            if (n >= A.refill || live == 0) {
                const int leader = __ffs(want) - 1;
                unsigned long long base = 0;
                int stop = 0;
                if (lane == leader) {
                    stop = *(volatile int*)&A.queue->abort;
                    if (!stop) base = atomicAdd(counter, (unsigned long long)n * A.rays_per_thread);
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
                    }
                }
            }
        }
        // A lane with ids left in its mini-queue (just refilled or not) starts
        // the next ray; one call site keeps one copy of start_ray in the loop
        // (two inlined copies cost 60 against 16 bytes of spills per binary32
        // lane and 2.3% per frame).
        // A lane is done only when the ids run out: start_ray also returns
        // false for a ray it leaves to another kernel or ends at once, and the
        // lane then refills.
        while (!active && !done && q_left > 0) {
            if (q_next >= total) { q_left = 0; done = true; break; }
            const long long id = q_next;
            q_next += q_stride;
            --q_left;
            active = start_ray<P, JET>(A, L, id);
        }
        if (__ballot_sync(kFull, active) == 0) {
            if (__ballot_sync(kFull, !done) == 0) break;
            continue;
        }
        if (active) {
            if (attempt<P, JET, SURF>(A, L)) {
                active = false;
                if (A.budget) atomicAdd(&A.queue->attempts, (unsigned long long)(L.attempts - L.att0));
            }
        }
        if (A.budget && lane == 0) {
            if (*(volatile unsigned long long*)&A.queue->attempts > A.budget &&
                *(volatile int*)&A.queue->abort == 0)
                atomicCAS(&A.queue->abort, 0, 2);
        }
    }
}

// Register caps (the launch parameter reg_variant picks one): binary32 lanes
// in 128 registers (16 warps per SM) or 168; binary64 lanes in 168 (12 warps
// per SM) or 232 (8 warps, no spills).
constexpr int kRegMixed = 128;
constexpr int kRegMixedWide = 168;
constexpr int kRegFp64 = 168;
constexpr int kRegFp64Wide = 232;

// The right-hand side the trace kernels integrate, evaluated at given
// states (known-answer tests of the device arithmetic): in = 8 doubles per
// state (t, r, th, phi, p_t, p_r, p_th, p_phi), out = their derivatives
// with respect to the affine parameter (dp_t = dp_phi = 0), with the lane
// constants set up as start_ray sets them.
template <class P>
__global__ void eval_rhs_kernel(const FrameParams* __restrict__ Fp, const double* __restrict__ in, long long n,
                                double* __restrict__ out) {
    using R = typename P::R;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const FrameParams& F = *Fp;
    const double* y = in + 8 * i;
    const double E = -y[4], Lz = y[7];
    Lane<P> L;
    L.E = (R)E;
    L.Lz = (R)Lz;
    L.aR = (R)F.a;
    L.a2R = (R)F.a2;
    L.aE = (R)(F.a * E);
    L.aLz = (R)(F.a * Lz);
    L.a2E2 = (R)(F.a2 * E * E);
    L.Lz2 = (R)(Lz * Lz);
    L.rp_hi = (R)F.r_plus;
    L.rp_lo = (R)(F.r_plus - (double)L.rp_hi);
    L.rm_hi = (R)F.r_minus;
    L.rm_lo = (R)(F.r_minus - (double)L.rm_hi);
    L.factored = F.factored_delta;
    R d[6];
    rhs<P>(L, (R)y[1], (R)y[2], (R)y[5], (R)y[6], d, nullptr);
    double* o = out + 8 * i;
    o[0] = (double)d[0];
    o[1] = (double)d[1];
    o[2] = (double)d[2];
    o[3] = (double)d[3];
    o[4] = 0.0;
    o[5] = (double)d[4];
    o[6] = (double)d[5];
    o[7] = 0.0;
}

template <class P, int MAXREG, bool JET, int SURF>
cudaError_t launch_t(const TraceLaunch& L, int resume, int grid, int block, cudaStream_t s, int select = 0,
                     int phase = 0) {
    TraceArgs A;
    A.frames = (select == 1) ? L.frames_side : L.frames;
    A.sel_flag = select ? L.sel_flag : nullptr;
    A.sel_list = (select == 1) ? L.sel_list : nullptr;
    A.list_cap = (long long)L.grid_side * 128;
    A.phase = phase;
    A.frame_ray_end = L.frame_ray_end;
    A.nframes = L.nframes;
    A.total_rays = L.total_rays;
    A.hits = L.hits;
    A.queue = L.queue;
    A.deferred = static_cast<Deferred*>(L.deferred);
    A.resume = resume;
    A.rays_per_thread = L.rays_per_thread < 1 ? 1 : L.rays_per_thread;
    A.refill = L.refill < 1 ? 1 : (L.refill > 32 ? 32 : L.refill);
    A.select = select;
    if (select == 1) {
        // few rays found among many looked at: refill a lane as soon as it
        // is idle, one id at a time, so a lane tracing a ray does not hold
        // up the search of the other 31
        A.rays_per_thread = 1;
        A.refill = 1;
    }
    A.budget = L.budget;
    A.jet = L.jet;
    A.xing = L.xing;
    A.band_done = L.band_done;
    A.rays_per_band = L.rays_per_band > 0 ? L.rays_per_band : 1;
    trace_kernel<P, MAXREG, JET, SURF><<<grid, block, 0, s>>>(A);
    return cudaGetLastError();
}

// Raises each band counter to its band's ray count (after the trace kernels).
__global__ void band_release_kernel(unsigned int* band_done, int nbands, long long total, long long per_band) {
    for (int b = threadIdx.x; b < nbands; b += blockDim.x) {
        const long long lo = (long long)b * per_band;
        const long long n = (total - lo < per_band) ? total - lo : per_band;
        atomicMax(&band_done[b], (unsigned int)(n > 0 ? n : 0));
    }
}

// The near-critical test of every ray's initial photon (grid-stride, one
// thread per ray): flag[id] = 1 and the id appended to `list` for the rays
// the binary64 kernel beside the binary32 one traces.
__global__ void classify_kernel(const FrameParams* __restrict__ frames, const long long* __restrict__ frame_ray_end,
                                int nframes, long long total, QueueState* queue, unsigned char* __restrict__ flag,
                                int* __restrict__ list) {
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const FrameParams& F = frames[find_frame(frame_ray_end, nframes, id)];
        double y8[8], Q0;
        ray_setup(F, id - F.ray_begin, y8, &Q0);
        const int cls = near_critical(F, y8, Q0);
        flag[id] = (unsigned char)cls;
        if (cls == kRayBinary64) list[atomicAdd(&queue->selected, 1ull)] = (int)id;
    }
}

// The kernels of a precision and register cap: plain, with the surface tests
// and the crossing record, with those and the jet's emission, with the
// crossing record alone.
template <class P, int MAXREG>
void family(const void* k[kFamily]) {
    k[0] = (const void*)trace_kernel<P, MAXREG, false, kSurfNone>;
    k[1] = (const void*)trace_kernel<P, MAXREG, false, kSurfAll>;
    k[2] = (const void*)trace_kernel<P, MAXREG, true, kSurfAll>;
    k[3] = (const void*)trace_kernel<P, MAXREG, false, kSurfCrossings>;
}

void kernels_of(int precision, int variant, const void* k[kFamily]) {
    if (precision == BH_PRECISION_MIXED) {
        if (variant) family<Mixed, kRegMixedWide>(k);
        else family<Mixed, kRegMixed>(k);
    } else {
        if (variant) family<Fp64, kRegFp64Wide>(k);
        else family<Fp64, kRegFp64>(k);
    }
}

// The kernels of launches with a jet accumulate its emission per ray, those
// of launches with the Sun or a neutron star test for the surfaces and record
// the crossings, those of the adjoint's render record the crossings alone
// (without the surface tests' code: 1.3% per gradient); the others are
// compiled without that code.
template <bool JET, int SURF>
cudaError_t launch_fp64(const TraceLaunch& L, int resume, int grid, int block, int variant, cudaStream_t s) {
    return variant ? launch_t<Fp64, kRegFp64Wide, JET, SURF>(L, resume, grid, block, s)
                   : launch_t<Fp64, kRegFp64, JET, SURF>(L, resume, grid, block, s);
}

template <bool JET, int SURF>
cudaError_t launch_trace_t(const TraceLaunch& L, cudaStream_t stream) {
    if (L.precision == BH_PRECISION_MIXED) {
        cudaError_t e;
        const bool side = L.near_critical && L.side_stream && L.fork_event && L.join_event;
        if (L.near_critical) {
            // The near-critical rays in binary64 (the kernel of the binary64
            // path's default cap, blocks of 128: the same arithmetic as a
            // binary64 frame) beside the binary32 launch (the two
            // share no data but the queue's separate counters and never wait
            // on each other), or before it on the same stream.  With a flag
            // array, a classification pass lists them first.
            if (L.sel_flag) {
                const long long want = (L.total_rays + 255) / 256;
                const int cgrid = (int)(want < 4LL * L.grid ? want : 4LL * L.grid);
                classify_kernel<<<cgrid > 0 ? cgrid : 1, 256, 0, stream>>>(L.frames, L.frame_ray_end, L.nframes,
                                                                          L.total_rays, L.queue, L.sel_flag,
                                                                          L.sel_list);
                if ((e = cudaGetLastError()) != cudaSuccess) return e;
            }
        }
        // Beside: the binary32 kernel on the side stream from the fork on, with
        // the block slots the binary64 kernel's blocks leave; on `stream` the
        // binary64 kernel, then binary32 blocks for those slots, which take
        // from the same queue whatever is left when the binary64 blocks are
        // done (neither kernel waits for the other).  The pass over rays the
        // binary32 kernels hand over runs after both, on `stream`.
        const int sel = L.near_critical ? 2 : 0;
        auto launch32 = [&](int grid, cudaStream_t s) {
            return L.reg_variant ? launch_t<Mixed, kRegMixedWide, JET, SURF>(L, 0, grid, L.block_size, s, sel)
                                 : launch_t<Mixed, kRegMixed, JET, SURF>(L, 0, grid, L.block_size, s, sel);
        };
        if (side) {
            if ((e = cudaEventRecord(L.fork_event, stream)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(L.side_stream, L.fork_event, 0)) != cudaSuccess) return e;
        }
        if (L.near_critical &&
            (e = launch_t<Fp64, kRegFp64, JET, SURF>(L, 0, L.grid_side, 128, stream, 1)) != cudaSuccess)
            return e;
        if ((e = launch32(L.grid, side ? L.side_stream : stream)) != cudaSuccess) return e;
        if (side) {
            if (L.grid_late > 0 && (e = launch32(L.grid_late, stream)) != cudaSuccess) return e;
            if ((e = cudaEventRecord(L.join_event, L.side_stream)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(stream, L.join_event, 0)) != cudaSuccess) return e;
        }
        // Listed near-critical rays beyond one per lane of the binary64 kernel
        // beside (a frame dense in them, like one centred on the photon ring):
        // on the whole GPU once the binary32 kernels are done.
        if (L.near_critical && L.sel_list &&
            (e = launch_t<Fp64, kRegFp64, JET, SURF>(L, 0, L.grid_list, 128, stream, 1, 1)) != cudaSuccess)
            return e;
        if (L.resume_event) cudaEventRecord(L.resume_event, stream);
        // The deferred rays, in binary64: every block reads the deferred count.
        return launch_fp64<JET, SURF>(L, 1, L.grid_resume, L.block_resume, L.reg_variant_resume, stream);
    }
    return launch_fp64<JET, SURF>(L, 0, L.grid, L.block_size, L.reg_variant, stream);
}

}  // namespace

size_t deferred_record_bytes() { return sizeof(Deferred); }

cudaError_t launch_eval_rhs(int precision, const FrameParams* d_frame, const double* d_in, long long n,
                            double* d_out, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((n + 127) / 128);
    if (precision == BH_PRECISION_MIXED) eval_rhs_kernel<Mixed><<<grid, 128, 0, stream>>>(d_frame, d_in, n, d_out);
    else eval_rhs_kernel<Fp64><<<grid, 128, 0, stream>>>(d_frame, d_in, n, d_out);
    return cudaGetLastError();
}

cudaError_t launch_trace(const TraceLaunch& L, cudaStream_t stream) {
    cudaError_t e;
    if (L.jet) e = launch_trace_t<true, kSurfAll>(L, stream);
    else if (L.surfaces) e = launch_trace_t<false, kSurfAll>(L, stream);
    else if (L.xing) e = launch_trace_t<false, kSurfCrossings>(L, stream);
    else e = launch_trace_t<false, kSurfNone>(L, stream);
    if (e != cudaSuccess || !L.band_done) return e;
    // Every band counter up to its band's size once all trace kernels are
    // done (rays a budget or an abort left untraced included), so a stream
    // waiting on a band never waits past the trace.
    band_release_kernel<<<1, 256, 0, stream>>>(L.band_done, L.nbands, L.total_rays,
                                               L.rays_per_band > 0 ? L.rays_per_band : 1);
    return cudaGetLastError();
}

int trace_blocks_per_sm(int precision, int block_size, int variant) {
    const void* k[kFamily];
    kernels_of(precision, variant, k);
    int least = 0;
    for (int i = 0; i < kFamily; ++i) {
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k[i], block_size, 0);
        if (i == 0 || n < least) least = n;
    }
    return least;
}

int trace_registers(int precision, int variant) {
    const void* k[kFamily];
    kernels_of(precision, variant, k);
    int most = 0;
    for (int i = 0; i < kFamily; ++i) {
        cudaFuncAttributes at;
        cudaFuncGetAttributes(&at, k[i]);
        if (at.numRegs > most) most = at.numRegs;
    }
    return most;
}

}  // namespace bhg
