// bh_adjoint_check.cu - Test harness: the per-ray adjoint run on the CPU.
//
// Builds libbh_adjoint_check.so, which the tests load to check the adjoint's
// mathematics without a GPU: the same __host__ __device__ functions the
// adjoint kernel runs (bh_adjoint.cuh), compiled for the host, differentiated
// against central finite differences of their own forward pass.  Not part of
// the render library and never loaded by it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../bh_adjoint.cuh"
#include "../bh_scene.h"

using namespace bhg;

namespace {

struct SkyCache {
    bool valid = false;
    int count = -1;
    uint64_t seed = 0;
    int mode = -1;
    std::vector<double> table;
    HostSky sky;
};
SkyCache g_sky;
std::mutex g_mu;

int prepare(const bh_render_config* cfg, FrameParams& F, AdjointFrame& X, SkyData& sd) {
    std::string err;
    bh_render_config c = *cfg;
    c.precision = BH_PRECISION_FP64;
    int rc = make_frame(c, F, err);
    if (rc != BH_OK) return rc;
    rc = make_adjoint_frame(c, F, X, err);
    if (rc != BH_OK) return rc;
    const int count = c.stars_enabled ? c.star_count : 0;
    if (!g_sky.valid || g_sky.count != count || g_sky.seed != c.seed || g_sky.mode != c.sky_mode) {
        build_blackbody_table(g_sky.table);
        g_sky.sky = HostSky{};
        rc = build_sky(count, c.seed, c.sky_mode, g_sky.table, g_sky.sky, err);
        if (rc != BH_OK) return rc;
        g_sky.valid = true;
        g_sky.count = count;
        g_sky.seed = c.seed;
        g_sky.mode = c.sky_mode;
    }
    std::memset(&sd, 0, sizeof sd);
    sd.star_pos = g_sky.sky.pos.data();
    sd.star_col = g_sky.sky.col.data();
    sd.bin_start = g_sky.sky.bin_start.data();
    sd.table = g_sky.table.data();
    sd.mw_x = g_sky.sky.mw_x;
    sd.mw_z = g_sky.sky.mw_z;
    sd.mw_inv = g_sky.sky.mw_inv;
    sd.diffuse_L = g_sky.sky.diffuse_L;
    sd.n_stars = static_cast<int32_t>(g_sky.sky.pos.size());
    return BH_OK;
}

adj::RayC ray_consts(const double c7[7]) {
    adj::RayC c;
    c.a = c7[0];
    c.a2 = c7[1];
    c.E = c7[2];
    c.Lz = c7[3];
    c.rp = c7[4];
    c.rm = c7[5];
    c.factored = c7[6] != 0.0;
    return c;
}

}  // namespace

extern "C" {

// Right-hand side at (r, th, p_r, p_th) for constants (a, a^2, E, L_z, r+, r-, factored).
int bhx_rhs(const double c7[7], const double x4[4], double d[6]) {
    double sn, cs;
    adj::rhs6_th(ray_consts(c7), x4[0], x4[1], x4[2], x4[3], d, &sn, &cs);
    return 0;
}

// Its vector-Jacobian product: out = (d/dr, d/dth, d/dp_r, d/dp_th, d/dE, d/dL_z, d/da) of db . rhs.
int bhx_rhs_vjp(const double c7[7], const double x4[4], const double db[6], double out[7]) {
    double g[4] = {0, 0, 0, 0};
    double Eb = 0, Lzb = 0, ab = 0;
    adj::rhs6_vjp(ray_consts(c7), x4[0], std::sin(x4[1]), std::cos(x4[1]), x4[2], x4[3], db, g, &Eb, &Lzb, &ab);
    for (int i = 0; i < 4; ++i) out[i] = g[i];
    out[4] = Eb;
    out[5] = Lzb;
    out[6] = ab;
    return 0;
}

// One ray of `cfg` (frame-local ray id in work order) with loss weight w:
// out = (Y, w dY/d spin, w dY/d incl, w dY/d eddington, w dY/d r_out, what,
// steps, replayed steps, checkpoint interval).  forward_only: Y only.
int bhx_ray(const bh_render_config* cfg, long long local_id, double w, int forward_only, int slots,
            double out[9]) {
    std::lock_guard<std::mutex> lock(g_mu);
    FrameParams F;
    AdjointFrame X;
    SkyData sd;
    const int rc = prepare(cfg, F, X, sd);
    if (rc != BH_OK) return rc;
    if (slots > 0) X.checkpoint_slots = slots;
    std::vector<double> ck(static_cast<size_t>(X.checkpoint_slots) * 8);
    adj::RayResult r;
    adj::adjoint_ray(F, X, sd, local_id, w, ck.data(), X.checkpoint_slots, forward_only != 0, &r);
    out[0] = r.Y;
    for (int q = 0; q < 4; ++q) out[1 + q] = r.grad[q];
    out[5] = r.what;
    out[6] = r.steps;
    out[7] = static_cast<double>(r.replay);
    out[8] = r.interval;
    return BH_OK;
}

// The frame's adjoint constants (AdjointFrame, as doubles) for inspection.
int bhx_frame_tangents(const bh_render_config* cfg, double out[32]) {
    std::lock_guard<std::mutex> lock(g_mu);
    FrameParams F;
    AdjointFrame X;
    SkyData sd;
    const int rc = prepare(cfg, F, X, sd);
    if (rc != BH_OK) return rc;
    int k = 0;
    for (int i = 0; i < 5; ++i)
        for (int q = 0; q < 2; ++q) out[k++] = X.d_tet[i][q];
    for (int i = 0; i < 5; ++i)
        for (int q = 0; q < 2; ++q) out[k++] = X.d_ml[i][q];
    out[k++] = X.d_x0;
    out[k++] = X.d_mdot_da;
    out[k++] = X.d_mdot_dedd;
    return BH_OK;
}

// The first two equatorial crossings of one ray (frame-local id, work
// order): their radii and accepted steps (0: none); *n_out = how many,
// *count (may be NULL) = all of the ray's crossings.
int bhx_crossings(const bh_render_config* cfg, long long local_id, double r[2], int steps[2], int* n_out,
                  int* count) {
    std::lock_guard<std::mutex> lock(g_mu);
    FrameParams F;
    AdjointFrame X;
    SkyData sd;
    const int rc = prepare(cfg, F, X, sd);
    if (rc != BH_OK) return rc;
    std::vector<double> ck(static_cast<size_t>(X.checkpoint_slots) * 8);
    adj::RayResult res;
    adj::Crossings xr;
    xr.n = 0;
    xr.count = 0;
    xr.r[0] = xr.r[1] = 0.0;
    xr.step[0] = xr.step[1] = 0;
    adj::adjoint_ray(F, X, sd, local_id, 0.0, ck.data(), X.checkpoint_slots, true, &res, &xr);
    for (int k = 0; k < 2; ++k) {
        r[k] = xr.r[k];
        steps[k] = xr.step[k];
    }
    *n_out = xr.n;
    if (count) *count = xr.count;
    return BH_OK;
}

// The edge term (edge_sample) of equatorial crossing number `crossing` (1 or
// 2) of sample k of pixel (px, py) for the edges `edges` (1 outer, 2 inner,
// 3 both):
// out = contributions to dLoss/d(r_out, spin, inclination) for pixel weight
// w; diag = (r_c, |grad r_c|, d r_c/d spin, d r_c/d incl, d r_c/d su,
// d r_c/d sv, L and dY of the outer edge, L and dY of the inner edge, cells
// crossed, steps integrated).
int bhx_edge(const bh_render_config* cfg, int px, int py, int k, int crossing, int edges, double w,
             double out[3], double diag[12]) {
    std::lock_guard<std::mutex> lock(g_mu);
    FrameParams F;
    AdjointFrame X;
    SkyData sd;
    const int rc = prepare(cfg, F, X, sd);
    if (rc != BH_OK) return rc;
    std::vector<double> ck(static_cast<size_t>(X.checkpoint_slots) * 8);
    for (int i = 0; i < 12; ++i) diag[i] = 0.0;
    int cells = 0;
    diag[11] = static_cast<double>(
        adj::edge_sample(F, X, sd, px, py, k, crossing, edges, w, ck.data(), X.checkpoint_slots, out, &cells,
                         diag));
    diag[10] = cells;
    return BH_OK;
}

// edge_mask: which edges the crossing at rc is examined for, given the
// spread dmax of its neighbours' same crossing.
int bhx_edge_mask(const bh_render_config* cfg, double rc, double dmax, int* mask) {
    std::lock_guard<std::mutex> lock(g_mu);
    FrameParams F;
    AdjointFrame X;
    SkyData sd;
    const int rc2 = prepare(cfg, F, X, sd);
    if (rc2 != BH_OK) return rc2;
    *mask = adj::edge_mask(F, rc, dmax);
    return BH_OK;
}

// The image-plane position (su, sv, x, y in pixels) of sample k of pixel (px, py).
int bhx_sample_position(const bh_render_config* cfg, int px, int py, int k, double out[4]) {
    std::lock_guard<std::mutex> lock(g_mu);
    FrameParams F;
    AdjointFrame X;
    SkyData sd;
    const int rc = prepare(cfg, F, X, sd);
    if (rc != BH_OK) return rc;
    adj::sample_position_at(F, px, py, k, &out[0], &out[1], &out[2], &out[3]);
    return BH_OK;
}

// The radius of equatorial crossing number `crossing` of the ray through
// image-plane position (su, sv), or NaN when the ray ends before it.
int bhx_crossing_radius(const bh_render_config* cfg, double su, double sv, int crossing, double* r_c) {
    std::lock_guard<std::mutex> lock(g_mu);
    FrameParams F;
    AdjointFrame X;
    SkyData sd;
    const int rc = prepare(cfg, F, X, sd);
    if (rc != BH_OK) return rc;
    double y0[6], E, Lz, dy0[2][6], dE[2], dLz[2];
    adj::ray_start_at(F, X, su, sv, y0, &E, &Lz, dy0, dE, dLz);
    const adj::RayC c = adj::ray_consts(F, E, Lz);
    adj::Integ s;
    adj::integ_start(F, y0, s);
    double r = 0.0;
    *r_c = (adj::forward_run(F, c, s, nullptr, nullptr, crossing, &r) == -1) ? r : std::nan("");
    return BH_OK;
}

}  // extern "C"
