"""The discrete adjoint's per-ray mathematics, checked on the CPU.

libbh_adjoint_check.so is the adjoint kernel's own __host__ __device__ code
(blackhole_b200/csrc/bh_adjoint.cuh) compiled for the host.  These tests hold
it against central finite differences of its own forward pass: the
right-hand side's vector-Jacobian product, whole rays (disc hits and star-lit
sky rays) for the spin, inclination and Eddington ratio, and the checkpoint
thinning, which must not change a single bit of the gradient.  For the edge
term (the motion of the disc's edges across the image): the gradient of an
equatorial crossing's radius with respect to the image-plane position, the
spin and the inclination, against central differences of the crossing
radius, and the rule that picks the crossings examined for an edge.
"""
import copy
import ctypes as C
import math
import os

import numpy as np
import pytest

from blackhole_b200 import abi, workloads
from blackhole_b200.build import CHECK_LIB, build_check

D = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def chk():
    if not os.path.exists(CHECK_LIB):
        build_check()
    lib = C.CDLL(CHECK_LIB)
    lib.bhx_rhs.argtypes = [D, D, D]
    lib.bhx_rhs_vjp.argtypes = [D, D, D, D]
    lib.bhx_ray.argtypes = [C.POINTER(abi.bh_render_config), C.c_longlong, C.c_double, C.c_int, C.c_int, D]
    P = C.POINTER(abi.bh_render_config)
    I = C.POINTER(C.c_int)
    lib.bhx_crossings.argtypes = [P, C.c_longlong, D, I, I, I]
    lib.bhx_edge.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, D, D]
    lib.bhx_crossing_radius.argtypes = [P, C.c_double, C.c_double, C.c_int, D]
    lib.bhx_sample_position.argtypes = [P, C.c_int, C.c_int, C.c_int, D]
    lib.bhx_edge_mask.argtypes = [P, C.c_double, C.c_double, I]
    return lib


def _a(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def _p(x):
    return x.ctypes.data_as(D)


def _ray(lib, cfg, rid, w=1.0, forward_only=False, slots=0):
    out = _a(np.zeros(9))
    c = cfg.to_c()
    rc = lib.bhx_ray(C.byref(c), rid, w, int(forward_only), slots, _p(out))
    assert rc == abi.OK, rc
    return out


def _with(cfg, k, v):
    c = copy.deepcopy(cfg)
    if k == 0:
        c.spin = v
    elif k == 1:
        c.cam.theta = v
    else:
        c.eddington = v
    return c


def _params(cfg):
    return [cfg.spin, cfg.cam.theta, cfg.eddington]


def test_rhs_vjp_matches_finite_differences(chk):
    rng = np.random.default_rng(7)
    for a in (0.0, 0.5, 0.9, 0.998):
        s = math.sqrt(1 - a * a)
        for _ in range(10):
            E, Lz = -1.0, rng.uniform(-6, 6)
            c7 = _a([a, a * a, E, Lz, 1 + s, 1 - s, 1])
            x = _a([rng.uniform(2.5, 80), rng.uniform(0.2, 2.9), rng.uniform(-1, 1), rng.uniform(-4, 4)])
            db = _a(rng.normal(size=6))
            got = _a(np.zeros(7))
            chk.bhx_rhs_vjp(_p(c7), _p(x), _p(db), _p(got))

            def f(cc, xx):
                d = _a(np.zeros(6))
                chk.bhx_rhs(_p(_a(cc)), _p(_a(xx)), _p(d))
                return float(d @ db)

            fd = []
            for i in range(4):
                h = 1e-6 * max(1.0, abs(x[i]))
                xp, xm = x.copy(), x.copy()
                xp[i] += h
                xm[i] -= h
                fd.append((f(c7, xp) - f(c7, xm)) / (2 * h))
            for i in (2, 3):
                cp, cm = c7.copy(), c7.copy()
                cp[i] += 1e-6
                cm[i] -= 1e-6
                fd.append((f(cp, x) - f(cm, x)) / 2e-6)

            def ca(v):
                q = math.sqrt(1 - v * v)
                return _a([v, v * v, E, Lz, 1 + q, 1 - q, 1])

            h = 1e-6 if a < 0.99 else 1e-7
            fd.append((f(ca(a + h), x) - f(ca(a - h), x)) / (2 * h))
            fd = np.array(fd)
            scale = np.abs(fd).max()
            assert np.allclose(got, fd, rtol=1e-4, atol=1e-6 * scale), (a, got, fd)


def _frame(n=64):
    cfg = workloads.adjoint_512()
    cfg.width = cfg.height = n
    return cfg


@pytest.mark.parametrize("rid", [2080, 2100, 3000, 640])
def test_disc_ray_gradient_matches_finite_differences(chk, rid):
    cfg = _frame()
    got = _ray(chk, cfg, rid)
    assert int(got[5]) == abi.HIT_DISC and got[0] > 0
    for k, v in enumerate(_params(cfg)):
        h = 1e-5 * abs(v)
        yp = _ray(chk, _with(cfg, k, v + h), rid, forward_only=True)
        ym = _ray(chk, _with(cfg, k, v - h), rid, forward_only=True)
        assert int(yp[5]) == int(ym[5]) == abi.HIT_DISC
        fd = (yp[0] - ym[0]) / (2 * h)
        assert got[1 + k] == pytest.approx(fd, rel=1e-4), (k, got[1 + k], fd)
    assert got[4] == 0.0          # r_out: no interior derivative


def test_star_lit_sky_ray_gradient_matches_finite_differences(chk):
    cfg = _frame(128)
    bg = None
    lit = []
    for rid in range(0, 2000):
        o = _ray(chk, cfg, rid, forward_only=True)
        if int(o[5]) != abi.HIT_SKY:
            continue
        bg = o[0] if bg is None else min(bg, o[0])
        if bg and o[0] > 3 * bg:
            lit.append(rid)
        if len(lit) >= 3:
            break
    assert lit
    for rid in lit:
        got = _ray(chk, cfg, rid)
        v = cfg.cam.theta
        h = 1e-7 * v
        yp = _ray(chk, _with(cfg, 1, v + h), rid, forward_only=True)
        ym = _ray(chk, _with(cfg, 1, v - h), rid, forward_only=True)
        fd = (yp[0] - ym[0]) / (2 * h)
        assert got[2] == pytest.approx(fd, rel=1e-4, abs=1e-6 * abs(got[0]) / h)


def test_checkpoint_thinning_keeps_the_gradient_bitwise(chk):
    cfg = _frame()
    for rid in (640, 2080):
        base = _ray(chk, cfg, rid)
        for slots in (4, 2):
            thin = _ray(chk, cfg, rid, slots=slots)
            assert np.array_equal(base[:5], thin[:5])
            assert thin[8] > base[8]          # the interval grew
            assert thin[7] > base[7]          # and more steps were replayed


def test_zero_weight_and_background_rays_have_no_gradient(chk):
    cfg = _frame()
    o = _ray(chk, cfg, 2080, w=0.0)
    assert o[0] > 0 and not np.any(o[1:5])
    # a sky ray with no star in its point-spread window sees the uniform background only
    o = _ray(chk, cfg, 100)
    assert int(o[5]) == abi.HIT_SKY and not np.any(o[1:5])


def test_unsupported_scenes_are_refused(chk):
    cfg = _frame(8)
    cfg.sun_enabled = True
    out = _a(np.zeros(9))
    c = cfg.to_c()
    assert chk.bhx_ray(C.byref(c), 0, 1.0, 0, 0, _p(out)) == abi.ERR_UNSUPPORTED


# ---- the edge term --------------------------------------------------------------------


def _isco(a, sense=1):
    z1 = 1 + (1 - a * a) ** (1 / 3) * ((1 + a) ** (1 / 3) + (1 - a) ** (1 / 3))
    z2 = math.sqrt(3 * a * a + z1 * z1)
    return 3 + z2 - sense * math.sqrt((3 - z1) * (3 + z1 + 2 * z2))


def _crossings(lib, cfg):
    """First two equatorial crossings of every sample, in trace_rays order."""
    n = cfg.width * cfg.height * cfg.sqrt_spp ** 2
    order = abi.work_order(cfg.width, cfg.height, cfg.sqrt_spp)
    R = np.zeros((n, 2))
    ST = np.zeros((n, 2), dtype=np.int64)
    c = cfg.to_c()
    r = (C.c_double * 2)()
    st = (C.c_int * 2)()
    m = C.c_int()
    for rid in range(n):
        assert lib.bhx_crossings(C.byref(c), rid, r, st, C.byref(m), None) == abi.OK
        R[order[rid]] = r[:]
        ST[order[rid]] = st[:]
    return R, ST


def _edge(lib, cfg, px, py, k, crossing, edges, w=1.0):
    out, diag = _a(np.zeros(3)), _a(np.zeros(12))
    c = cfg.to_c()
    assert lib.bhx_edge(C.byref(c), px, py, k, crossing, edges, w, _p(out), _p(diag)) == abi.OK
    return out, diag


def _rc(lib, cfg, su, sv, crossing):
    c = cfg.to_c()
    r = C.c_double()
    assert lib.bhx_crossing_radius(C.byref(c), su, sv, crossing, C.byref(r)) == abi.OK
    return r.value


@pytest.fixture(scope="module")
def edge_frame(chk):
    cfg = workloads.adjoint_512()
    cfg.width = cfg.height = 48
    R, ST = _crossings(chk, cfg)
    return cfg, R, ST


def test_crossing_radius_gradient_matches_finite_differences(chk, edge_frame):
    """d r_c/d(su, sv, spin, inclination) from the reverse sweep of the
    crossing radius, at crossings next to both edges, against central
    differences of the radius of the same crossing."""
    cfg, R, ST = edge_frame
    r_in = _isco(cfg.spin)
    picked = []
    for edge, re in ((1, cfg.disc_r_out), (2, r_in)):
        near = np.argwhere((ST > 0) & (np.abs(R - re) < 0.05 * re))
        assert len(near) >= 3, edge
        picked += [(edge, int(o), int(j)) for o, j in near[:: max(1, len(near) // 3)][:3]]
    for edge, o, j in picked:
        px, py = o % cfg.width, o // cfg.width
        step = j + 1                  # crossing number
        _, diag = _edge(chk, cfg, px, py, 0, step, edge)
        assert diag[0] == pytest.approx(R[o, j], rel=1e-12)
        pos = _a(np.zeros(4))
        c = cfg.to_c()
        assert chk.bhx_sample_position(C.byref(c), px, py, 0, _p(pos)) == abi.OK
        su, sv = pos[0], pos[1]
        h = 1e-6
        fd = [
            (_rc(chk, _with(cfg, 0, cfg.spin + h), su, sv, step) - _rc(chk, _with(cfg, 0, cfg.spin - h), su, sv, step)) / (2 * h),
            (_rc(chk, _with(cfg, 1, cfg.cam.theta + h), su, sv, step)
             - _rc(chk, _with(cfg, 1, cfg.cam.theta - h), su, sv, step)) / (2 * h),
            (_rc(chk, cfg, su + h, sv, step) - _rc(chk, cfg, su - h, sv, step)) / (2 * h),
            (_rc(chk, cfg, su, sv + h, step) - _rc(chk, cfg, su, sv - h, step)) / (2 * h),
        ]
        scale = max(abs(x) for x in fd)
        for got, want in zip(diag[2:6], fd):
            assert got == pytest.approx(want, rel=1e-4, abs=1e-5 * scale), (edge, o, diag[2:6], fd)


def test_edge_term_of_a_cell_is_the_swept_area(chk, edge_frame):
    """For a crossing whose cell the outer edge crosses: the r_out part is
    w (Y_disc - Y_beyond) L / |grad r_c|, the spin and inclination parts that
    times -d r_c/dq, and the edge line r_c = r_out (linearised) meets the
    cell's boundary at both ends of a segment of length L."""
    cfg, R, ST = edge_frame
    near = np.argwhere((ST > 0) & (np.abs(R - cfg.disc_r_out) < 0.5))
    seen = 0
    for o, j in near:
        px, py = int(o) % cfg.width, int(o) // cfg.width
        out, d = _edge(chk, cfg, px, py, 0, int(j) + 1, 1, w=3.0)
        rc, gn, drq, L, dY = d[0], d[1], d[2:4], d[6], d[7]
        if L == 0.0 or dY == 0.0:
            assert not out.any()
            continue
        assert 0.0 < L <= math.sqrt(2.0) * (1 + 1e-12)
        swept = 3.0 * dY * L / gn
        assert out[0] == pytest.approx(swept, rel=1e-12)
        assert out[1] == pytest.approx(-swept * drq[0], rel=1e-12)
        assert out[2] == pytest.approx(-swept * drq[1], rel=1e-12)
        # the line's distance from the sample is |r_out - r_c| / |grad r_c|,
        # at most the cell's half diagonal from its centre region
        assert abs(cfg.disc_r_out - rc) / gn <= math.sqrt(2.0)
        seen += 1
    assert seen >= 5


def test_candidate_rule_finds_every_cell_an_edge_crosses(chk, edge_frame):
    """Every crossing whose cell an edge crosses (examined with a band of a
    quarter of the edge radius) is picked by the neighbour-spread rule."""
    cfg, R, ST = edge_frame
    W = cfg.width
    r_in = _isco(cfg.spin)
    c = cfg.to_c()
    m = C.c_int()
    crossed = picked = 0
    for o in range(W * W):
        x, y = o % W, o // W
        for j in range(2):
            if ST[o, j] == 0:
                break
            rc = R[o, j]
            dmax = 0.0
            for nx, ny in ((x + 1, y), (x - 1, y), (x, y + 1), (x, y - 1)):
                if 0 <= nx < W and 0 <= ny < W and ST[ny * W + nx, j] > 0:
                    dmax = max(dmax, abs(rc - R[ny * W + nx, j]))
            assert chk.bhx_edge_mask(C.byref(c), rc, dmax, C.byref(m)) == abi.OK
            for bit, re, ok in ((1, cfg.disc_r_out, rc >= r_in), (2, r_in, rc <= cfg.disc_r_out)):
                if not ok or abs(rc - re) > 0.25 * re:
                    continue
                _, d = _edge(chk, cfg, x, y, 0, j + 1, bit)
                if d[6 if bit == 1 else 8] > 0.0:
                    crossed += 1
                    assert m.value & bit, (o, j, bit, rc, dmax)
                    picked += 1
    assert crossed >= 20
