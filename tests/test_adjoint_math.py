"""The discrete adjoint's per-ray mathematics, checked on the CPU.

libbh_adjoint_check.so is the adjoint kernel's own __host__ __device__ code
(blackhole_b200/csrc/bh_adjoint.cuh) compiled for the host.  These tests hold
it against central finite differences of its own forward pass: the
right-hand side's vector-Jacobian product, whole rays (disc hits and star-lit
sky rays) for the spin, inclination and Eddington ratio, and the checkpoint
thinning, which must not change a single bit of the gradient.
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
