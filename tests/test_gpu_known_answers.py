"""The reference's known answers (validate.cpp) re-run with the device functions.

The render path's arithmetic as the GPU runs it, evaluated through
bh_gpu_eval and bh_gpu_trace_rays, against the closed forms and thresholds
of the reference's own validation suite and against the oracle (which
restates the reference bit for bit and passes the same checks on the CPU,
tests/test_oracle.py):

  * section 1 (metric, validate.cpp:277-330): the trace kernels' right-hand
    side, written in Carter's separated form with one reciprocal, equals the
    oracle's Hamiltonian form built from g^{mu nu} and its derivatives
    (geodesic.h:50-71) at random states over four spins, near the horizon
    and near the axis included, to 16 units of the format's roundoff of the
    size of each component's terms;
  * section 3 (orbits, validate.cpp:393-455): the frame's horizons, ISCO and
    radiative efficiency against the closed forms;
  * section 4 (null geodesics, validate.cpp:463-495): rays from r0 = 60,
    th0 = 1.3 at a = 0.9 sweeping past the shadow's edge, rtol 1e-10 /
    atol 1e-12, stopped at 1.01 r_+, traced by the binary64 kernel: the worst
    null norm and Carter drift along each whole trajectory equal the
    reference algorithm's (the oracle's), the drift stays below 1e-8;
    E = -p_t and L_z = p_phi come back bit for bit;
  * section 6 (disc, validate.cpp:857-889): the device's Novikov-Thorne
    temperature equals the oracle's to 1e-12 (1e-9 within 1 % of the ISCO,
    where W is a small difference of large terms);
  * section 7 (spectrum, validate.cpp:1005-1015): the device's blackbody
    lookup is within 2e-3 of the exact colour-matching integral and equals
    the oracle's table lookup to 1e-12.
"""
import math

import numpy as np
import pytest

from blackhole_b200 import abi
from blackhole_b200.config import Camera, RenderConfig

pytestmark = pytest.mark.gpu

M_SUN = 1.98847e30


def _cfg(spin, precision=abi.PRECISION_FP64, **kw):
    cfg = RenderConfig(M_kg=10.0 * M_SUN, spin=spin, width=8, height=8, disc_r_out=30.0, eddington=0.1,
                       precision=precision, quiet=True)
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def _random_states(orc, a, n, rng):
    """States over the whole exterior: r log-uniform from just outside r_+
    to 1000 M, th over (0, pi) with a share next to the axis, momenta of
    both signs (the right-hand side is a function of any state, null or
    not)."""
    rp = orc.scalar("horizon_outer", a)
    r = rp + np.exp(rng.uniform(math.log(1e-3), math.log(1000.0), n))
    th = rng.uniform(0.02, math.pi - 0.02, n)
    th[: n // 10] = rng.choice([1e-4, math.pi - 1e-4, 3e-3], n // 10)
    y = np.zeros((n, 8))
    y[:, 1] = r
    y[:, 2] = th
    y[:, 3] = rng.uniform(0, 2 * math.pi, n)
    y[:, 4] = -rng.uniform(0.5, 1.5, n)                 # p_t = -E
    y[:, 5] = rng.normal(0, 1, n) * (1.0 + 1.0 / (r - rp))
    y[:, 6] = rng.normal(0, 5, n)
    y[:, 7] = rng.normal(0, 4, n)                       # p_phi = L_z
    return y


def _term_scale(a, y):
    """Per state and component, the sum of the magnitudes of the terms the
    right-hand side adds (Carter's form, geodesic.h:50-71 rewritten), each
    term that holds Delta multiplied by the condition number of
    Delta = r^2 - 2r + a^2 as the reference forms it: the size a rounding
    error of either form is measured against."""
    r, th, pr, pth = y[:, 1], y[:, 2], y[:, 5], y[:, 6]
    E, Lz = -y[:, 4], y[:, 7]
    sn, cs = np.sin(th), np.cos(th)
    sn = np.where(np.abs(sn) < 1e-9, np.copysign(1e-9, sn), sn)
    sn2, cs2, r2 = sn * sn, cs * cs, r * r
    S = r2 + a * a * cs2
    Dl = r2 - 2 * r + a * a
    iS, iD, isn2 = 1 / S, 1 / np.abs(Dl), 1 / sn2
    r2a2 = r2 + a * a
    K = r2a2 * E - a * Lz
    Lp = Lz - a * E * sn2
    KiD = np.abs(K) * iD
    B = np.abs(Dl) * pr * pr + pth * pth + Lp * Lp * isn2 + np.abs(K) * KiD
    Dr = np.abs(2 * r - 2)
    out = np.zeros((len(r), 8))
    out[:, 0] = iS * (np.abs(a * Lp) + r2a2 * KiD)
    out[:, 1] = np.abs(Dl * pr) * iS
    out[:, 2] = np.abs(pth) * iS
    out[:, 3] = iS * (np.abs(Lp) * isn2 + np.abs(a) * KiD)
    out[:, 5] = 0.5 * iS * (Dr * pr * pr + 4 * r * np.abs(E) * KiD + Dr * KiD * KiD + 2 * r * B * iS)
    out[:, 6] = np.abs(sn * cs) * iS * (a * a * E * E + Lz * Lz * isn2 * isn2 + a * a * B * iS)
    return out * ((r2 + 2 * r + a * a) / np.abs(Dl))[:, None]


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_right_hand_side_equals_the_metric_form(renderer, orc, precision):
    """|device - oracle| <= 16 eps (sum of |terms|) per component, eps the
    unit roundoff of the kernel's format (measured: 4.4 for binary64 with the
    same Carter form compiled for the host).  The binary32 kernel rounds the
    state, E and L_z to binary32 first; the oracle is evaluated at those
    rounded values (the rounding of the inputs is the mixed path's, not an
    error of its arithmetic), at the states the mixed kernel integrates in
    binary32 (r >= r_+ + 0.5: it hands closer rays to binary64)."""
    rng = np.random.default_rng(20240921)
    eps = 2.0 ** -53 if precision == abi.PRECISION_FP64 else 2.0 ** -24
    worst = 0.0
    for a in (0.0, 0.5, 0.9, 0.998):
        y = _random_states(orc, a, 1000, rng)
        if precision == abi.PRECISION_MIXED:
            y = y[y[:, 1] >= orc.scalar("horizon_outer", a) + 0.5]
            y[:, [1, 2, 4, 5, 6, 7]] = y[:, [1, 2, 4, 5, 6, 7]].astype(np.float32).astype(np.float64)
        got = renderer.eval(_cfg(a, precision), abi.EVAL_RHS, y)
        want = np.array([orc.geodesic_rhs(a, yi) for yi in y])
        assert not got[:, 4].any() and not got[:, 7].any()
        scale = _term_scale(a, y)
        for j in (0, 1, 2, 3, 5, 6):
            worst = max(worst, float(np.max(np.abs(got[:, j] - want[:, j]) / (eps * scale[:, j]))))
    assert worst < 16.0, worst


def test_horizons_isco_and_efficiency(renderer, orc):
    close = lambda x, v, t: abs(x - v) <= t * max(abs(v), 1e-300)  # noqa: E731
    f0 = renderer.eval(_cfg(0.0), abi.EVAL_FRAME)
    assert close(f0[0], 2.0, 1e-15) and f0[1] == 0.0
    assert close(f0[2], 6.0, 1e-12)
    assert close(f0[4], 1.0 - math.sqrt(8.0 / 9.0), 1e-12)
    # the disc clamps its spin to 0.9999 (disc.h:75): the ISCO of 0.9999,
    # against the closed form
    for sense in (1, -1):
        f = renderer.eval(_cfg(1.0, disc_sense=sense), abi.EVAL_FRAME)
        assert close(f[2], orc.scalar("isco_radius", 0.9999, sense), 1e-12)
    assert 0.30 < renderer.eval(_cfg(0.998), abi.EVAL_FRAME)[4] < 0.33
    for a in (0.3, 0.7, 0.95):
        f = renderer.eval(_cfg(a), abi.EVAL_FRAME)
        assert close(f[0], 1.0 + math.sqrt(1.0 - a * a), 1e-15)
        assert close(f[1], 1.0 - math.sqrt(1.0 - a * a), 1e-12)
        assert close(f[2], orc.scalar("isco_radius", a, 1), 1e-14)
        assert close(f[4], orc.scalar("disc_efficiency", a, 1), 1e-14)
    # the limits of validate.cpp:393-455, approached
    f = renderer.eval(_cfg(0.9999, disc_sense=1), abi.EVAL_FRAME)
    assert 1.0 < f[2] < 1.2
    f = renderer.eval(_cfg(0.9999, disc_sense=-1), abi.EVAL_FRAME)
    assert 8.99 < f[2] < 9.0


def test_null_geodesics_conserve_norm_and_carter_constant(renderer, orc):
    """Two 24 x 24 sweeps from the reference's point (a = 0.9, r0 = 60,
    th0 = 1.3): one across the shadow and its edge (fov 0.4 rad), one out to
    1.2 rad from the hole (fov 2.4 rad), with the reference test's rtol,
    atol and stop radius.  The reference checks its 24 rays at their end
    (null norm < 1e-10, Carter drift < 1e-8); the render path records the
    worst along each whole trajectory, which on these sweeps reaches 3.7e-10
    in the reference's own algorithm (the oracle) too.  So: every ray's worst
    null norm and Carter drift equal the oracle's (to 2 %, binary32
    bookkeeping of the maxima), the drift stays below 1e-8 and the norm below
    1e-9; E = -p_t and L_z = p_phi, constants of the kernel's form, equal the
    oracle's initial photon bit for bit."""
    horizon = 0
    for fov in (0.4, 2.4):
        cfg = RenderConfig(
            M_kg=10.0 * M_SUN, spin=0.9,
            cam=Camera(r=60.0, theta=1.3, phi=0.0, fov=fov),
            width=24, height=24, sqrt_spp=1, disc_enabled=False, stars_enabled=False,
            rtol=1e-10, atol=1e-12, r_escape=2000.0, max_steps=20000,
            stop_mode=abi.STOP_RELATIVE, stop_epsilon=0.01, quiet=True,
        )
        rec = renderer.trace_rays(cfg)
        o, _ = orc.trace_rays(cfg)
        assert np.array_equal(rec["what"], o["what"])
        assert (rec["what"] != abi.HIT_EXHAUSTED).all()
        horizon += int((rec["what"] == abi.HIT_HORIZON).sum())
        assert np.allclose(rec["max_norm"], o["max_norm"], rtol=0.02, atol=1e-14)
        assert np.allclose(rec["max_q"], o["max_q"], rtol=0.02, atol=1e-14)
        assert float(rec["max_norm"].max()) < 1e-9
        assert float(rec["max_q"].max()) < 1e-8
        assert np.array_equal(rec["y"][:, 4], o["y"][:, 4]) and np.array_equal(rec["y"][:, 7], o["y"][:, 7])
    assert horizon > 20


def test_disc_temperature_equals_the_oracle(renderer, orc):
    """The three prograde discs glow from just outside the ISCO to r_out.
    The counter-rotating disc is dark in the reference (its Page-Thorne W,
    disc.h:46-64, is evaluated with +a whatever the sense, and comes out
    negative), and so it is here."""
    worst = 0.0
    for a, sense in ((0.0, 1), (0.9, 1), (0.998, 1), (0.7, -1)):
        cfg = _cfg(a, disc_sense=sense, eddington=0.3, disc_r_out=80.0)
        f = renderer.eval(cfg, abi.EVAL_FRAME)
        r = np.concatenate([f[2] * (1.0 + np.geomspace(1e-6, 1.0, 200)), np.linspace(2 * f[2], f[3], 200)])
        T = renderer.eval(cfg, abi.EVAL_DISC_TEMPERATURE, r)
        want = np.array([orc.scalar("disc_temperature", cfg.M_kg, a, cfg.disc_r_out, cfg.eddington, sense, x)
                         for x in r])
        if sense < 0:
            assert not T.any() and not want.any()
            continue
        assert (T > 0).all()
        err = np.abs(T - want) / want
        # next to the ISCO, W is a difference of terms up to 1e6 times its
        # size: both forms' rounding shows there
        near = r < 1.01 * f[2]
        assert float(err[near].max()) < 1e-9
        worst = max(worst, float(err[~near].max()))
        # outside the disc: no emission
        out = renderer.eval(cfg, abi.EVAL_DISC_TEMPERATURE, np.array([0.5 * f[2], f[2], f[3] * 1.01]))
        assert not out.any()
    assert worst < 1e-12, worst


def test_blackbody_lookup_against_the_exact_integral(renderer, orc):
    T = 10.0 ** np.arange(2.0, 8.0 + 1e-9, 0.13)
    got = renderer.eval(_cfg(0.5), abi.EVAL_BLACKBODY, T)
    exact = np.array([orc.blackbody_xyz_exact(t) for t in T])
    table = np.array([orc.blackbody_xyz(t) for t in T])
    assert float(np.max(np.abs(got[:, 1] - exact[:, 1]) / exact[:, 1])) < 2e-3
    assert float(np.max(np.abs(got - table) / table)) < 1e-12


def test_eval_refuses_bad_requests(renderer):
    import ctypes as C

    from blackhole_b200.gpu import BHError

    with pytest.raises(BHError) as e:
        renderer.eval(_cfg(0.5, disc_enabled=False), abi.EVAL_DISC_TEMPERATURE, np.array([10.0]))
    assert e.value.code == abi.ERR_INVALID_ARG
    c = _cfg(0.5).to_c()
    out = np.zeros(8)
    dp = C.POINTER(C.c_double)
    rc = renderer.lib.bh_gpu_eval(renderer.handle, C.byref(c), 7, out.ctypes.data_as(dp), 1, out.ctypes.data_as(dp))
    assert rc == abi.ERR_INVALID_ARG
    rc = renderer.lib.bh_gpu_eval(renderer.handle, C.byref(c), abi.EVAL_RHS, None, 4, out.ctypes.data_as(dp))
    assert rc == abi.ERR_INVALID_ARG
    # nothing to evaluate is no error
    assert renderer.eval(_cfg(0.5), abi.EVAL_BLACKBODY, np.zeros(0)).shape == (0, 3)
