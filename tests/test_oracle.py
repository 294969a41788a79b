"""The CPU oracle: pinned against the reference and its known answers.

The oracle (oracle/bh_oracle.c) is a restatement of the reference's render
path.  These tests hold it to
  * the golden vectors under tests/golden/ (made by the reference renderer
    itself, tests/golden/make_golden.py), bit for bit;
  * the reference compiled here (oracle/_ref), bit for bit, where it exists;
  * the known-answer checks of the reference's validation suite
    (validate.cpp sections 1, 3, 4, 6, 7) with the same thresholds.
"""
import hashlib
import json
import math
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from cases import CASES, RENDER_CASE  # noqa: E402

from blackhole_b200 import abi  # noqa: E402

GOLDEN = os.path.join(HERE, "golden")


def _load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


# ---------------------------------------------------------------------------
# Pinning
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_golden_bit_for_bit(orc, name):
    make, (x0, y0, w, h) = CASES[name]
    g = _load(name)
    arr, st = orc.trace_rays(make(), x0, y0, w, h)
    assert np.array_equal(arr["what"], g["what"].astype(np.int32))
    assert np.array_equal(arr["steps"], g["steps"])
    for f in ("y", "g", "dir", "xyz"):
        assert np.array_equal(arr[f], g[f]), f
    stats = [st.rays, st.steps, st.captured, st.disc_hits, st.sun_hits, st.star_hits, st.escaped, st.exhausted]
    assert stats == g["stats"].tolist()
    assert [st.max_norm_error, st.max_carter_drift] == g["drift"].tolist()


def test_oracle_frame_matches_reference_render(orc):
    name, make = RENDER_CASE
    g = _load(name)
    cfg = make()
    px, st = orc.render_window(cfg)
    assert np.array_equal(px, g["pixels"])
    stats = [st.rays, st.steps, st.captured, st.disc_hits, st.sun_hits, st.star_hits, st.escaped, st.exhausted]
    assert stats == g["stats"].tolist()


@pytest.mark.parametrize("name", ["a09_i60_centre", "sun_hotspot_spp2"])
def test_oracle_matches_reference_build(orc, ref, name):
    """Same windows, against the reference compiled from its sources now."""
    make, (x0, y0, w, h) = CASES[name]
    a, _ = orc.trace_rays(make(), x0, y0, w, h)
    b, _ = ref.trace_rays(make(), x0, y0, w, h)
    for f in ("what", "steps", "y", "g", "dir", "xyz"):
        assert np.array_equal(a[f], b[f]), f


def test_catalogue_and_table_match_reference_digest(orc):
    meta = json.load(open(os.path.join(GOLDEN, "catalogue.json")))
    cat = orc.star_catalogue(meta["count"], meta["seed"])
    assert hashlib.sha256(cat.astype("<f8").tobytes()).hexdigest() == meta["sha256_float64_le"]
    for T, xyz in zip(meta["blackbody_T"], meta["blackbody_xyz"]):
        assert orc.blackbody_xyz(T).tolist() == xyz


def test_uniform_sky_catalogue_properties(orc):
    """The BH_SKY_UNIFORM catalogue: isotropic, m <= 6.5, B-V in [-0.3, 1.8]."""
    cat = orc.star_catalogue(200000, 7, abi.SKY_UNIFORM)
    assert np.allclose(np.linalg.norm(cat[:, :3], axis=1), 1.0, atol=1e-12)
    assert cat[:, 3].max() <= 6.5 and cat[:, 3].min() >= -1.5
    lo = orc.scalar("bv_to_temperature", 1.8)
    hi = orc.scalar("bv_to_temperature", -0.3)
    assert cat[:, 4].min() >= lo - 1e-9 and cat[:, 4].max() <= hi + 1e-9
    assert abs(cat[:, 2].mean()) < 0.01 and abs(cat[:, 0].mean()) < 0.01
    # log N(<m) = 0.45 m: N(<m+1)/N(<m) ~ 10^0.45 well above the bright end
    n5 = (cat[:, 3] < 5.0).sum()
    n6 = (cat[:, 3] < 6.0).sum()
    assert abs(n6 / n5 - 10 ** 0.45) < 0.15


# ---------------------------------------------------------------------------
# Known answers (validate.cpp)
# ---------------------------------------------------------------------------

SPINS = (0.0, 0.3, 0.7, 0.9, 0.998)
RADII = (2.6, 4.0, 9.5, 30.0, 250.0)
THETAS = (0.35, 1.0, math.pi / 2, 2.3, 2.9)


def _full(five):
    m = np.zeros((4, 4))
    m[0, 0], m[1, 1], m[2, 2], m[3, 3] = five[0], five[2], five[3], five[4]
    m[0, 3] = m[3, 0] = five[1]
    return m


def test_metric_inverse_identity(orc):
    """validate.cpp:277-300: g^{ik} g_kj = delta to 1e-11."""
    worst = 0.0
    for a in SPINS:
        rh = orc.scalar("horizon_outer", a)
        for r in RADII:
            if r <= rh * 1.02:
                continue
            for th in THETAS:
                up = orc.metric_upper_deriv(a, r, th)[:5]
                lo = orc.metric_lower(a, r, th)
                worst = max(worst, np.abs(_full(up) @ _full(lo) - np.eye(4)).max())
    assert worst < 1e-11


def test_metric_derivatives_match_finite_differences(orc):
    """validate.cpp:302-330: analytic d g^{mu nu} vs 4th-order FD."""
    worst = 0.0
    for a in SPINS:
        rh = orc.scalar("horizon_outer", a)
        for r in RADII:
            if r <= rh * 1.02:
                continue
            for th in THETAS:
                d = orc.metric_upper_deriv(a, r, th)
                for direction, off in ((1, 5), (2, 10)):
                    h = 1e-4 * max(1.0, r) if direction == 1 else 1e-4

                    def at(o):
                        rr = r + (o if direction == 1 else 0.0)
                        tt = th + (o if direction == 2 else 0.0)
                        return orc.metric_upper_deriv(a, rr, tt)[:5]

                    num = (-at(2 * h) + 8 * at(h) - 8 * at(-h) + at(-2 * h)) / (12.0 * h)
                    ana = d[off:off + 5]
                    noise = 50.0 * 2.22e-16 * np.abs(at(0.0)) / h
                    tol = 1e-6 * np.abs(ana) + noise
                    worst = max(worst, (np.abs(num - ana) / np.maximum(tol, 1e-300)).max())
    assert worst < 1.0


def test_orbits(orc):
    """validate.cpp:393-455."""
    close = lambda a, b, t: abs(a - b) / max(abs(a), abs(b), 1e-300) <= t  # noqa: E731
    assert close(orc.scalar("isco_radius", 0.0, 1), 6.0, 1e-12)
    assert close(orc.scalar("isco_radius", 1.0, 1), 1.0, 1e-9)
    assert close(orc.scalar("isco_radius", 1.0, -1), 9.0, 1e-9)
    assert close(orc.scalar("photon_circular_orbit", 0.0, 1), 3.0, 1e-12)
    assert close(orc.scalar("photon_circular_orbit", 1.0, 1), 1.0, 1e-9)
    assert close(orc.scalar("photon_circular_orbit", 1.0, -1), 4.0, 1e-9)
    eta0 = orc.scalar("disc_efficiency", 0.0, 1)
    eta1 = orc.scalar("disc_efficiency", 0.998, 1)
    assert close(eta0, 1.0 - math.sqrt(8.0 / 9.0), 1e-12) and 0.30 < eta1 < 0.33
    import ctypes as C

    worst = 0.0
    for a in (0.0, 0.5, 0.95):
        r = orc.scalar("isco_radius", a, 1)
        while r < 200.0:
            u = (C.c_double * 4)()
            orc.scalar("keplerian_four_velocity", a, r, 1, u)
            ml = orc.metric_lower(a, r, math.pi / 2)
            n = ml[0] * u[0] ** 2 + 2 * ml[1] * u[0] * u[3] + ml[4] * u[3] ** 2
            worst = max(worst, abs(n + 1.0))
            r *= 1.7
    assert worst < 1e-11


def test_null_geodesic_conservation(orc):
    """validate.cpp:463-495: 24 rays at a = 0.9 from r0 = 60, th0 = 1.3,
    rtol 1e-10 / atol 1e-12: null norm < 1e-10, Carter drift < 1e-8, E exact."""
    a, r0, th0 = 0.9, 60.0, 1.3
    rh = orc.scalar("horizon_outer", a)
    wn = wq = we = 0.0
    for i in range(24):
        ang = 0.02 + 0.05 * i
        d = np.array([-math.cos(ang), 0.2 * math.sin(ang),
                      math.sqrt(max(0.0, 1.0 - math.cos(ang) ** 2 - 0.04 * math.sin(ang) ** 2))])
        y0 = orc.make_photon(a, r0, th0, 0.0, d)
        iv0 = orc.invariants(a, y0)
        y = np.zeros(8)
        yc = np.ascontiguousarray(y0)
        import ctypes as C

        orc.scalar("integrate", a, yc.ctypes.data_as(C.POINTER(C.c_double)), 0.5, 1e-10, 1e-12, 20000,
                   rh * 1.01, 2000.0, y.ctypes.data_as(C.POINTER(C.c_double)))
        iv = orc.invariants(a, y)
        wn = max(wn, abs(iv[4]))
        wq = max(wq, abs(iv[2] - iv0[2]) / (abs(iv0[2]) + 1e-12))
        we = max(we, abs(iv[0] - iv0[0]) / abs(iv0[0]))
    assert wn < 1e-10
    assert wq < 1e-8
    assert we < 1e-14


def test_page_thorne_closed_form_matches_quadrature(orc):
    """validate.cpp:857-889 (fewer quadrature nodes): relative difference < 1e-6."""
    worst = 0.0
    for a in (0.0, 0.9, 0.998):
        r_isco = orc.scalar("isco_radius", a, 1)
        for r_end in (8.0, 30.0):
            if r_end <= r_isco * 1.2:
                continue
            u = np.linspace(math.sqrt(r_isco), math.sqrt(r_end), 40001)
            r = u * u
            h = 1e-6 * r
            L = lambda x: np.array([orc.scalar("circular_angmom", a, xx, 1) for xx in x])  # noqa: E731
            E = np.array([orc.scalar("circular_energy", a, xx, 1) for xx in r])
            dL = (-L(r + 2 * h) + 8 * L(r + h) - 8 * L(r - h) + L(r - 2 * h)) / (12.0 * h)
            Om = 1.0 / (r * np.sqrt(r) + a)
            f = (E - Om * L(r)) * dL * 2.0 * u
            W = float(np.sum((f[1:] + f[:-1]) * np.diff(u)) / 2.0)
            # trapezoid to Simpson: Richardson on half the nodes
            W2 = float(np.sum((f[2::2] + f[:-2:2]) * np.diff(u[::2])) / 2.0)
            W = (4.0 * W - W2) / 3.0
            closed = orc.scalar("page_thorne_W", a, r_end, r_isco)
            worst = max(worst, abs(W - closed) / abs(closed))
    assert worst < 1e-6


def test_blackbody_table_matches_direct_integration(orc):
    """validate.cpp:1005-1015: table vs exact Y within 2e-3."""
    worst = 0.0
    for lg in np.arange(2.0, 8.0 + 1e-9, 0.13):
        T = 10.0 ** lg
        e = orc.blackbody_xyz_exact(T)
        t = orc.blackbody_xyz(T)
        worst = max(worst, abs(t[1] - e[1]) / max(e[1], 1e-300))
    assert worst < 2e-3


def test_planck_integrates_to_stefan_boltzmann(orc):
    """validate.cpp:958-977: integral of B_lambda = sigma T^4 / pi within 1e-5."""
    worst = 0.0
    for T in (1000.0, 5772.0, 1.0e5, 1.0e7):
        lo, hi, N = math.log(1e-11), math.log(1e-1), 200000
        x = lo + (hi - lo) * (np.arange(N) + 0.5) / N
        lam = np.exp(x)
        total = sum(orc.scalar("planck_radiance", float(l), T) * float(l) for l in lam[::1]) * (hi - lo) / N
        expect = 5.670374419e-8 * T ** 4 / math.pi
        worst = max(worst, abs(total - expect) / expect)
    assert worst < 1e-5


def test_redshift_stop_rule_variant(orc):
    """BH_STOP_RELATIVE stops at r_+ (1 + eps): captured rays end inside the
    reference's stop radius but outside r_+."""
    from cases import kerr_a09_i60

    cfg = kerr_a09_i60(width=64, height=64, stop_mode=abi.STOP_RELATIVE, stop_epsilon=1e-6)
    arr, _ = orc.trace_rays(cfg, 24, 24, 16, 16)
    cap = arr["what"] == abi.HIT_HORIZON
    assert cap.sum() > 0
    rp = orc.scalar("horizon_outer", 0.9)
    r = arr["y"][cap, 1]
    assert (r <= rp * (1 + 1e-6)).all() and (r > rp).all()
