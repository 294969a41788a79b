"""The mixed-precision path's step limiter and early capture (bh_gpu.h:
BH_STEP_LIMIT_*, BH_CAPTURE_*).

  * without the reference's step cap (the AUTO default for a scene of disc and
    sky) the mixed frame needs fewer than half the steps and stays within the
    accuracy target against the binary64 frame (g <= 1e-3 relative, final
    direction <= 1e-4 rad, class agreement >= 99.9 %); AUTO equals NONE bit
    for bit there, and equals REFERENCE bit for bit once the Sun, a neutron
    star or a jet is in the scene (and, with a neutron star or a jet, no
    captured ray is ended early);
  * ending ingoing rays inside the innermost photon orbit as captured (the
    AUTO default) changes no ray's class and no pixel: every such ray ends
    on the horizon when traced on;
  * the binary64 path ignores both knobs;
  * near-critical rays (their radial potential's minimum just below zero:
    they circle close to the photon shell before escaping) are the binary64
    frame's rays bit for bit under BH_NEAR_CRITICAL_AUTO, and no other ray
    is (BH_NEAR_CRITICAL_BINARY32 leaves all of them in binary32);
  * unknown values are refused.
"""
import copy
import os
import sys

import numpy as np
import pytest

from blackhole_b200 import abi
from blackhole_b200.gpu import BHError

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))


def _edge_on(n=256, **kw):
    from cases import edge_on_a0998

    cfg = edge_on_a0998(n, n, stop_mode=abi.STOP_RELATIVE, stop_epsilon=1e-6)
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def _with(cfg, **kw):
    c = copy.deepcopy(cfg)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _errors(a, b):
    """Class agreement and the g / direction errors of a against b."""
    same = a["what"] == b["what"]
    disc = same & (b["what"] == abi.HIT_DISC)
    sky = same & (b["what"] == abi.HIT_SKY)
    g = np.abs(a["g"][disc] - b["g"][disc]) / np.abs(b["g"][disc])
    d = np.arccos(np.clip(np.sum(a["dir"][sky] * b["dir"][sky], axis=1), -1.0, 1.0))
    return same.mean(), g, d


def test_no_step_cap_halves_the_steps_within_the_accuracy_target(renderer):
    """Without the reference's cap (AUTO: the loose cap h <= 0.3 max(1, r - r_+);
    NONE: the error control alone) fewer than half the reference cap's steps,
    AUTO with fewer attempts than NONE, all within the target."""
    base = _edge_on(precision=abi.PRECISION_MIXED)
    fp64 = renderer.trace_rays(_with(base, precision=abi.PRECISION_FP64))
    auto = renderer.trace_rays(base)
    none = renderer.trace_rays(_with(base, mixed_step_limit=abi.STEP_LIMIT_NONE))
    capped = renderer.trace_rays(_with(base, mixed_step_limit=abi.STEP_LIMIT_REFERENCE))
    assert auto["steps"].mean() < 0.5 * capped["steps"].mean()
    assert none["steps"].mean() < 0.5 * capped["steps"].mean()
    assert auto["attempts"].mean() < none["attempts"].mean()
    for run in (auto, none, capped):
        agree, g, d = _errors(run, fp64)
        assert agree >= 0.999
        assert g.max() <= 1e-3 and d.max() <= 1e-4, (g.max(), d.max())


@pytest.mark.parametrize("content", ["sun", "jet", "star"])
def test_step_cap_stays_where_an_event_samples_within_a_step(renderer, content):
    from cases import neutron_star, sun_hotspot_spp2

    if content == "sun":
        cfg = sun_hotspot_spp2()
    elif content == "star":
        cfg = neutron_star()
    else:
        from blackhole_b200 import workloads

        cfg = workloads.quasar_jets(96, 54, abi.PRECISION_MIXED)
    cfg.precision = abi.PRECISION_MIXED
    auto = renderer.trace_rays(cfg)
    capped = renderer.trace_rays(_with(cfg, mixed_step_limit=abi.STEP_LIMIT_REFERENCE))
    assert np.array_equal(auto["y"], capped["y"]) and np.array_equal(auto["what"], capped["what"])
    if content != "sun":
        # a surface or an emission on the way in: captured rays are traced on
        traced = renderer.trace_rays(_with(cfg, mixed_capture=abi.CAPTURE_REFERENCE))
        assert np.array_equal(auto["y"], traced["y"])


def test_early_capture_changes_no_class_and_no_pixel(renderer):
    base = _edge_on(precision=abi.PRECISION_MIXED)
    early = renderer.trace_rays(base)
    traced = renderer.trace_rays(_with(base, mixed_capture=abi.CAPTURE_REFERENCE))
    assert np.array_equal(early["what"], traced["what"])
    assert (early["what"] == abi.HIT_HORIZON).sum() > 100
    assert np.array_equal(renderer.render(base), renderer.render(_with(base, mixed_capture=abi.CAPTURE_REFERENCE)))
    cap = early["what"] == abi.HIT_HORIZON
    assert early["steps"][cap].sum() < traced["steps"][cap].sum()


def test_binary64_path_ignores_the_mixed_knobs(renderer):
    base = _edge_on(96, precision=abi.PRECISION_FP64)
    a = renderer.trace_rays(base)
    b = renderer.trace_rays(_with(base, mixed_step_limit=abi.STEP_LIMIT_NONE, mixed_capture=abi.CAPTURE_AUTO))
    c = renderer.trace_rays(_with(base, mixed_step_limit=abi.STEP_LIMIT_REFERENCE,
                                  mixed_capture=abi.CAPTURE_REFERENCE))
    assert np.array_equal(a["y"], b["y"]) and np.array_equal(a["y"], c["y"])


@pytest.mark.parametrize("knob,value", [("mixed_step_limit", 3), ("mixed_step_limit", -1),
                                        ("mixed_capture", 2), ("mixed_near_critical", 2)])
def test_unknown_knob_values_are_refused(renderer, knob, value):
    cfg = _edge_on(16, precision=abi.PRECISION_MIXED)
    setattr(cfg, knob, value)
    with pytest.raises(BHError) as e:
        renderer.render(cfg)
    assert e.value.code == abi.ERR_INVALID_ARG


def _near_critical(cfg, fp64):
    """The near-critical rule restated on the binary64 frame's constants of
    motion (E, L_z from p_t, p_phi; Q from th, p_th at the end of the ray):
    the minimum of R(r) / r^4 at the largest root of R' in (-0.1, 0), for rays
    that start moving inwards from outside that root."""
    y = fp64["y"]
    a = cfg.spin
    E, Lz, th, pth = -y[:, 4], y[:, 7], y[:, 2], y[:, 6]
    b = Lz / E
    q = (pth ** 2 + np.cos(th) ** 2 * (-(a * a) * E * E + Lz ** 2 / np.sin(th) ** 2)) / E ** 2
    c2 = a * a - b * b - q
    c1 = 2.0 * (q + (b - a) ** 2)
    r = np.sqrt(np.maximum(-c2, 0.0))
    for _ in range(60):
        r = r - (4 * r ** 3 + 2 * c2 * r + c1) / np.where(12 * r ** 2 + 2 * c2 > 0, 12 * r ** 2 + 2 * c2, 1.0)
    Rn = (r ** 4 + c2 * r ** 2 + c1 * r - a * a * q) / r ** 4
    r_plus = 1.0 + np.sqrt(1.0 - a * a)
    return (c2 < 0) & (r > r_plus) & (Rn < 0) & (Rn > -0.1)


def test_near_critical_rays_are_the_binary64_frames(renderer):
    cfg = _edge_on(192, precision=abi.PRECISION_FP64, stop_mode=abi.STOP_REFERENCE)
    fp64 = renderer.trace_rays(cfg)
    auto = renderer.trace_rays(_with(cfg, precision=abi.PRECISION_MIXED))
    b32 = renderer.trace_rays(_with(cfg, precision=abi.PRECISION_MIXED,
                                    mixed_near_critical=abi.NEAR_CRITICAL_BINARY32))
    same = np.all(auto["y"] == fp64["y"], axis=1) & (auto["steps"] == fp64["steps"])
    nc = _near_critical(cfg, fp64)     # most of them end on the disc after their orbit
    # the restated rule reads Q at the end of the ray (conserved to ~1e-9):
    # rays within that of the bound may fall on either side
    assert nc.sum() >= 50, nc.sum()
    assert same[nc].mean() >= 0.99, same[nc].mean()
    # every ray the binary64 kernel took is near-critical (or a ray whose
    # binary32 and binary64 integrations agree to the last bit, which a
    # frame of this size does not have)
    assert (same & ~nc).sum() <= 0.01 * nc.sum() + 2, (same & ~nc).sum()
    # under BINARY32 the near-critical rays are integrated in binary32
    assert not np.all(b32["y"][nc] == fp64["y"][nc])
    # classes and pixels of everything else are those of BINARY32
    assert np.array_equal(auto["what"][~nc & ~same], b32["what"][~nc & ~same])
