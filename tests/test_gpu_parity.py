"""GPU render path against the reference: per-sample parity through the C-ABI.

The checker is the reference renderer itself (golden vectors made from it by
tests/golden/make_golden.py) and, for the settings the reference does not
have (uniform sky, relative horizon stop), the CPU oracle.

Tolerances.  The FP64 path evaluates the same Hamiltonian system as the
reference in a different but algebraically identical form, with CUDA's libm
and FMA contraction, so results agree to rounding except where a rounding
difference flips an accept/reject decision or a class (shadow edge, disc
edge, photon ring).  Measured on every golden window: no ray in another
class, g and direction within 2e-11 (relative, rad), luminance within
1.2e-6.  Held: at most MAX_CLASS_FLIPS rays of another class per window;
among rays of equal class every g and direction within FP64_MAX and the
99th percentiles of g, direction and luminance within 1e-6, medians within
1e-9.  The mixed path is held to the stated accuracy target on every ray
of equal class: g within 1e-3, direction within 1e-4 rad, the jet integral
within 1e-3 (measured maxima 2.4e-5, 1.3e-5 rad, 2.5e-4), with the same
bound on class flips.
"""
import math
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)

from cases import CASES, RENDER_CASE, kerr_a09_i60  # noqa: E402
from parity import compare, q, summary, window_of  # noqa: E402

from blackhole_b200 import BHError, RenderConfig, RenderStats, abi  # noqa: E402

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-6
FP64_MAX = 1e-7
MIXED_G_TOL = 1e-3
MIXED_DIR_TOL = 1e-4
# Rays of another class than the checker's, at most, per golden window.
MAX_CLASS_FLIPS = 2


def _golden(name):
    return np.load(os.path.join(HERE, "golden", f"{name}.npz"))


def _gpu_window(renderer, cfg, window):
    x0, y0, w, h = window
    full = renderer.trace_rays(cfg)
    return window_of(full, cfg.width, cfg.height, max(1, cfg.sqrt_spp), x0, y0, w, h)


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_matches_reference_golden(renderer, name):
    make, window = CASES[name]
    cfg = make()
    cfg.precision = abi.PRECISION_FP64
    gw = _gpu_window(renderer, cfg, window)
    s = compare(gw, _golden(name))
    msg = summary(s)
    print(name, msg)
    assert round((1 - s["class_agree"]) * s["n"]) <= MAX_CLASS_FLIPS, msg
    assert s["jet_missing"] <= MAX_CLASS_FLIPS, msg
    for k in ("g_rel", "dir_rad", "Y_rel", "jet_rel"):
        assert q(s[k], 0.99) <= FP64_TOL, f"{k}: {msg}"
        # most rays reproduce the reference to rounding
        if len(s[k]) >= 20:
            assert q(s[k], 0.5) <= 1e-9, f"{k}: {msg}"
    for k in ("g_rel", "dir_rad"):
        if len(s[k]):
            assert s[k].max() <= FP64_MAX, f"{k}: {msg}"


@pytest.mark.parametrize("name", ["a09_i60_centre", "a09_i60_corner", "a0998_i85_ring", "quasar_jets", "m87_jets"])
def test_mixed_meets_accuracy_target_against_reference(renderer, name):
    make, window = CASES[name]
    cfg = make()
    cfg.precision = abi.PRECISION_MIXED
    gw = _gpu_window(renderer, cfg, window)
    s = compare(gw, _golden(name))
    msg = summary(s)
    print(name, "mixed", msg)
    assert round((1 - s["class_agree"]) * s["n"]) <= MAX_CLASS_FLIPS, msg
    # every ray of equal class within the target
    for k, tol in (("g_rel", MIXED_G_TOL), ("dir_rad", MIXED_DIR_TOL), ("jet_rel", MIXED_G_TOL)):
        v = s[k]
        if len(v):
            assert v.max() <= tol, f"{k}: {msg}"


def test_fp64_frame_pixels_match_reference_render(renderer):
    name, make = RENDER_CASE
    g = _golden(name)
    cfg = make()
    st = RenderStats()
    px = renderer.render(cfg, st)
    ref = g["pixels"]
    lit = ref[..., 1] > 0
    rel = np.abs(px[..., 1][lit] - ref[..., 1][lit]) / ref[..., 1][lit]
    assert q(rel, 0.95) <= FP64_TOL, q(rel, 0.95)
    assert (px[~lit] == 0).mean() > 0.95
    r = g["stats"]
    assert st.rays == r[0]
    # class counts agree to within the boundary rays
    for got, want in zip([st.captured, st.disc_hits, st.escaped], [r[2], r[3], r[6]]):
        assert abs(got - want) <= max(3, 0.02 * r[0])
    assert abs(st.steps - r[1]) / r[1] < 0.02
    assert st.max_norm_error < 1e-6 and st.max_carter_drift < 1e-4


@pytest.mark.parametrize("sky_mode,stop_mode", [(abi.SKY_UNIFORM, abi.STOP_RELATIVE),
                                                 (abi.SKY_GALACTIC, abi.STOP_RELATIVE),
                                                 (abi.SKY_UNIFORM, abi.STOP_REFERENCE)])
def test_fp64_matches_oracle_on_extension_settings(renderer, orc, sky_mode, stop_mode):
    cfg = kerr_a09_i60(width=96, height=96, sky_mode=sky_mode, stop_mode=stop_mode, stop_epsilon=1e-6)
    window = (30, 30, 36, 36)
    chk, _ = orc.trace_rays(cfg, *window)
    gw = _gpu_window(renderer, cfg, window)
    s = compare(gw, chk)
    msg = summary(s)
    assert s["class_agree"] >= 0.98, msg
    assert s["jet_missing"] <= 0.01 * s["n"], msg
    for k in ("g_rel", "dir_rad", "Y_rel", "jet_rel"):
        assert q(s[k], 0.99) <= FP64_TOL, f"{k}: {msg}"


def test_fp64_sky_window_matches_oracle(renderer, orc):
    """Escaped rays only: star lookups and the diffuse background."""
    cfg = kerr_a09_i60(width=200, height=200, sky_mode=abi.SKY_UNIFORM)
    window = (0, 0, 40, 40)
    chk, _ = orc.trace_rays(cfg, *window)
    gw = _gpu_window(renderer, cfg, window)
    s = compare(gw, chk)
    assert s["class_agree"] == 1.0
    assert q(s["Y_rel"], 0.99) <= FP64_TOL, summary(s)


# ---- edge cases --------------------------------------------------------------

@pytest.mark.parametrize("w,h,spp", [(1, 1, 1), (37, 23, 3), (5, 9, 2), (64, 1, 1), (1, 50, 1)])
def test_ragged_sizes_match_oracle(renderer, orc, w, h, spp):
    cfg = kerr_a09_i60(width=w, height=h, sqrt_spp=spp)
    cfg.cam.fov = 2.0 * math.atan(12.0 / 1000.0)
    chk, cst = orc.trace_rays(cfg)
    st = RenderStats()
    gpu = renderer.trace_rays(cfg, st)
    assert len(gpu) == w * h * spp * spp
    s = compare(gpu, chk)
    assert s["class_agree"] >= 0.97, summary(s)
    assert st.rays == cst.rays
    px = renderer.render(cfg)
    opx, _ = orc.render_window(cfg)
    lit = opx[..., 1] > 0
    if lit.any():
        rel = np.abs(px[..., 1][lit] - opx[..., 1][lit]) / opx[..., 1][lit]
        assert q(rel, 0.9) <= FP64_TOL


def test_zero_and_tiny_step_budgets_exhaust(renderer, orc):
    cfg = kerr_a09_i60(width=8, height=8, max_steps=0)
    g = renderer.trace_rays(cfg)
    assert (g["what"] == abi.HIT_EXHAUSTED).all() and (g["steps"] == 0).all()
    cfg = kerr_a09_i60(width=8, height=8, max_steps=3)
    g = renderer.trace_rays(cfg)
    o, _ = orc.trace_rays(cfg)
    assert (g["what"] == o["what"]).all()
    assert (g["what"] == abi.HIT_EXHAUSTED).all() and (g["steps"] == 3).all()
    # Far from the hole the embedded error estimate is a 1e-10 cancellation of
    # the stages, so the separated-form RHS changes the step-size choice at
    # the 1e-6 level: states agree to that, not to rounding.
    assert np.allclose(g["y"], o["y"], rtol=1e-5, atol=1e-10), np.abs(g["y"] - o["y"]).max(axis=0)


def test_content_switches(renderer, orc):
    for kw in ({"disc_enabled": False}, {"stars_enabled": False}, {"milky_way": False},
               {"star_count": 0}, {"disc_sense": -1}):
        cfg = kerr_a09_i60(width=48, height=48, **kw)
        chk, _ = orc.trace_rays(cfg, 8, 8, 32, 32)
        gw = _gpu_window(renderer, cfg, (8, 8, 32, 32))
        s = compare(gw, chk)
        assert s["class_agree"] >= 0.98, (kw, summary(s))
        assert q(s["Y_rel"], 0.99) <= FP64_TOL, (kw, summary(s))


def test_invalid_configs_are_rejected(renderer):
    bad = [
        dict(width=0), dict(height=-3), dict(precision=7),
        dict(sky_mode=9), dict(stop_mode=5), dict(rtol=-1.0), dict(star_count=-1),
    ]
    for kw in bad:
        cfg = kerr_a09_i60(width=8, height=8)
        for k, v in kw.items():
            setattr(cfg, k, v)
        with pytest.raises(BHError) as e:
            renderer.render(cfg)
        assert e.value.code in (abi.ERR_INVALID_ARG, abi.ERR_UNSUPPORTED), kw
    c = kerr_a09_i60(width=8, height=8).to_c()
    c.struct_size = 12
    with pytest.raises(BHError):
        renderer.render(c)
    # the context stays usable
    renderer.render(kerr_a09_i60(width=8, height=8))


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_deterministic_and_independent_of_launch_shape(renderer, precision):
    """Each ray's arithmetic does not depend on which lane, warp or launch
    shape traces it: within one compiled kernel (register cap) frames are
    bitwise identical across block sizes, refill thresholds and rays per
    thread.  The two register caps are two compilations, whose mul+add
    fusion may differ: they agree to the parity tolerance."""
    cfg = kerr_a09_i60(width=64, height=48, sqrt_spp=2, precision=precision)
    old = renderer.get_launch(precision)
    # pixel luminance: the blackbody Y of g T moves like g^3..g^5 in the
    # visible tail, so the mixed path's 1e-3 in g is up to ~1e-2 in Y
    tol = FP64_TOL if precision == abi.PRECISION_FP64 else 10 * MIXED_G_TOL
    try:
        frames = {}
        for rv in (1, 2):
            renderer.set_launch(block_size=128, rays_per_thread=1, refill=32, reg_variant=rv, precision=precision)
            a = renderer.render(cfg)
            assert np.array_equal(a, renderer.render(cfg))
            for bs, rpt, refill in ((64, 1, 1), (256, 2, 32), (96, 4, 8)):
                renderer.set_launch(block_size=bs, rays_per_thread=rpt, refill=refill, precision=precision)
                assert np.array_equal(renderer.render(cfg), a), (rv, bs, rpt, refill)
            frames[rv] = a
        lit = frames[1][..., 1] > 0
        rel = np.abs(frames[1][..., 1][lit] - frames[2][..., 1][lit]) / frames[1][..., 1][lit]
        assert q(rel, 0.99) <= tol
    finally:
        renderer.set_launch(precision=precision, **{k: v for k, v in old.items()})


def test_autotune_keeps_results_and_picks_a_shape(renderer):
    cfg = kerr_a09_i60(width=48, height=48, precision=abi.PRECISION_MIXED)
    a = renderer.render(cfg)
    old = renderer.get_launch(abi.PRECISION_MIXED)
    try:
        best, ms = renderer.autotune(cfg)
        assert ms > 0 and best["block_size"] in (64, 128, 256, 512)
        assert renderer.get_launch(abi.PRECISION_MIXED) == best
        b = renderer.render(cfg)
        if best["reg_variant"] == old["reg_variant"]:
            assert np.array_equal(b, a)
        else:
            # the other register cap is another compilation (its mul+add
            # fusion may differ): the same frame to the parity tolerance
            lit = a[..., 1] > 0
            rel = np.abs(b[..., 1][lit] - a[..., 1][lit]) / a[..., 1][lit]
            assert q(rel, 0.99) <= 10 * MIXED_G_TOL
    finally:
        renderer.set_launch(precision=abi.PRECISION_MIXED, **{k: v for k, v in old.items()})


def test_autotune_batch_picks_a_shape_in_the_search_space(renderer):
    cfgs = [kerr_a09_i60(width=40, height=24, precision=abi.PRECISION_MIXED),
            kerr_a09_i60(width=24, height=40, spin=0.5, precision=abi.PRECISION_MIXED)]
    before = renderer.render_batch(cfgs)
    old = renderer.get_launch(abi.PRECISION_MIXED)
    try:
        best, ms = renderer.autotune_batch(cfgs)
        assert ms > 0
        assert best["block_size"] in (64, 128, 256, 512) and best["rays_per_thread"] in (1, 2, 4, 8)
        assert best["refill"] in (8, 16, 24, 32) and best["reg_variant"] in (1, 2)
        assert renderer.get_launch(abi.PRECISION_MIXED) == best
        for a, b in zip(before, renderer.render_batch(cfgs)):
            lit = a[..., 1] > 0
            rel = np.abs(a[..., 1][lit] - b[..., 1][lit]) / a[..., 1][lit]
            assert q(rel, 0.99) <= 1e-2      # the two register caps are two compilations
    finally:
        renderer.set_launch(precision=abi.PRECISION_MIXED, **{k: v for k, v in old.items()})


def test_stats_accumulate_like_reference(renderer):
    cfg = kerr_a09_i60(width=32, height=32)
    st = RenderStats()
    renderer.render(cfg, st)
    first = (st.rays, st.steps, st.captured + st.disc_hits + st.escaped + st.exhausted)
    renderer.render(cfg, st)
    assert st.rays == 2 * first[0] and st.steps == 2 * first[1]
    assert first[2] == first[0]
    assert st.seconds > 0 and st.kernel_ms > 0


def test_batch_equals_single_frames(renderer):
    cfgs = [kerr_a09_i60(width=40, height=24), kerr_a09_i60(width=17, height=31, spin=0.5),
            kerr_a09_i60(width=64, height=64, sqrt_spp=2)]
    cfgs[1].cam.theta = math.radians(80.0)
    stats = []
    outs = renderer.render_batch(cfgs, stats)
    for c, o, s in zip(cfgs, outs, stats):
        single = RenderStats()
        assert np.array_equal(o, renderer.render(c, single))
        assert s.rays == single.rays and s.steps == single.steps
        assert s.disc_hits == single.disc_hits
    # into caller-owned arrays, reused: the same frames, every call
    mine = [np.full((c.height, c.width, 3), np.nan) for c in cfgs]
    for _ in range(2):
        got = renderer.render_batch(cfgs, outs=mine)
        assert all(g is m for g, m in zip(got, mine))
        assert all(np.array_equal(m, o) for m, o in zip(mine, outs))
    with pytest.raises(ValueError):
        renderer.render_batch(cfgs, outs=mine[:2])


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_batch_graph_replay_follows_new_frame_constants(renderer, precision):
    """The batch graph is captured once per shape; a second batch of the same
    shape with other cameras and spins replays it and must still match the
    single-frame renders, and a change of shape recaptures."""
    def batch(spin, incl):
        cfgs = [kerr_a09_i60(width=32, height=24, spin=spin), kerr_a09_i60(width=24, height=32, spin=spin)]
        for c in cfgs:
            c.cam.theta = math.radians(incl)
            c.precision = precision
        return cfgs

    for cfgs in (batch(0.9, 60.0), batch(0.5, 75.0), batch(0.99, 85.0)):
        outs = renderer.render_batch(cfgs)
        for c, o in zip(cfgs, outs):
            assert np.array_equal(o, renderer.render(c))
    grown = batch(0.7, 70.0) + [kerr_a09_i60(width=16, height=16, spin=0.7)]
    grown[-1].precision = precision
    outs = renderer.render_batch(grown)
    for c, o in zip(grown, outs):
        assert np.array_equal(o, renderer.render(c))


def test_batch_rejects_mixed_catalogues(renderer):
    a = kerr_a09_i60(width=8, height=8)
    b = kerr_a09_i60(width=8, height=8, seed=5)
    with pytest.raises(BHError):
        renderer.render_batch([a, b])


def test_step_budget_returns_budget_error(renderer):
    cfg = kerr_a09_i60(width=64, height=64)
    renderer.set_step_budget(2000)
    try:
        with pytest.raises(BHError) as e:
            renderer.render(cfg)
        assert e.value.code == abi.ERR_BUDGET
    finally:
        renderer.set_step_budget(0)
    renderer.render(cfg)


@pytest.mark.parametrize("stop", ["budget", "abort"])
def test_banded_render_ends_when_the_launch_stops_early(renderer, stop):
    """A frame of 128 rows or more goes through the row-band pipeline; when a
    step budget or an abort stops the trace before every band's rays are
    done, the band waits still end (each counter is raised to its band's size
    after the trace kernels) and the call returns the launch's status."""
    cfg = kerr_a09_i60(width=160, height=192)
    if stop == "budget":
        renderer.set_step_budget(5000)
    else:
        renderer.request_abort()
    try:
        with pytest.raises(BHError) as e:
            renderer.render(cfg)
        assert e.value.code == (abi.ERR_BUDGET if stop == "budget" else abi.ERR_ABORTED)
    finally:
        renderer.set_step_budget(0)
        renderer.clear_abort()
    assert np.isfinite(renderer.render(cfg)).all()


def test_abort_flag_stops_the_launch(renderer):
    cfg = kerr_a09_i60(width=64, height=64)
    renderer.request_abort()
    try:
        with pytest.raises(BHError) as e:
            renderer.render(cfg)
        assert e.value.code == abi.ERR_ABORTED
    finally:
        renderer.clear_abort()
    renderer.render(cfg)


def test_device_output_matches_host_output(renderer):
    torch = pytest.importorskip("torch")
    cfg = kerr_a09_i60(width=48, height=40)
    host = renderer.render(cfg)
    dev = torch.empty((40, 48, 3), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    renderer.render_device(cfg, dev.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    assert np.array_equal(dev.cpu().numpy(), host)


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_banded_render_equals_the_device_path(renderer, precision):
    """bh_gpu_render shades and copies a frame of 128 rows or more band by
    band while it is traced (rows 64 at a time, each started when the trace
    has counted all its rays): the same pixels and stats as the device path,
    which shades the whole frame after the trace; ragged last band."""
    torch = pytest.importorskip("torch")
    cfg = kerr_a09_i60(width=200, height=150, sqrt_spp=2, precision=precision)
    host = np.full((150, 200, 3), np.nan)
    sh = abi.bh_render_stats()
    renderer.render_into(cfg, host, sh)
    dev = torch.empty((150, 200, 3), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    sd = abi.bh_render_stats()
    renderer.render_device(cfg, dev.data_ptr(), stream.cuda_stream, stats=sd)
    stream.synchronize()
    assert np.array_equal(dev.cpu().numpy(), host)
    for f in ("rays", "steps", "attempts", "captured", "disc_hits", "escaped", "total_flux"):
        assert getattr(sh, f) == getattr(sd, f), f
    assert np.array_equal(renderer.render(cfg), host)


def test_invariant_diagnostics_of_a_full_frame(renderer):
    """Null-norm and Carter drift stay at the integration tolerance."""
    cfg = kerr_a09_i60(width=128, height=128)
    st = RenderStats()
    renderer.render(cfg, st)
    assert 0 < st.max_norm_error < 1e-6
    assert 0 < st.max_carter_drift < 1e-4
    cfg.precision = abi.PRECISION_MIXED
    sm = RenderStats()
    renderer.render(cfg, sm)
    assert sm.max_norm_error < 1e-2 and sm.max_carter_drift < 1e-1
