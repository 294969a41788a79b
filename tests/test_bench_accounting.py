"""The bench's bookkeeping on the CPU: the FLOP count per accepted step, the
roofline arithmetic, and the per-ray accuracy report (class flips, g and
direction errors against the target, the conditioning probe's exclusion),
on small synthetic result arrays with known answers."""
import math
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import bench  # noqa: E402
from blackhole_b200 import abi, flops  # noqa: E402


def test_flop_count_per_accepted_step():
    m, d = flops.FLOPS_PER_STEP["mixed"], flops.FLOPS_PER_STEP["fp64"]
    # six right-hand sides, five angle-addition stages, the stage sums, the
    # error estimate, the step control and the diagnostics
    assert m["alu_flop"] == 6 * 62 + 5 * 20 + 271 + 6 * 17 + 5 + 37 == 887
    assert d["alu_flop"] == 6 * 62 + 5 * 34 + 271 + 6 * 17 + 5 + 37 == 957
    assert m["f64_flop"] == 0 and d["f64_flop"] == 0


def test_roofline_arithmetic():
    r = bench.roofline(2.0, 10_000_000, 11_000_000, "mixed", 72.0, "test")
    want = 887 * 10_000_000 / 2e-3 / 1e12
    assert r["achieved"] == pytest.approx(want, rel=1e-3)
    assert r["frac"] == pytest.approx(want / 72.0, rel=1e-3)
    assert r["flop_per_step"] == 887 and r["accepted_steps"] == 10_000_000


def _frame(n):
    a = np.zeros(n, dtype=abi.ray_result_dtype())
    a["what"][: n // 2] = abi.HIT_DISC
    a["g"][: n // 2] = np.linspace(0.5, 1.5, n // 2)
    a["what"][n // 2:] = abi.HIT_SKY
    th = np.linspace(0.1, 3.0, n - n // 2)
    a["dir"][n // 2:] = np.stack([np.sin(th), np.zeros_like(th), np.cos(th)], axis=1)
    return a


def _turn(d, angle):
    """Rotate unit vectors in the x-z plane by `angle`."""
    c, s = math.cos(angle), math.sin(angle)
    return np.stack([c * d[:, 0] + s * d[:, 2], d[:, 1], -s * d[:, 0] + c * d[:, 2]], axis=1)


def test_compare_rays_counts_errors_flips_and_ill_conditioned_rays():
    n = 400
    a = _frame(n)
    b = a.copy()
    disc = np.arange(n // 2)
    sky = np.arange(n // 2, n)
    b["g"][disc[:10]] *= 1.0 + 2e-3              # ten disc rays beyond 1e-3
    b["g"][disc[10:20]] *= 1.0 + 5e-4            # ten within
    b["dir"][sky[:5]] = _turn(a["dir"][sky[:5]], 3e-4)   # five sky rays beyond 1e-4 rad
    b["dir"][sky[5:9]] = _turn(a["dir"][sky[5:9]], 5e-5)
    b["what"][sky[-3:]] = abi.HIT_HORIZON        # three class flips
    out = bench.compare_rays(a, b)
    assert out["rays"] == n and out["class_mismatch"] == 3
    assert out["class_mismatch_pairs"] == {"Sky->Horizon": 3}
    assert out["g_rel"]["n_above_target"] == 10
    assert out["g_rel"]["max"] == pytest.approx(2e-3, rel=1e-6)
    assert out["dir_rad"]["n_above_target"] == 5
    assert out["dir_rad"]["max"] == pytest.approx(3e-4, rel=1e-6)
    assert out["dir_rad"]["n"] == n - n // 2 - 3

    # the probe marks the five far-off sky rays as ill-conditioned: their
    # FP64 result moves by 1e-3 rad under the turn, the others not at all
    probe = a.copy()
    probe["dir"][sky[:5]] = _turn(a["dir"][sky[:5]], 1e-3)
    out = bench.compare_rays(a, b, probe=probe)
    cond = out["dir_rad"]["conditioning"]
    assert cond["ill_conditioned_rays"] == 5
    assert cond["n_above_target_well_conditioned"] == 0
    assert cond["max_well_conditioned"] == pytest.approx(5e-5, rel=1e-6)
    assert cond["their_fp64_move_min"] == pytest.approx(1e-3, rel=1e-6)
    # the disc rays' errors are not excused: their FP64 g does not move
    assert out["g_rel"]["ill_conditioned_rays"] == 0
    assert out["g_rel"]["n_above_target_well_conditioned"] == 10


def test_conditioning_marks_class_changes_as_infinite():
    a = _frame(40)
    probe = a.copy()
    probe["what"][:3] = abi.HIT_SKY
    moved = bench.conditioning(a, probe)
    assert np.isinf(moved[:3]).all()
    assert (moved[3:] == 0).all()
