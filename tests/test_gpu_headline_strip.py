"""The benchmark frame itself against the CPU checkers, per ray.

The timed workload is the 1024x1024 near edge-on frame (a = 0.998,
inclination 85 deg, disc r_isco..50 M at 0.3 Eddington, +-25 M from
r = 1000 M).  These tests trace a 128-row strip through its centre (the
shadow, both disc images and the photon ring) and every 8th row elsewhere
(the sky above and below the disc), 240 rows in all, with the FP64 oracle
(oracle/bh_oracle.c, the restatement pinned bit for bit to the reference) on
the frame's own settings (uniform sky, r_+(1+1e-6) horizon stop), and 16
central rows with every 16th row (79 rows) with the reference itself
(oracle/_ref) on the reference's settings (galactic sky, its horizon stop),
and hold both GPU precisions to them ray by ray:

  * every ray of equal class: the redshift g of a disc ray within 1e-3
    (relative) and the final direction of a sky ray within 1e-4 rad - the
    mixed path's stated accuracy target, and FP64's too - except the rays
    the conditioning probe marks: rays whose FP64 result moves by more than
    1e-5 (rad, or relative in g) when the camera turns by 1.5e-10 rad, i.e.
    whose answer is not determined to the target by binary64 rounding of the
    camera ray itself;
  * the FP64 path besides to rounding in bulk: 99th percentiles of the g and
    direction errors <= 1e-6;
  * rays whose class differs (a ray at the shadow's or the disc's edge that
    an ulp sends the other way) at most a handful per strip, counted.
"""
import copy
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from parity import compare, q, summary  # noqa: E402

from blackhole_b200 import abi, workloads  # noqa: E402

pytestmark = pytest.mark.gpu

G_TOL = 1e-3
DIR_TOL = 1e-4
COND_YAW = 1.5e-10
COND_LIMIT = 1e-5
FP64_BULK = 1e-6
# Rays whose class differs from the checker's, at most, per strip and precision.
MAX_CLASS_MISMATCH = {abi.PRECISION_FP64: 4, abi.PRECISION_MIXED: 8}


def _rows(full, cfg, rows):
    ss = max(1, cfg.sqrt_spp) ** 2
    return full.reshape(cfg.height, cfg.width * ss)[np.asarray(rows)].reshape(-1)


def _moved(fp64, probe):
    """How far each ray's FP64 result moves under the camera turn (inf where
    its class changes): angle for sky rays, relative change of g for disc rays."""
    moved = np.full(len(fp64), np.inf)
    sky = (fp64["what"] == abi.HIT_SKY) & (probe["what"] == abi.HIT_SKY)
    d = np.linalg.norm(probe["dir"][sky] - fp64["dir"][sky], axis=1)
    moved[sky] = 2.0 * np.arcsin(np.clip(d / 2.0, 0.0, 1.0))
    disc = (fp64["what"] == abi.HIT_DISC) & (probe["what"] == abi.HIT_DISC) & (fp64["g"] > 0)
    moved[disc] = np.abs(probe["g"][disc] - fp64["g"][disc]) / fp64["g"][disc]
    return moved


def _strip(renderer, port, cfg, rows):
    """Checker results of the strip, and the GPU's in both precisions with the
    conditioning of each ray (from the FP64 GPU frame and its turned copy)."""
    cd = copy.deepcopy(cfg)
    cd.precision = abi.PRECISION_FP64
    cm = copy.deepcopy(cfg)
    cm.precision = abi.PRECISION_MIXED
    chk, _ = port.trace_rows(cd, rows)
    gpu = {abi.PRECISION_FP64: _rows(renderer.trace_rays(cd), cd, rows),
           abi.PRECISION_MIXED: _rows(renderer.trace_rays(cm), cm, rows)}
    turned = copy.deepcopy(cd)
    turned.cam.yaw += COND_YAW
    moved = _moved(gpu[abi.PRECISION_FP64], _rows(renderer.trace_rays(turned), cd, rows))
    return chk, gpu, moved


def _check(chk, got, moved, precision):
    s = compare(got, chk)
    msg = summary(s)
    same = got["what"] == chk["what"]
    assert (~same).sum() <= MAX_CLASS_MISMATCH[precision], msg
    well = moved <= COND_LIMIT
    disc = same & (chk["what"] == abi.HIT_DISC) & (chk["g"] > 0)
    g_err = np.abs(got["g"] - chk["g"]) / np.where(chk["g"] > 0, chk["g"], 1.0)
    bad_g = disc & well & (g_err > G_TOL)
    assert not bad_g.any(), (f"{bad_g.sum()} well-conditioned disc rays beyond {G_TOL}: "
                             f"max {g_err[bad_g].max():.3e} | {msg}")
    sky = same & (chk["what"] == abi.HIT_SKY)
    ang = 2.0 * np.arcsin(np.clip(np.linalg.norm(got["dir"] - chk["dir"], axis=1) / 2.0, 0.0, 1.0))
    bad_d = sky & well & (ang > DIR_TOL)
    assert not bad_d.any(), (f"{bad_d.sum()} well-conditioned sky rays beyond {DIR_TOL} rad: "
                             f"max {ang[bad_d].max():.3e} | {msg}")
    # the probe excludes few rays: it is not a way around the target
    assert (~well & (disc | sky)).sum() <= 0.002 * len(chk), ((~well & (disc | sky)).sum(), msg)
    if precision == abi.PRECISION_FP64:
        assert q(s["g_rel"], 0.99) <= FP64_BULK, msg
        assert q(s["dir_rad"], 0.99) <= FP64_BULK, msg
    return s


ORACLE_ROWS = sorted(set(range(448, 576)) | set(range(0, 1024, 8)))
REFERENCE_ROWS = sorted(set(range(504, 520)) | set(range(0, 1024, 16)))


@pytest.fixture(scope="module")
def oracle_strip(renderer, orc):
    return _strip(renderer, orc, workloads.edge_on_1024(), ORACLE_ROWS)


@pytest.fixture(scope="module")
def reference_strip(renderer, ref):
    cfg = workloads.edge_on_1024()
    cfg.sky_mode = abi.SKY_GALACTIC
    cfg.stop_mode = abi.STOP_REFERENCE
    return _strip(renderer, ref, cfg, REFERENCE_ROWS)


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_benchmark_frame_strip_against_oracle(oracle_strip, precision):
    chk, gpu, moved = oracle_strip
    assert len(ORACLE_ROWS) == 240 and len(chk) == 240 * 1024
    s = _check(chk, gpu[precision], moved, precision)
    # the rows hold every kind of ray the frame has
    assert len(s["g_rel"]) > 50000 and len(s["dir_rad"]) > 50000
    assert (chk["what"] == abi.HIT_HORIZON).sum() > 1000


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_benchmark_frame_strip_against_reference(reference_strip, precision):
    chk, gpu, moved = reference_strip
    assert len(chk) == len(REFERENCE_ROWS) * 1024
    s = _check(chk, gpu[precision], moved, precision)
    assert len(s["g_rel"]) > 10000 and len(s["dir_rad"]) > 10000
