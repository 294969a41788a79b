"""The display transform on the GPU (bh_gpu_develop, bh_gpu_render_rgb)
against the CPU restatement, which tests/test_display_oracle.py pins byte for
byte to the reference's img:: functions.  The metered exposure must be the
same binary64 number; the 8-bit image the same bytes, except where the
device's pow/log10/tanh and the host libm differ in the last bit exactly at a
rounding boundary of 255 v (tolerated: at most 1 in 10^4 bytes, off by 1)."""
import os
import sys

import numpy as np
import pytest

import oracle
from blackhole_b200 import abi
from blackhole_b200.gpu import BHError

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from cases import kerr_a09_i60  # noqa: E402

pytestmark = pytest.mark.gpu


def _same_bytes(a, b):
    d = np.abs(a.astype(np.int16) - b.astype(np.int16))
    assert d.max() <= 1 and (d > 0).mean() <= 1e-4, (int(d.max()), float((d > 0).mean()))


def _images():
    rng = np.random.default_rng(5)
    a = np.exp(rng.normal(0.0, 6.0, size=(123, 77, 3))) * 1e-3
    a[3, 4] = [-1.0, 2.0, np.inf]
    a[5, 6] = [np.nan, 1.0, 1.0]
    big = np.exp(rng.normal(0.0, 4.0, size=(512, 768, 3)))
    flat = np.full((40, 40, 3), 0.25)       # every luminance ties
    empty = np.zeros((9, 8, 3))
    return [a, big, flat, empty]


@pytest.mark.parametrize("tm", range(5))
def test_develop_matches_oracle(renderer, tm):
    o = oracle.oracle()
    for img in _images():
        rgb, e = renderer.develop(img, tonemap=tm)
        assert e == o.auto_exposure(img)
        _same_bytes(rgb, o.develop(img, e, tm, 16.0))


def test_glare_then_develop_matches_oracle(renderer):
    o = oracle.oracle()
    for img in _images()[:2]:
        for strength, radius in ((0.3, 3.0), (0.8, 1.2)):
            rgb, e = renderer.develop(img, glare=strength, glare_radius=radius, tonemap=abi.TONEMAP_ACES)
            g = o.add_glare(img, strength, radius)
            assert e == o.auto_exposure(g)
            _same_bytes(rgb, o.develop(g, e, abi.TONEMAP_ACES, 16.0))


def test_fixed_exposure_and_meter_only(renderer):
    o = oracle.oracle()
    img = _images()[0]
    rgb, e = renderer.develop(img, exposure=123.5, tonemap=abi.TONEMAP_REINHARD)
    assert e == 123.5
    _same_bytes(rgb, o.develop(img, 123.5, abi.TONEMAP_REINHARD, 16.0))
    none, e2 = renderer.develop(img, meter_only=True)
    assert none is None and e2 == o.auto_exposure(img)


def test_render_rgb_is_render_then_develop(renderer):
    o = oracle.oracle()
    cfg = kerr_a09_i60(width=96, height=64)
    xyz = renderer.render(cfg)
    for kw in ({}, {"glare": 0.2, "glare_radius": 2.0}, {"tonemap": "log", "log_decades": 8.0}):
        rgb, e = renderer.render_rgb(cfg, **kw)
        ref_img = o.add_glare(xyz, kw["glare"], kw["glare_radius"]) if "glare" in kw else xyz
        assert e == o.auto_exposure(ref_img)
        tm = abi.TONEMAP_NAMES.index(kw.get("tonemap", "hdr"))
        _same_bytes(rgb, o.develop(ref_img, e, tm, kw.get("log_decades", 16.0)))


def test_bad_display_settings_are_refused(renderer):
    img = np.ones((4, 4, 3))
    with pytest.raises(BHError):
        renderer.develop(img, tonemap=7)
    with pytest.raises(BHError):
        renderer.develop(img, glare=1.5)
