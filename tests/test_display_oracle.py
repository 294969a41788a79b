"""The display transform's CPU restatement (oracle/bh_oracle.c) against the
reference's own img::auto_exposure, img::add_glare and img::develop
(image.cpp:22-191, compiled from the reference's sources into oracle/_ref):
byte-for-byte on images that hold every tone curve's range, negative and
out-of-gamut colours, non-finite values and empty frames."""
import numpy as np
import pytest

import oracle
from blackhole_b200 import abi


def _images():
    rng = np.random.default_rng(11)
    a = np.exp(rng.normal(0.0, 6.0, size=(37, 53, 3))) * 1e-3
    a[3, 4] = [-1.0, 2.0, np.inf]
    a[5, 6] = [np.nan, 1.0, 1.0]
    a[7, 8] = [1e-9, -1e-3, 1e-9]
    b = np.abs(rng.normal(0.0, 1.0, size=(16, 16, 3)))
    b[:, :, 1] *= 1e9                       # a disc-bright frame
    c = np.zeros((8, 9, 3))                 # nothing to meter
    d = rng.uniform(-0.5, 2.0, size=(64, 3, 3))
    return [a, b, c, d]


@pytest.fixture(scope="module")
def ports():
    ref = oracle.reference()
    if ref is None or not ref.has("develop"):
        pytest.skip("the reference sources are not present to build oracle/_ref")
    return oracle.oracle(), ref


def test_auto_exposure_matches_reference(ports):
    o, r = ports
    for img in _images():
        for key in (1.0, 0.5):
            assert o.auto_exposure(img, key) == r.auto_exposure(img, key)


@pytest.mark.parametrize("strength,radius", [(0.3, 2.0), (0.05, 0.7), (1.0, 5.0)])
def test_add_glare_matches_reference(ports, strength, radius):
    o, r = ports
    for img in _images():
        assert np.array_equal(o.add_glare(img, strength, radius), r.add_glare(img, strength, radius),
                              equal_nan=True)


@pytest.mark.parametrize("tm", range(5))
def test_develop_matches_reference(ports, tm):
    o, r = ports
    for img in _images():
        e = r.auto_exposure(img)
        for decades in (16.0, 6.0, 0.5, 30.0):
            assert np.array_equal(o.develop(img, e, tm, decades), r.develop(img, e, tm, decades))
