"""Animation through the batched launch (bh_gpu_render_batch_rgb): the film
of an orbiting hot spot as the reference CLI makes it (main.cpp:931-989) --
exposure metered once on a low-resolution probe of the middle frame, then
locked -- must give, frame by frame, the bytes of the single-frame path with
the same exposure, and the probe's exposure must be the reference meter's
(restated in the oracle) on the probe frame."""
import numpy as np
import pytest

import oracle
from blackhole_b200 import workloads

pytestmark = pytest.mark.gpu


def test_film_frames_equal_single_frames_with_locked_exposure(renderer):
    frames = workloads.hotspot_orbit(frames=6, width=96, height=54)
    probe = workloads.exposure_probe(frames[len(frames) // 2])
    _, e = renderer.render_rgb(probe, meter_only=True)
    assert e == oracle.oracle().auto_exposure(renderer.render(probe))
    film, used = renderer.render_batch_rgb(frames, exposure=e)
    assert used == [e] * len(frames)
    for cfg, rgb in zip(frames, film):
        single, e1 = renderer.render_rgb(cfg, exposure=e)
        assert e1 == e
        assert np.array_equal(rgb, single)
    # the hot spot moves: frames differ, and the film loops (frame 0 != frame n)
    assert not np.array_equal(film[0], film[3])


def test_film_frames_metered_one_by_one(renderer):
    frames = workloads.hotspot_orbit(frames=3, width=64, height=36)
    film, used = renderer.render_batch_rgb(frames)
    o = oracle.oracle()
    for cfg, rgb, e in zip(frames, film, used):
        assert e == o.auto_exposure(renderer.render(cfg))
