"""Jets: the CPU restatement and the library's host set-up against the
reference's own jet code (jet.h:77-315, spectrum.cpp:77-92, render.cpp:44-122,
compiled from its sources into oracle/_ref), bit for bit.

  - Jet::configure (Blandford-Znajek power, emissivity normalisation) as the
    library (bh_jet_configure), the restatement and the reference compute it;
  - the power-law colour, the emissivity shape and the plasma four-velocity
    at points inside, at the edge of and outside the jet;
  - whole rays of the `quasar` and `m87` presets with jets: class, final
    state, jet integral and colour of every sample of a window.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from blackhole_b200 import abi, workloads
from blackhole_b200.gpu import load_library


@pytest.fixture(scope="module")
def ports():
    ref = oracle.reference()
    if ref is None or not ref.has("jet_configure"):
        pytest.skip("the reference sources are not present to build oracle/_ref")
    return oracle.oracle(), ref


PRESETS = [("quasar", workloads.quasar_jets), ("m87", workloads.m87_jets)]


@pytest.mark.parametrize("name,make", PRESETS)
def test_configure_matches_reference(ports, name, make):
    o, r = ports
    cfg = make(32, 18)
    assert cfg.jet_enabled and cfg.jet.j_nu0 > 0.0
    c = cfg.to_c()
    spin, M = cfg.spin, cfg.M_kg
    r_g = 6.67430e-11 * M / (2.99792458e8 * 2.99792458e8)
    mdot_c2 = 1.234e38
    lib = load_library()
    mine = abi.bh_jet.from_buffer_copy(c.jet)
    lib.bh_jet_configure(C.byref(mine), spin, mdot_c2, r_g)
    a = o.jet_configure(c.jet, spin, mdot_c2, r_g)
    b = r.jet_configure(c.jet, spin, mdot_c2, r_g)
    for k in abi.JET_CONFIGURED:
        assert getattr(mine, k) == getattr(b, k) == getattr(a, k), k


def test_powerlaw_colour_matches_reference(ports):
    o, r = ports
    for alpha in (0.7, 0.0, 1.0, -0.5, 2.3):
        assert np.array_equal(o.powerlaw_xyz(alpha), r.powerlaw_xyz(alpha))


@pytest.mark.parametrize("name,make", PRESETS)
def test_shape_and_four_velocity_match_reference(ports, name, make):
    o, r = ports
    cfg = make(32, 18)
    jc = cfg.to_c().jet
    rng = np.random.default_rng(3)
    for _ in range(300):
        z = rng.uniform(-140.0, 140.0)
        rho = abs(rng.normal(0.0, 0.8)) * (1.6 * (max(abs(z), 1e-6) / 3.0) ** 0.58)
        assert o.jet_shape(jc, z, rho) == r.jet_shape(jc, z, rho)
        rr = rng.uniform(1.5, 150.0)
        th = rng.uniform(0.01, np.pi - 0.01)
        assert np.array_equal(o.jet_four_velocity(jc, cfg.spin, rr, th),
                              r.jet_four_velocity(jc, cfg.spin, rr, th))


@pytest.mark.parametrize("name,make,window", [("quasar", workloads.quasar_jets, (150, 40, 20, 12)),
                                              ("m87", workloads.m87_jets, (150, 60, 20, 12))])
def test_jet_rays_match_reference(ports, name, make, window):
    o, r = ports
    cfg = make(320, 180)
    cfg.star_count = 20000
    x0, y0, w, h = window
    a, _ = o.trace_rays(cfg, x0, y0, w, h)
    b, _ = r.trace_rays(cfg, x0, y0, w, h)
    assert (b["jet"] > 0).any(), "the window must see the jet"
    for f in ("what", "steps", "y", "jet", "xyz", "g", "dir"):
        assert np.array_equal(a[f], b[f]), f
