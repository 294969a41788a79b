"""Parity cases shared by the golden generator and the tests.

Every case is a RenderConfig plus a pixel window.  Only the reference's own
rules (BH_SKY_GALACTIC, BH_STOP_REFERENCE) appear here, because the golden
vectors come from the reference renderer itself.  The jet cases are the
reference CLI's `quasar` and `m87` presets with their jets configured as the
CLI does it.
"""
import math

from blackhole_b200 import abi, workloads
from blackhole_b200.config import M_SUN, Camera, HotSpot, NeutronStar, RenderConfig, SunBody


def _fov(half, r=1000.0):
    return 2.0 * math.atan(half / r)


def kerr_a09_i60(width=256, height=256, **kw):
    """a = 0.9, inclination 60 deg, +-25 M from r = 1000 M, disc r_isco..30 M."""
    cfg = RenderConfig(
        M_kg=4.3e6 * M_SUN, spin=0.9,
        cam=Camera(r=1000.0, theta=math.radians(60.0), phi=0.0, fov=_fov(25.0)),
        width=width, height=height, sqrt_spp=1, disc_r_out=30.0, eddington=0.1,
        rtol=1e-8, atol=1e-10, r_escape=1100.0, quiet=True,
    )
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def edge_on_a0998(width=1024, height=1024, **kw):
    """a = 0.998, inclination 85 deg, +-25 M, disc r_isco..50 M, M = 10 M_sun."""
    cfg = RenderConfig(
        M_kg=10.0 * M_SUN, spin=0.998,
        cam=Camera(r=1000.0, theta=math.radians(85.0), phi=0.0, fov=_fov(25.0)),
        width=width, height=height, sqrt_spp=1, disc_r_out=50.0, eddington=0.3,
        rtol=1e-8, atol=1e-10, r_escape=1100.0, quiet=True,
    )
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def sun_hotspot_spp2():
    """Close camera, the Sun in view beside the hole, an orbiting hot spot,
    four samples per pixel."""
    hs = HotSpot(enabled=True, r=8.0, phi0=0.3, sigma=0.6, contrast=25.0)
    hs.set_spin(0.9, 1)
    return RenderConfig(
        M_kg=4.3e6 * M_SUN, spin=0.9,
        cam=Camera(r=60.0, theta=math.radians(80.0), phi=0.0, fov=1.0, yaw=0.15),
        width=24, height=16, sqrt_spp=2, disc_r_out=24.0, eddington=0.1,
        sun_enabled=True, sun=SunBody(centre=(0.0, 22.0, 0.0), radius=4.0, T_eff=5772.0),
        hotspot=hs, observer_time=40.0,
        rtol=1e-9, atol=1e-11, r_escape=280.0, quiet=True,
    )


def neutron_star():
    """a = 0 with a neutron-star surface at R = 5.8 M, caps on, disc off."""
    ns = NeutronStar(enabled=True, R=5.8, T_eff=1.0e6, Omega=0.01, caps=True)
    return RenderConfig(
        M_kg=1.4 * M_SUN, spin=0.0,
        cam=Camera(r=80.0, theta=math.radians(60.0), phi=0.0, fov=0.3),
        width=24, height=24, sqrt_spp=1, disc_enabled=False,
        star=ns, observer_time=5.0,
        rtol=1e-9, atol=1e-11, r_escape=340.0, quiet=True,
    )


# name -> (config factory, window (x0, y0, w, h))
CASES = {
    "a09_i60_centre": (lambda: kerr_a09_i60(), (112, 112, 32, 32)),
    "a09_i60_corner": (lambda: kerr_a09_i60(), (0, 0, 24, 24)),
    "a0998_i85_ring": (lambda: edge_on_a0998(), (468, 500, 40, 24)),
    "sun_hotspot_spp2": (sun_hotspot_spp2, (0, 0, 24, 16)),
    "neutron_star": (neutron_star, (0, 0, 24, 24)),
    "quasar_jets": (lambda: workloads.quasar_jets(320, 180), (150, 40, 20, 12)),
    "m87_jets": (lambda: workloads.m87_jets(320, 180), (150, 60, 20, 12)),
}

# A whole small frame through the reference's own bh::render (pixels).
RENDER_CASE = ("a09_i60_small_render", lambda: kerr_a09_i60(width=48, height=27, sqrt_spp=2))
