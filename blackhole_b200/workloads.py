"""Named render workloads.

Each function returns a ``RenderConfig`` (or a list of them) for one of the
measured scenes.  Common to all of them: observer at r = 1000 M (unless
stated), field of view covering +-25 M at the hole (fov = 2 atan(25/1000)),
one sample per pixel, escape radius 1.1 r_obs, horizon stop at
r_+ (1 + 1e-6), and a seeded 250,000-star sky that is isotropic, with
magnitudes from log N(<m) = 0.45 m up to m = 6.5, B-V uniform in
[-0.3, 1.8] and a uniform 21.5 mag/arcsec^2 diffuse background.
"""
from __future__ import annotations

import math
import random

from . import abi
from .config import M_SUN, Camera, RenderConfig

R_OBS = 1000.0


def _fov(half_width_m: float, r_obs: float = R_OBS) -> float:
    return 2.0 * math.atan(half_width_m / r_obs)


def _base(**kw) -> RenderConfig:
    cfg = RenderConfig(
        sqrt_spp=1,
        rtol=1e-8,
        atol=1e-10,
        r_escape=1.1 * R_OBS,
        star_count=250000,
        seed=20240921,
        sky_mode=abi.SKY_UNIFORM,
        stop_mode=abi.STOP_RELATIVE,
        stop_epsilon=1e-6,
        quiet=True,
    )
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def kerr_fp64_256() -> RenderConfig:
    """Plain FP64 render, 256x256: a = 0.9, inclination 60 deg,
    M = 4.3e6 M_sun, disc r_isco..30 M at 0.1 Eddington."""
    return _base(
        M_kg=4.3e6 * M_SUN, spin=0.9,
        cam=Camera(r=R_OBS, theta=math.radians(60.0), phi=0.0, fov=_fov(25.0)),
        width=256, height=256, disc_r_out=30.0, eddington=0.1,
        precision=abi.PRECISION_FP64,
    )


def edge_on_1024(precision: int = abi.PRECISION_MIXED) -> RenderConfig:
    """1024x1024 near edge-on frame: a = 0.998, inclination 85 deg,
    M = 10 M_sun, disc r_isco..50 M at 0.3 Eddington."""
    return _base(
        M_kg=10.0 * M_SUN, spin=0.998,
        cam=Camera(r=R_OBS, theta=math.radians(85.0), phi=0.0, fov=_fov(25.0)),
        width=1024, height=1024, disc_r_out=50.0, eddington=0.3,
        precision=precision,
    )


def batch_64_frames(seed: int = 64, precision: int = abi.PRECISION_MIXED) -> list:
    """64 frames of uneven size in a seeded shuffle: spins {0, 0.5, 0.9, 0.998}
    x inclinations {15, 45, 70, 85} deg x resolutions {256, 512, 1024, 2048}^2
    (every combination once), observer radius uniform in [500, 2000] M, disc
    r_isco..30 M at 0.1 Eddington, M = 4.3e6 M_sun.  The field of view keeps
    +-25 M at each observer radius."""
    rng = random.Random(seed)
    combos = [(a, i, n) for a in (0.0, 0.5, 0.9, 0.998) for i in (15.0, 45.0, 70.0, 85.0)
              for n in (256, 512, 1024, 2048)]
    rng.shuffle(combos)
    frames = []
    for a, inc, n in combos:
        r_obs = rng.uniform(500.0, 2000.0)
        frames.append(_base(
            M_kg=4.3e6 * M_SUN, spin=a,
            cam=Camera(r=r_obs, theta=math.radians(inc), phi=0.0, fov=_fov(25.0, r_obs)),
            width=n, height=n, disc_r_out=30.0, eddington=0.1,
            r_escape=1.1 * r_obs, precision=precision,
        ))
    return frames


def adjoint_512(target: bool = False) -> RenderConfig:
    """512x512 luminance frame for the gradient check: a = 0.7, inclination
    50 deg, 0.2 Eddington, r_out = 25 M (target: a = 0.75, 53 deg, 0.22,
    27 M), M = 4.3e6 M_sun."""
    if target:
        a, inc, edd, r_out = 0.75, 53.0, 0.22, 27.0
    else:
        a, inc, edd, r_out = 0.7, 50.0, 0.2, 25.0
    return _base(
        M_kg=4.3e6 * M_SUN, spin=a,
        cam=Camera(r=R_OBS, theta=math.radians(inc), phi=0.0, fov=_fov(25.0)),
        width=512, height=512, disc_r_out=r_out, eddington=edd,
        precision=abi.PRECISION_FP64,
    )


def critical_curve_prograde_edge(a: float, inclination: float) -> float:
    """Image-plane abscissa (in M, Bardeen's alpha = -xi / sin i) where the
    critical curve of a Kerr hole of spin a seen from inclination i crosses the
    equator line on the prograde side: the spherical photon orbit radius r_p
    in [r_ph+, r_ph-] with beta^2 = eta + a^2 cos^2 i - xi^2 cot^2 i = 0,
    xi = -(r^3 - 3 r^2 + a^2 r + a^2) / (a (r - 1)),
    eta = -r^3 (r^3 - 6 r^2 + 9 r - 4 a^2) / (a^2 (r - 1)^2)  (Bardeen 1973).
    Negative: on the camera's left, where prograde photons pass."""
    aa = abs(a)
    if aa < 1e-6:
        return -math.sqrt(27.0)
    r_lo = 2.0 * (1.0 + math.cos((2.0 / 3.0) * math.acos(-aa)))
    r_hi = 2.0 * (1.0 + math.cos((2.0 / 3.0) * math.acos(aa)))

    def xi(r):
        return -(r ** 3 - 3.0 * r * r + aa * aa * r + aa * aa) / (aa * (r - 1.0))

    def beta2(r):
        eta = -r ** 3 * (r ** 3 - 6.0 * r * r + 9.0 * r - 4.0 * aa * aa) / (aa * aa * (r - 1.0) ** 2)
        return eta + aa * aa * math.cos(inclination) ** 2 - xi(r) ** 2 / math.tan(inclination) ** 2

    # beta^2 < 0 just above r_ph+ and > 0 inside the curve: scan for the
    # first sign change, then bisect.
    n = 4000
    prev_r, prev_v = r_lo + 1e-9, beta2(r_lo + 1e-9)
    for k in range(1, n + 1):
        r = r_lo + (r_hi - r_lo) * k / n
        v = beta2(r)
        if (v > 0.0) != (prev_v > 0.0):
            lo, hi = prev_r, r
            for _ in range(100):
                mid = 0.5 * (lo + hi)
                if (beta2(mid) > 0.0) == (prev_v > 0.0):
                    lo = mid
                else:
                    hi = mid
            return -xi(0.5 * (lo + hi)) / math.sin(inclination) * (1.0 if a >= 0 else -1.0)
        prev_r, prev_v = r, v
    raise ValueError("no equatorial point of the critical curve")


def photon_ring_4096(precision: int = abi.PRECISION_MIXED, size: int = 4096) -> RenderConfig:
    """Narrow +-8 M frame at a = 0.998, inclination 75 deg, M = 6.5e9 M_sun,
    disc r_isco..100 M at 0.5 Eddington, centred (yaw) on the prograde
    equatorial point of the critical curve (alpha = -2.18 M), where rays
    skim the photon orbits before escaping, falling in or meeting the disc."""
    cfg = _base(
        M_kg=6.5e9 * M_SUN, spin=0.998,
        cam=Camera(r=R_OBS, theta=math.radians(75.0), phi=0.0, fov=_fov(8.0)),
        width=size, height=size, disc_r_out=100.0, eddington=0.5,
        precision=precision,
    )
    cfg.cam.yaw = math.atan(critical_curve_prograde_edge(0.998, math.radians(75.0)) / R_OBS)
    return cfg


def photon_ring_crop(size: int = 1024, target: bool = False) -> RenderConfig:
    """The central size x size crop of the 4096^2 photon-ring frame (same
    pixel scale, same centre on the critical curve), in binary64, for the
    adjoint with respect to spin and inclination.  target: the frame at
    a = 0.99, inclination 76 deg the loss is measured against."""
    cfg = photon_ring_4096(abi.PRECISION_FP64)
    cfg.cam.fov = 2.0 * math.atan(math.tan(0.5 * cfg.cam.fov) * size / 4096.0)
    cfg.width = cfg.height = size
    if target:
        cfg.spin = 0.99
        cfg.cam.theta = math.radians(76.0)
    return cfg


def _jet_preset(cfg: RenderConfig, z_top: float, gamma_max: float) -> RenderConfig:
    """Jets on, configured the way the CLI does (main.cpp:399-423), and the
    escape sphere outside them (main.cpp:881-890)."""
    cfg.jet_enabled = True
    cfg.jet.z_top = z_top
    cfg.jet.gamma_max = gamma_max
    cfg.setup_jet()
    far = cfg.cam.r * 3.0 + 100.0
    if cfg.jet_enabled:
        far = max(far, cfg.jet.r_bound * 1.5)
    cfg.r_escape = far
    return cfg


def quasar_jets(width: int = 320, height: int = 180, precision: int = abi.PRECISION_FP64) -> RenderConfig:
    """The reference's `quasar` preset (main.cpp:300-330): a = 0.998,
    M = 1e9 M_sun, 84 deg, r_cam 80 M, fov 0.90, disc to 20 M at 0.5
    Eddington, Blandford-Znajek jets to z = 130 M with Gamma_max = 10; the
    reference's galactic sky and stop radius, 1 sample per pixel."""
    cfg = RenderConfig(
        M_kg=1.0e9 * M_SUN, spin=0.998,
        cam=Camera(r=80.0, theta=math.radians(84.0), phi=0.0, fov=0.90),
        width=width, height=height, sqrt_spp=1, disc_r_out=20.0, eddington=0.5,
        quiet=True, precision=precision,
    )
    return _jet_preset(cfg, 130.0, 10.0)


def m87_jets(width: int = 320, height: int = 180, precision: int = abi.PRECISION_FP64) -> RenderConfig:
    """The reference's `m87` preset (main.cpp:252-267): a = 0.94,
    M = 6.5e9 M_sun, 17 deg, r_cam 120 M, fov 0.78, disc to 30 M at 1e-5
    Eddington, jets to z = 130 M with Gamma_max = 8."""
    cfg = RenderConfig(
        M_kg=6.5e9 * M_SUN, spin=0.94,
        cam=Camera(r=120.0, theta=math.radians(17.0), phi=0.0, fov=0.78),
        width=width, height=height, sqrt_spp=1, disc_r_out=30.0, eddington=1e-5,
        quiet=True, precision=precision,
    )
    return _jet_preset(cfg, 130.0, 8.0)


def hotspot_orbit(frames: int = 24, width: int = 256, height: int = 144, orbits: float = 1.0,
                  precision: int = abi.PRECISION_FP64) -> list:
    """The frames of a hot-spot film as the CLI builds them (main.cpp:78-86,
    826-835, 950-958): a = 0.9, M = 4.3e6 M_sun, 80 deg from r = 60 M,
    fov 0.6, disc to 24 M at 0.1 Eddington, a hot spot at r = 8 M
    (contrast 25, sigma 0.6 M) orbiting progradely; the sequence covers
    `orbits` orbital periods and frame f sits at u = f / frames of it."""
    from .config import HotSpot

    base = RenderConfig(
        M_kg=4.3e6 * M_SUN, spin=0.9,
        cam=Camera(r=60.0, theta=math.radians(80.0), phi=0.0, fov=0.6),
        width=width, height=height, sqrt_spp=1, disc_r_out=24.0, eddington=0.1,
        hotspot=HotSpot(enabled=True, r=8.0, sigma=0.6, contrast=25.0),
        r_escape=60.0 * 3.0 + 100.0, quiet=True, precision=precision,
    )
    base.hotspot.set_spin(base.spin, base.disc_sense)
    span = orbits * 2.0 * math.pi / abs(base.hotspot.omega)
    out = []
    for f in range(frames):
        c = base.replace()
        c.observer_time = f / frames * span
        out.append(c)
    return out


def exposure_probe(cfg: RenderConfig) -> RenderConfig:
    """The low-resolution probe the CLI meters a film's locked exposure on
    (main.cpp:931-944), for the frame `cfg` (the sequence's middle frame)."""
    p = cfg.replace()
    p.width = max(64, cfg.width // 6)
    p.height = max(36, cfg.height // 6)
    p.sqrt_spp = 1
    p.star_count = min(cfg.star_count, 40000)
    p.quiet = True
    return p
