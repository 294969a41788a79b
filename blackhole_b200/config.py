"""Host-side mirror of the reference's scene and render configuration.

``RenderConfig``, ``Camera``, ``SunBody``, ``HotSpot``, ``NeutronStar`` and
``RenderStats`` carry the same field names, meanings and defaults as the
reference's C++ structs (render.h:15-69, scene.h:232-351,
neutronstar.h:43-70), so code written against ``bh::RenderConfig`` reads the
same here.  ``to_c()`` packs a config into the C-ABI struct of
include/bh_gpu.h.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

from . import abi

M_SUN = 1.98847e30          # kg (constants.h:38)
T_SUN = 5772.0              # K  (constants.h:41)


@dataclass
class Camera:
    """bh::Camera (scene.h:343-351)."""

    r: float = 60.0
    theta: float = math.pi / 2.0
    phi: float = 0.0
    fov: float = 0.6
    yaw: float = 0.0
    pitch: float = 0.0
    roll: float = 0.0


@dataclass
class SunBody:
    """bh::SunBody (scene.h:232-236)."""

    centre: tuple = (0.0, 0.0, 0.0)
    radius: float = 1.0
    T_eff: float = T_SUN


@dataclass
class HotSpot:
    """bh::HotSpot (scene.h:306-313)."""

    enabled: bool = False
    r: float = 8.0
    phi0: float = 0.0
    sigma: float = 0.6
    contrast: float = 25.0
    omega: float = 0.0
    sense: int = 1

    def set_spin(self, a: float, prograde: int) -> None:
        """scene.h:315-318."""
        self.sense = prograde
        self.omega = prograde / (self.r * math.sqrt(self.r) + prograde * a)


@dataclass
class NeutronStar:
    """bh::NeutronStar (neutronstar.h:43-70)."""

    enabled: bool = False
    M_kg: float = 1.4 * M_SUN
    R_m: float = 12000.0
    R: float = 5.8
    T_eff: float = 1.0e6
    spin_hz: float = 0.0
    Omega: float = 0.0
    caps: bool = False
    cap_tilt: float = 60.0 * math.pi / 180.0
    cap_radius: float = 20.0 * math.pi / 180.0
    cap_T: float = 3.0e6
    cap_phase0: float = 0.0
    two_caps: bool = True


@dataclass
class Jet:
    """bh::Jet (jet.h:96-146) without `enabled` (RenderConfig.jet_enabled).
    The last block is what Jet::configure sets (``configure`` below, or
    ``RenderConfig.setup_jet()`` for the CLI's set-up)."""

    z_base: float = 3.0
    z_top: float = 120.0
    R_base: float = 1.6
    k: float = 0.58
    gamma_max: float = 10.0
    z_sat: float = 80.0
    alpha: float = 0.7
    u_peak: float = 0.82
    u_wid: float = 0.17
    spine: float = 0.06
    spine_wid: float = 0.40
    zeta: float = 2.0
    eps_rad: float = 0.02
    phi_flux: float = 50.0
    a: float = 0.0
    Omega_F: float = 0.0
    P_jet: float = 0.0
    L_rad: float = 0.0
    j_nu0: float = 0.0
    r_bound: float = 0.0
    volume_rg3: float = 0.0

    def to_c(self) -> abi.bh_jet:
        j = abi.bh_jet()
        for k in abi.JET_PARAMS + abi.JET_CONFIGURED:
            setattr(j, k, float(getattr(self, k)))
        return j

    def update_from(self, j: abi.bh_jet) -> None:
        for k in abi.JET_PARAMS + abi.JET_CONFIGURED:
            setattr(self, k, getattr(j, k))


@dataclass
class RenderConfig:
    """bh::RenderConfig (render.h:15-53) plus the GPU extensions.

    Extensions (absent from the reference):
      precision   abi.PRECISION_FP64 or abi.PRECISION_MIXED
      sky_mode    abi.SKY_GALACTIC (the reference sky) or abi.SKY_UNIFORM
      stop_mode   abi.STOP_REFERENCE (render.cpp:73) or abi.STOP_RELATIVE
      stop_epsilon  r_stop = r_+ (1 + stop_epsilon) under STOP_RELATIVE
      milky_way   diffuse background on/off
      mixed_rtol, mixed_atol  tolerances of the mixed path (0: rtol/atol)
      mixed_step_limit  abi.STEP_LIMIT_* of the mixed path (AUTO: no step cap
                  unless the Sun, a neutron star or a jet is in the scene)
      mixed_capture  abi.CAPTURE_* of the mixed path (AUTO: a ray moving inwards
                  inside the innermost photon orbit ends there as captured,
                  unless a neutron star or a jet is in the scene)
      mixed_near_critical  abi.NEAR_CRITICAL_* of the mixed path (AUTO: rays
                  that circle close to the photon shell before escaping are
                  traced in binary64 by a kernel beside the binary32 one)
    """

    M_kg: float = 10.0 * M_SUN
    spin: float = 0.9
    cam: Camera = field(default_factory=Camera)
    width: int = 1280
    height: int = 720
    sqrt_spp: int = 2
    disc_enabled: bool = True
    disc_r_out: float = 24.0
    eddington: float = 0.1
    disc_sense: int = 1
    stars_enabled: bool = True
    star_count: int = 250000
    seed: int = 20240921
    sun_enabled: bool = False
    sun: SunBody = field(default_factory=SunBody)
    hotspot: HotSpot = field(default_factory=HotSpot)
    star: NeutronStar = field(default_factory=NeutronStar)
    jet_enabled: bool = False
    jet: Jet = field(default_factory=Jet)
    observer_time: float = 0.0
    rtol: float = 1e-9
    atol: float = 1e-11
    r_escape: float = 4000.0
    max_steps: int = 20000
    threads: int = 0
    quiet: bool = False
    # ---- extensions ----
    precision: int = abi.PRECISION_FP64
    sky_mode: int = abi.SKY_GALACTIC
    stop_mode: int = abi.STOP_REFERENCE
    milky_way: bool = True
    stop_epsilon: float = 0.0
    mixed_rtol: float = 0.0
    mixed_atol: float = 0.0
    mixed_step_limit: int = abi.STEP_LIMIT_AUTO
    mixed_capture: int = abi.CAPTURE_AUTO
    mixed_near_critical: int = abi.NEAR_CRITICAL_AUTO

    @property
    def n_rays(self) -> int:
        s = max(1, self.sqrt_spp)
        return self.width * self.height * s * s

    def to_c(self) -> abi.bh_render_config:
        c = abi.bh_render_config()
        c.struct_size = C.sizeof(abi.bh_render_config)
        c.abi_version = abi.ABI_VERSION
        c.M_kg = self.M_kg
        c.spin = self.spin
        for k in ("r", "theta", "phi", "fov", "yaw", "pitch", "roll"):
            setattr(c.cam, k, float(getattr(self.cam, k)))
        c.width, c.height, c.sqrt_spp = self.width, self.height, self.sqrt_spp
        c.disc_enabled = int(bool(self.disc_enabled))
        c.disc_r_out = self.disc_r_out
        c.eddington = self.eddington
        c.disc_sense = self.disc_sense
        c.stars_enabled = int(bool(self.stars_enabled))
        c.star_count = self.star_count
        c.sun_enabled = int(bool(self.sun_enabled))
        c.seed = self.seed & 0xFFFFFFFFFFFFFFFF
        for i in range(3):
            c.sun.centre[i] = float(self.sun.centre[i])
        c.sun.radius = self.sun.radius
        c.sun.T_eff = self.sun.T_eff
        hs = self.hotspot
        c.hotspot.enabled = int(bool(hs.enabled))
        c.hotspot.sense = hs.sense
        c.hotspot.r, c.hotspot.phi0, c.hotspot.sigma = hs.r, hs.phi0, hs.sigma
        c.hotspot.contrast, c.hotspot.omega = hs.contrast, hs.omega
        st = self.star
        c.star.enabled = int(bool(st.enabled))
        c.star.caps = int(bool(st.caps))
        for k in ("M_kg", "R_m", "R", "T_eff", "spin_hz", "Omega", "cap_tilt", "cap_radius",
                  "cap_T", "cap_phase0"):
            setattr(c.star, k, float(getattr(st, k)))
        c.star.two_caps = int(bool(st.two_caps))
        c.jet_enabled = int(bool(self.jet_enabled))
        c.observer_time = self.observer_time
        c.rtol, c.atol, c.r_escape = self.rtol, self.atol, self.r_escape
        c.max_steps = self.max_steps
        c.threads = self.threads
        c.quiet = int(bool(self.quiet))
        c.precision = self.precision
        c.sky_mode = self.sky_mode
        c.stop_mode = self.stop_mode
        c.milky_way = int(bool(self.milky_way))
        c.stop_epsilon = self.stop_epsilon
        c.mixed_rtol = self.mixed_rtol
        c.mixed_atol = self.mixed_atol
        c.jet = self.jet.to_c()
        c.mixed_step_limit = self.mixed_step_limit
        c.mixed_capture = self.mixed_capture
        c.mixed_near_critical = self.mixed_near_critical
        return c

    def setup_jet(self) -> "RenderConfig":
        """The CLI's jet set-up (main.cpp:399-423) through the library:
        configures ``jet`` from the disc's accretion rate, or switches the
        jet off where the reference does.  Returns self."""
        from .gpu import load_library

        c = self.to_c()
        rc = load_library().bh_render_config_setup_jet(C.byref(c))
        if rc != abi.OK:
            raise ValueError(f"bh_render_config_setup_jet failed ({rc})")
        self.jet_enabled = bool(c.jet_enabled)
        self.jet.update_from(c.jet)
        return self

    def replace(self, **kw) -> "RenderConfig":
        import copy

        out = copy.deepcopy(self)
        for k, v in kw.items():
            if not hasattr(out, k):
                raise AttributeError(f"RenderConfig has no field {k!r}")
            setattr(out, k, v)
        return out


@dataclass
class RenderStats:
    """bh::RenderStats (render.h:55-69) plus the GPU extensions."""

    rays: int = 0
    steps: int = 0
    captured: int = 0
    disc_hits: int = 0
    sun_hits: int = 0
    star_hits: int = 0
    jet_rays: int = 0
    escaped: int = 0
    exhausted: int = 0
    max_norm_error: float = 0.0
    max_carter_drift: float = 0.0
    seconds: float = 0.0
    total_flux: float = 0.0
    attempts: int = 0
    kernel_ms: float = 0.0
    shade_ms: float = 0.0
    h2d_bytes: int = 0
    d2h_bytes: int = 0

    def to_c(self) -> abi.bh_render_stats:
        s = abi.bh_render_stats()
        for name, _ in abi.bh_render_stats._fields_:
            setattr(s, name, getattr(self, name))
        return s

    def update_from(self, s: abi.bh_render_stats) -> None:
        for name, _ in abi.bh_render_stats._fields_:
            setattr(self, name, getattr(s, name))
