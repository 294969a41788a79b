"""Python binding of the C-ABI in include/bh_gpu.h.

``Renderer`` wraps a ``bh_ctx``.  ``render(cfg, stats)`` is the drop-in for the
reference's ``bh::render(cfg, stats)`` (render.h:72): it returns the frame's
CIE XYZ radiance as a float64 array of shape (height, width, 3) and adds the
frame's counters into ``stats`` (``seconds`` is overwritten), exactly as the
reference does.  There is no CPU fallback: without the built library or an
sm_100 GPU every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from . import abi
from .config import RenderConfig, RenderStats

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libbh_gpu.so")

_lib = None
_lock = threading.Lock()


class BHError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def load_library():
    """Load libbh_gpu.so (building it first if this tree has no copy)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            from . import build as _build

            _build.build()
        lib = C.CDLL(LIB_PATH)
        P = C.POINTER
        ctx_p = C.c_void_p
        cfg_p = P(abi.bh_render_config)
        st_p = P(abi.bh_render_stats)
        sigs = {
            "bh_gpu_abi_version": (C.c_int, []),
            "bh_render_config_default": (None, [cfg_p]),
            "bh_gpu_create": (C.c_int, [C.c_int, P(ctx_p)]),
            "bh_gpu_destroy": (None, [ctx_p]),
            "bh_gpu_last_error": (C.c_char_p, [ctx_p]),
            "bh_gpu_render": (C.c_int, [ctx_p, cfg_p, P(abi.bh_xyz), st_p]),
            "bh_gpu_render_device": (C.c_int, [ctx_p, cfg_p, C.c_void_p, st_p, C.c_void_p]),
            "bh_gpu_trace_rays": (C.c_int, [ctx_p, cfg_p, P(abi.bh_ray_result), st_p]),
            "bh_gpu_render_batch": (C.c_int, [ctx_p, cfg_p, C.c_int, P(P(abi.bh_xyz)), st_p]),
            "bh_gpu_set_launch": (C.c_int, [ctx_p, C.c_int, P(abi.bh_launch_params)]),
            "bh_gpu_get_launch": (C.c_int, [ctx_p, C.c_int, P(abi.bh_launch_params)]),
            "bh_gpu_autotune": (C.c_int, [ctx_p, cfg_p, P(abi.bh_launch_params), P(C.c_double)]),
            "bh_gpu_autotune_batch": (C.c_int, [ctx_p, cfg_p, C.c_int, P(abi.bh_launch_params), P(C.c_double)]),
            "bh_gpu_set_step_budget": (C.c_int, [ctx_p, C.c_longlong]),
            "bh_gpu_request_abort": (None, [ctx_p]),
            "bh_gpu_clear_abort": (None, [ctx_p]),
            "bh_star_catalogue": (C.c_int, [C.c_int, C.c_uint64, C.c_int, P(C.c_double)]),
            "bh_blackbody_table": (C.c_int, [P(C.c_double)]),
            "bh_gpu_fma_peak": (C.c_int, [C.c_int, C.c_int, P(C.c_double)]),
            "bh_gpu_trace_noalloc": (C.c_int, [C.c_int, cfg_p, C.c_void_p, C.c_void_p]),
            "bh_display_default": (None, [P(abi.bh_display)]),
            "bh_jet_configure": (None, [P(abi.bh_jet), C.c_double, C.c_double, C.c_double]),
            "bh_render_config_setup_jet": (C.c_int, [cfg_p]),
            "bh_gpu_develop": (C.c_int, [ctx_p, P(abi.bh_xyz), C.c_int, C.c_int, P(abi.bh_display),
                                         P(C.c_uint8), P(C.c_double)]),
            "bh_gpu_render_rgb": (C.c_int, [ctx_p, cfg_p, P(abi.bh_display), P(C.c_uint8), P(C.c_double), st_p]),
            "bh_gpu_render_batch_rgb": (C.c_int, [ctx_p, cfg_p, C.c_int, P(abi.bh_display), P(P(C.c_uint8)),
                                                  P(C.c_double), st_p]),
            "bh_gpu_eval": (C.c_int, [ctx_p, cfg_p, C.c_int, P(C.c_double), C.c_longlong, P(C.c_double)]),
            "bh_gpu_adjoint": (C.c_int, [ctx_p, cfg_p, P(C.c_float), P(abi.bh_grad4)]),
            "bh_gpu_adjoint_rays": (C.c_int, [ctx_p, cfg_p, P(C.c_float), P(abi.bh_grad4), P(C.c_double),
                                              P(C.c_double)]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        if lib.bh_gpu_abi_version() != abi.ABI_VERSION:
            raise RuntimeError("libbh_gpu.so ABI version does not match blackhole_b200.abi")
        _lib = lib
        return lib


def default_config_c() -> abi.bh_render_config:
    c = abi.bh_render_config()
    load_library().bh_render_config_default(C.byref(c))
    return c


def _as_c(cfg) -> abi.bh_render_config:
    return cfg.to_c() if isinstance(cfg, RenderConfig) else cfg


class Renderer:
    """One GPU context (bh_ctx) on `device`."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.bh_gpu_create(device, C.byref(h))
        if rc != abi.OK:
            raise BHError(rc, f"bh_gpu_create(device={device}) failed: a CUDA sm_100 GPU is required")
        self._h = h

    # -- lifetime --------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.bh_gpu_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def _check(self, rc: int) -> None:
        if rc != abi.OK:
            msg = self.lib.bh_gpu_last_error(self._h)
            raise BHError(rc, msg.decode() if msg else "")

    # -- the render path -------------------------------------------------------
    def render(self, cfg, stats: RenderStats | None = None) -> np.ndarray:
        c = _as_c(cfg)
        # invalid sizes are rejected by the library, not here
        out = np.empty((max(c.height, 0), max(c.width, 0), 3), dtype=np.float64)
        st = stats.to_c() if stats is not None else abi.bh_render_stats()
        rc = self.lib.bh_gpu_render(self._h, C.byref(c), out.ctypes.data_as(C.POINTER(abi.bh_xyz)),
                                    C.byref(st))
        if stats is not None:
            stats.update_from(st)
        self._check(rc)
        return out

    def render_into(self, cfg, out: np.ndarray, stats: abi.bh_render_stats | None = None) -> None:
        """Render into a caller-owned (H, W, 3) float64 host array."""
        c = _as_c(cfg)
        if out.shape != (c.height, c.width, 3) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (H, W, 3)")
        rc = self.lib.bh_gpu_render(self._h, C.byref(c), out.ctypes.data_as(C.POINTER(abi.bh_xyz)),
                                    C.byref(stats) if stats is not None else None)
        self._check(rc)

    def render_device(self, cfg, d_pixels: int, stream: int = 0, stats: abi.bh_render_stats | None = None) -> None:
        """Render into a device buffer of W*H bh_xyz (e.g. a torch tensor's data_ptr())."""
        c = _as_c(cfg)
        rc = self.lib.bh_gpu_render_device(self._h, C.byref(c), C.c_void_p(d_pixels),
                                           C.byref(stats) if stats is not None else None,
                                           C.c_void_p(stream) if stream else None)
        self._check(rc)

    def trace_rays(self, cfg, stats: RenderStats | None = None) -> np.ndarray:
        """Per-sample results (structured array, see abi.ray_result_dtype)."""
        c = _as_c(cfg)
        s = max(1, c.sqrt_spp)
        n = c.width * c.height * s * s
        out = np.empty(n, dtype=abi.ray_result_dtype())
        st = stats.to_c() if stats is not None else abi.bh_render_stats()
        rc = self.lib.bh_gpu_trace_rays(self._h, C.byref(c), out.ctypes.data_as(C.POINTER(abi.bh_ray_result)),
                                        C.byref(st))
        if stats is not None:
            stats.update_from(st)
        self._check(rc)
        return out

    def render_batch(self, cfgs, stats: list | None = None, outs: list | None = None) -> list:
        """The frames of `cfgs` in one launch (bh_gpu_render_batch), into new
        (H, W, 3) arrays or into `outs` (C-contiguous float64 arrays of those
        shapes, e.g. pinned buffers reused from call to call)."""
        cs = (abi.bh_render_config * len(cfgs))(*[_as_c(c) for c in cfgs])
        if outs is None:
            outs = [np.empty((c.height, c.width, 3), dtype=np.float64) for c in cs]
        elif len(outs) != len(cfgs) or any(o.shape != (c.height, c.width, 3) or o.dtype != np.float64
                                           or not o.flags.c_contiguous for o, c in zip(outs, cs)):
            raise ValueError("outs must hold one C-contiguous float64 (H, W, 3) array per frame")
        ptrs = (C.POINTER(abi.bh_xyz) * len(cfgs))(*[o.ctypes.data_as(C.POINTER(abi.bh_xyz)) for o in outs])
        sts = (abi.bh_render_stats * len(cfgs))()
        rc = self.lib.bh_gpu_render_batch(self._h, cs, len(cfgs), ptrs, sts)
        if stats is not None:
            stats.clear()
            for s in sts:
                r = RenderStats()
                r.update_from(s)
                stats.append(r)
        self._check(rc)
        return outs

    # -- display transform -----------------------------------------------------------
    def display_settings(self, **kw) -> abi.bh_display:
        """bh_display with the reference CLI's defaults (HDR, metered exposure,
        no glare, 16 decades), fields overridden by keyword."""
        d = abi.bh_display()
        self.lib.bh_display_default(C.byref(d))
        for k, v in kw.items():
            if k == "tonemap" and isinstance(v, str):
                v = abi.TONEMAP_NAMES.index(v)
            setattr(d, k, v)
        return d

    def develop(self, xyz, display=None, meter_only: bool = False, **kw):
        """add_glare + auto_exposure + develop of a (H, W, 3) XYZ image on the
        GPU: returns (rgb uint8 (H, W, 3) or None, exposure)."""
        a = np.ascontiguousarray(xyz, dtype=np.float64)
        h, w = a.shape[0], a.shape[1]
        d = display if display is not None else self.display_settings(**kw)
        out = None if meter_only else np.empty((h, w, 3), dtype=np.uint8)
        e = C.c_double(0.0)
        u8 = out.ctypes.data_as(C.POINTER(C.c_uint8)) if out is not None else None
        self._check(self.lib.bh_gpu_develop(self._h, a.ctypes.data_as(C.POINTER(abi.bh_xyz)), w, h,
                                            C.byref(d), u8, C.byref(e)))
        return out, e.value

    def render_rgb(self, cfg, display=None, stats: RenderStats | None = None, meter_only: bool = False, **kw):
        """Render and develop on the device: returns (rgb uint8 (H, W, 3) or
        None, exposure); only the 8-bit image crosses to the host."""
        c = _as_c(cfg)
        d = display if display is not None else self.display_settings(**kw)
        out = None if meter_only else np.empty((c.height, c.width, 3), dtype=np.uint8)
        e = C.c_double(0.0)
        st = stats.to_c() if stats is not None else abi.bh_render_stats()
        u8 = out.ctypes.data_as(C.POINTER(C.c_uint8)) if out is not None else None
        rc = self.lib.bh_gpu_render_rgb(self._h, C.byref(c), C.byref(d), u8, C.byref(e), C.byref(st))
        if stats is not None:
            stats.update_from(st)
        self._check(rc)
        return out, e.value

    def render_batch_rgb(self, cfgs, display=None, stats: list | None = None, **kw):
        """Frames of an animation traced in one launch and developed on the
        device: returns ([rgb uint8 (H, W, 3)], [exposure])."""
        cs = (abi.bh_render_config * len(cfgs))(*[_as_c(c) for c in cfgs])
        d = display if display is not None else self.display_settings(**kw)
        outs = [np.empty((c.height, c.width, 3), dtype=np.uint8) for c in cs]
        ptrs = (C.POINTER(C.c_uint8) * len(cfgs))(*[o.ctypes.data_as(C.POINTER(C.c_uint8)) for o in outs])
        ex = (C.c_double * len(cfgs))()
        sts = (abi.bh_render_stats * len(cfgs))()
        rc = self.lib.bh_gpu_render_batch_rgb(self._h, cs, len(cfgs), C.byref(d), ptrs, ex, sts)
        if stats is not None:
            stats.clear()
            for st in sts:
                r = RenderStats()
                r.update_from(st)
                stats.append(r)
        self._check(rc)
        return outs, list(ex)

    # -- discrete adjoint ----------------------------------------------------------
    def eval(self, cfg, what: int, inputs=None):
        """The render path's device functions at given inputs (bh_gpu_eval):
        abi.EVAL_RHS (states (n, 8) -> derivatives (n, 8), in cfg's
        precision), EVAL_DISC_TEMPERATURE (radii (n,) -> kelvin (n,)),
        EVAL_BLACKBODY (kelvin (n,) -> XYZ (n, 3)), EVAL_FRAME (-> the 8 frame
        constants r_+, r_-, r_in, r_out, efficiency, accretion rate, stop and
        escape radius)."""
        c = _as_c(cfg)
        dp = C.POINTER(C.c_double)
        if what == abi.EVAL_FRAME:
            out = np.zeros(8)
            self._check(self.lib.bh_gpu_eval(self._h, C.byref(c), what, None, 1, out.ctypes.data_as(dp)))
            return out
        x = np.ascontiguousarray(inputs, dtype=np.float64)
        if what == abi.EVAL_RHS:
            x = x.reshape(-1, 8)
            shape = x.shape
        elif what == abi.EVAL_BLACKBODY:
            x = x.reshape(-1)
            shape = (x.shape[0], 3)
        else:
            x = x.reshape(-1)
            shape = x.shape
        out = np.zeros(shape)
        self._check(self.lib.bh_gpu_eval(self._h, C.byref(c), what, x.ctypes.data_as(dp), x.shape[0],
                                         out.ctypes.data_as(dp)))
        return out

    def adjoint(self, cfg, target, per_ray: bool = False):
        """Loss sum((Y - target)^2) over the pixels of the binary64 frame of
        `cfg` (Y = CIE Y, W m^-2 sr^-1) and its gradient with respect to
        (spin, inclination, eddington, r_out), as a dict (bh_grad4's fields),
        the disc-edge term included (edge_* fields: its part).  With per_ray:
        also each ray's discrete-adjoint contribution (edge term not
        included), shape (n_rays, 4), and luminance, shape (n_rays,), in
        trace_rays order."""
        c = _as_c(cfg)
        t = np.ascontiguousarray(target, dtype=np.float32)
        if t.size != c.width * c.height:
            raise ValueError("target must hold width * height luminances")
        g = abi.bh_grad4()
        fp = C.POINTER(C.c_float)
        dp = C.POINTER(C.c_double)
        if not per_ray:
            self._check(self.lib.bh_gpu_adjoint(self._h, C.byref(c), t.ctypes.data_as(fp), C.byref(g)))
            return g.as_dict()
        s = max(1, c.sqrt_spp)
        n = c.width * c.height * s * s
        rg = np.empty((n, 4), dtype=np.float64)
        ry = np.empty(n, dtype=np.float64)
        self._check(self.lib.bh_gpu_adjoint_rays(self._h, C.byref(c), t.ctypes.data_as(fp), C.byref(g),
                                                 rg.ctypes.data_as(dp), ry.ctypes.data_as(dp)))
        return g.as_dict(), rg, ry

    # -- launch control ----------------------------------------------------------
    def set_launch(self, block_size=0, rays_per_thread=0, refill=0, blocks_per_sm=0, reg_variant=0,
                   precision: int = -1) -> None:
        """Launch shape of the trace kernel of `precision` (-1: both)."""
        p = abi.bh_launch_params(block_size, rays_per_thread, refill, blocks_per_sm, reg_variant)
        self._check(self.lib.bh_gpu_set_launch(self._h, precision, C.byref(p)))

    def get_launch(self, precision: int = abi.PRECISION_FP64) -> dict:
        p = abi.bh_launch_params()
        self._check(self.lib.bh_gpu_get_launch(self._h, precision, C.byref(p)))
        return {k: getattr(p, k) for k, _ in p._fields_}

    def autotune(self, cfg) -> tuple:
        """Sweep the launch shapes on `cfg`; keeps and returns (best, ms)."""
        c = _as_c(cfg)
        p = abi.bh_launch_params()
        ms = C.c_double(0.0)
        self._check(self.lib.bh_gpu_autotune(self._h, C.byref(c), C.byref(p), C.byref(ms)))
        return {k: getattr(p, k) for k, _ in p._fields_}, ms.value

    def autotune_batch(self, cfgs) -> tuple:
        """The launch-shape search on a batch of frames; keeps and returns (best, ms)."""
        cs = (abi.bh_render_config * len(cfgs))(*[_as_c(c) for c in cfgs])
        p = abi.bh_launch_params()
        ms = C.c_double(0.0)
        self._check(self.lib.bh_gpu_autotune_batch(self._h, cs, len(cfgs), C.byref(p), C.byref(ms)))
        return {k: getattr(p, k) for k, _ in p._fields_}, ms.value

    def set_step_budget(self, budget: int) -> None:
        self._check(self.lib.bh_gpu_set_step_budget(self._h, budget))

    def request_abort(self) -> None:
        self.lib.bh_gpu_request_abort(self._h)

    def clear_abort(self) -> None:
        self.lib.bh_gpu_clear_abort(self._h)


def fma_peak_tflops(device: int = 0, precision: int = abi.PRECISION_MIXED) -> float:
    """Measured FMA throughput (TFLOP/s) in binary32 (MIXED) or binary64 (FP64)."""
    v = C.c_double(0.0)
    rc = load_library().bh_gpu_fma_peak(device, precision, C.byref(v))
    if rc != abi.OK:
        raise BHError(rc, "bh_gpu_fma_peak failed")
    return v.value


def star_catalogue(count: int, seed: int, sky_mode: int = abi.SKY_GALACTIC) -> np.ndarray:
    """The catalogue the render path uses: (count, 6) = x, y, z, mag, T, irradiance."""
    out = np.empty((count, 6), dtype=np.float64)
    rc = load_library().bh_star_catalogue(count, seed, sky_mode, out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != abi.OK:
        raise BHError(rc, "bh_star_catalogue failed")
    return out


def blackbody_table() -> np.ndarray:
    """ln X, ln Y, ln Z of the 4096-entry blackbody table, shape (3, 4096)."""
    out = np.empty((3, 4096), dtype=np.float64)
    rc = load_library().bh_blackbody_table(out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != abi.OK:
        raise BHError(rc, "bh_blackbody_table failed")
    return out


_default: Renderer | None = None


def render(cfg: RenderConfig, stats: RenderStats | None = None) -> np.ndarray:
    """Module-level drop-in for bh::render on GPU 0."""
    global _default
    if _default is None:
        _default = Renderer(0)
    return _default.render(cfg, stats)
