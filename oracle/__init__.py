"""CPU oracle of the geodesic render path (test infrastructure).

Loads oracle/lib/libbh_oracle.so (the plain-C restatement) and, when it was
built, oracle/_ref/libbh_ref.so (the reference renderer compiled from its own
sources).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
use this module, and only as the checker; the GPU library never links it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from blackhole_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "lib", "libbh_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbh_ref.so")
# The reference's src/ directory: $BH_REFERENCE_SRC, else a checkout named
# `reference` beside this repository (the same rule as oracle/Makefile).
REF_SRC = os.environ.get("BH_REFERENCE_SRC") or os.path.join(os.path.dirname(os.path.dirname(HERE)),
                                                             "reference", "src")

_oracle = None
_ref = None

_D = C.c_double
_PD = C.POINTER(C.c_double)
_CFG = C.POINTER(abi.bh_render_config)
_ST = C.POINTER(abi.bh_render_stats)
_RR = C.POINTER(abi.bh_ray_result)


def build(force: bool = False) -> None:
    """Compile the restatement (and the reference harness where the reference
    sources exist) with oracle/Makefile."""
    if force or not os.path.exists(ORACLE_SO) or (
        os.path.isdir(REF_SRC) and not os.path.exists(REF_SO)
    ):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


def _declare(lib, prefix: str) -> None:
    def fn(name, res, *args):
        f = getattr(lib, prefix + name, None)
        if f is None:
            return
        f.restype = res
        f.argtypes = list(args)

    fn("metric_upper_deriv", None, _D, _D, _D, _PD)
    fn("metric_upper", None, _D, _D, _D, _PD)
    fn("metric_lower", None, _D, _D, _D, _PD)
    fn("geodesic_rhs", None, _D, _PD, _PD)
    fn("horizon_outer", _D, _D)
    fn("horizon_inner", _D, _D)
    fn("isco_radius", _D, _D, C.c_int)
    fn("photon_circular_orbit", _D, _D, C.c_int)
    fn("circular_energy", _D, _D, _D, C.c_int)
    fn("circular_angmom", _D, _D, _D, C.c_int)
    fn("disc_efficiency", _D, _D, C.c_int)
    fn("keplerian_four_velocity", None, _D, _D, C.c_int, _PD)
    fn("zamo_tetrad", None, _D, _D, _D, _PD)
    fn("carter_constant", _D, _D, _D, _D, _D, _D)
    fn("make_photon", None, _D, _D, _D, _D, _PD, _PD)
    fn("invariants", None, _D, _PD, _PD)
    fn("integrate", C.c_long, _D, _PD, _D, _D, _D, C.c_int, _D, _D, _PD)
    fn("page_thorne_W", _D, _D, _D, _D)
    fn("disc_temperature", _D, _D, _D, _D, _D, C.c_int, _D)
    fn("planck_radiance", _D, _D, _D)
    fn("blackbody_xyz_exact", None, _D, _PD)
    fn("blackbody_xyz", None, _D, _PD)
    fn("bv_to_temperature", _D, _D)
    fn("blackbody_table", None, _PD)
    fn("ray_direction", None, C.POINTER(abi.bh_camera), _D, _D, _D, _PD)
    fn("trace_rays", C.c_int, _CFG, C.c_int, C.c_int, C.c_int, C.c_int, _RR, _ST)
    fn("trace_rows", C.c_int, _CFG, C.POINTER(C.c_int), C.c_int, C.c_int, _RR, _ST)
    fn("render_window", C.c_int, _CFG, C.c_int, C.c_int, C.c_int, C.c_int,
       C.POINTER(abi.bh_xyz), _ST)
    fn("render", C.c_int, _CFG, C.POINTER(abi.bh_xyz), _ST)
    fn("render_rows", C.c_int, _CFG, C.POINTER(C.c_int), C.c_int, C.c_int,
       C.POINTER(abi.bh_xyz), _ST, _PD)
    _PJ = C.POINTER(abi.bh_jet)
    fn("jet_configure", None, _PJ, _D, _D, _D)
    fn("powerlaw_xyz", None, _D, _PD)
    fn("jet_shape", _D, _PJ, _D, _D)
    fn("jet_four_velocity", None, _PJ, _D, _D, _D, _PD)
    _PX = C.POINTER(abi.bh_xyz)
    _U8 = C.POINTER(C.c_uint8)
    if prefix == "orc_":
        fn("auto_exposure", _D, _PX, C.c_long, _D)
        fn("add_glare", None, _PX, C.c_int, C.c_int, _D, _D)
        fn("develop", None, _PX, C.c_long, _D, C.c_int, _D, _U8)
    else:
        fn("auto_exposure", _D, _PX, C.c_int, C.c_int, _D)
        fn("add_glare", None, _PX, C.c_int, C.c_int, _D, _D)
        fn("develop", None, _PX, C.c_int, C.c_int, _D, C.c_int, _D, _U8)
    if prefix == "orc_":
        fn("star_catalogue", C.c_int, C.c_int, C.c_uint64, C.c_int, _PD)
        fn("sky_radiance", C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int, _PD, C.c_int, _D, _PD)
    else:
        fn("star_catalogue", C.c_int, C.c_int, C.c_uint64, _PD)
        fn("sky_radiance", C.c_int, C.c_int, C.c_uint64, C.c_int, _PD, C.c_int, _D, _PD)


def oracle_lib():
    """The restatement (always available once built)."""
    global _oracle
    if _oracle is None:
        build()
        _oracle = C.CDLL(ORACLE_SO)
        _declare(_oracle, "orc_")
    return _oracle


def ref_lib():
    """The reference renderer harness, or None where it was never built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO) and os.path.isdir(REF_SRC):
            build()
        if not os.path.exists(REF_SO):
            return None
        _ref = C.CDLL(REF_SO)
        _declare(_ref, "ref_")
    return _ref


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_PD)


class Port:
    """numpy-friendly calls into one of the two libraries ('orc_' or 'ref_')."""

    def __init__(self, lib, prefix: str):
        self.lib = lib
        self.prefix = prefix

    def _f(self, name):
        return getattr(self.lib, self.prefix + name)

    def has(self, name: str) -> bool:
        return hasattr(self.lib, self.prefix + name)

    def metric_upper_deriv(self, a, r, th):
        out = np.zeros(15)
        self._f("metric_upper_deriv")(a, r, th, _ptr(out))
        return out

    def metric_lower(self, a, r, th):
        out = np.zeros(5)
        self._f("metric_lower")(a, r, th, _ptr(out))
        return out

    def geodesic_rhs(self, a, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros(8)
        self._f("geodesic_rhs")(a, _ptr(y), _ptr(out))
        return out

    def make_photon(self, a, r, th, phi, d):
        d = np.ascontiguousarray(d, dtype=np.float64)
        out = np.zeros(8)
        self._f("make_photon")(a, r, th, phi, _ptr(d), _ptr(out))
        return out

    def invariants(self, a, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros(5)
        self._f("invariants")(a, _ptr(y), _ptr(out))
        return out

    def blackbody_xyz(self, T):
        out = np.zeros(3)
        self._f("blackbody_xyz")(T, _ptr(out))
        return out

    def blackbody_xyz_exact(self, T):
        out = np.zeros(3)
        self._f("blackbody_xyz_exact")(T, _ptr(out))
        return out

    def blackbody_table(self):
        out = np.zeros((3, 4096))
        self._f("blackbody_table")(_ptr(out))
        return out

    def star_catalogue(self, count, seed, sky_mode=abi.SKY_GALACTIC):
        out = np.zeros((count, 6))
        if self.prefix == "orc_":
            rc = self._f("star_catalogue")(count, seed, sky_mode, _ptr(out))
        else:
            if sky_mode != abi.SKY_GALACTIC:
                raise ValueError("the reference has only the galactic sky")
            rc = self._f("star_catalogue")(count, seed, _ptr(out))
        if rc != 0:
            raise RuntimeError(f"star_catalogue failed: {rc}")
        return out

    def sky_radiance(self, count, seed, dirs, sigma, sky_mode=abi.SKY_GALACTIC, milky_way=1):
        dirs = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
        out = np.zeros((len(dirs), 3))
        if self.prefix == "orc_":
            rc = self._f("sky_radiance")(count, seed, sky_mode, milky_way, _ptr(dirs), len(dirs),
                                         sigma, _ptr(out))
        else:
            rc = self._f("sky_radiance")(count, seed, milky_way, _ptr(dirs), len(dirs), sigma,
                                         _ptr(out))
        if rc != 0:
            raise RuntimeError(f"sky_radiance failed: {rc}")
        return out

    def trace_rays(self, cfg, x0=0, y0=0, w=None, h=None):
        """Per-sample results of a window as a structured numpy array, plus stats."""
        c = cfg.to_c() if hasattr(cfg, "to_c") else cfg
        w = c.width - x0 if w is None else w
        h = c.height - y0 if h is None else h
        s = max(1, c.sqrt_spp)
        n = w * h * s * s
        buf = (abi.bh_ray_result * max(n, 1))()
        st = abi.bh_render_stats()
        rc = self._f("trace_rays")(C.byref(c), x0, y0, w, h, buf, C.byref(st))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}trace_rays failed: {abi.STATUS_NAMES.get(rc, rc)}")
        arr = np.frombuffer(buf, dtype=abi.ray_result_dtype(), count=n).copy()
        return arr, st

    def trace_rows(self, cfg, rows, threads=0):
        """Per-sample results of whole rows (in the listed order, each row
        pixel then sample) on `threads` workers (0: one per host core), plus
        stats."""
        c = cfg.to_c() if hasattr(cfg, "to_c") else cfg
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        s = max(1, c.sqrt_spp)
        n = len(rows) * c.width * s * s
        buf = (abi.bh_ray_result * max(n, 1))()
        st = abi.bh_render_stats()
        threads = threads if threads > 0 else (os.cpu_count() or 1)
        rc = self._f("trace_rows")(C.byref(c), rows.ctypes.data_as(C.POINTER(C.c_int)), len(rows), threads,
                                   buf, C.byref(st))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}trace_rows failed: {abi.STATUS_NAMES.get(rc, rc)}")
        return np.frombuffer(buf, dtype=abi.ray_result_dtype(), count=n).copy(), st

    def render_window(self, cfg, x0=0, y0=0, w=None, h=None):
        c = cfg.to_c() if hasattr(cfg, "to_c") else cfg
        w = c.width - x0 if w is None else w
        h = c.height - y0 if h is None else h
        out = np.zeros((h, w, 3))
        st = abi.bh_render_stats()
        rc = self._f("render_window")(C.byref(c), x0, y0, w, h,
                                      out.ctypes.data_as(C.POINTER(abi.bh_xyz)), C.byref(st))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}render_window failed: {abi.STATUS_NAMES.get(rc, rc)}")
        return out, st

    def render(self, cfg):
        """The reference's own bh::render (only in the reference harness)."""
        c = cfg.to_c() if hasattr(cfg, "to_c") else cfg
        out = np.zeros((c.height, c.width, 3))
        st = abi.bh_render_stats()
        rc = self._f("render")(C.byref(c), out.ctypes.data_as(C.POINTER(abi.bh_xyz)), C.byref(st))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}render failed: {abi.STATUS_NAMES.get(rc, rc)}")
        return out, st

    def render_rows(self, cfg, rows, threads=0):
        """The reference's trace()+shade() over the given rows on `threads`
        workers; returns (pixels[len(rows), W, 3], stats, setup_seconds)."""
        c = cfg.to_c() if hasattr(cfg, "to_c") else cfg
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        out = np.zeros((len(rows), c.width, 3))
        st = abi.bh_render_stats()
        setup = C.c_double(0.0)
        rc = self._f("render_rows")(C.byref(c), rows.ctypes.data_as(C.POINTER(C.c_int)), len(rows),
                                    threads, out.ctypes.data_as(C.POINTER(abi.bh_xyz)), C.byref(st),
                                    C.byref(setup))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}render_rows failed: {abi.STATUS_NAMES.get(rc, rc)}")
        return out, st, setup.value

    # -- jets (jet.h:77-315) --------------------------------------------------------
    def jet_configure(self, jet_c, spin, mdot_c2, r_g_m):
        """Jet::configure on a copy of a bh_jet; returns the copy."""
        j = abi.bh_jet.from_buffer_copy(jet_c)
        self._f("jet_configure")(C.byref(j), spin, mdot_c2, r_g_m)
        return j

    def powerlaw_xyz(self, alpha):
        out = np.zeros(3)
        self._f("powerlaw_xyz")(alpha, _ptr(out))
        return out

    def jet_shape(self, jet_c, z, rho):
        return self._f("jet_shape")(C.byref(jet_c), z, rho)

    def jet_four_velocity(self, jet_c, a, r, th):
        out = np.zeros(4)
        self._f("jet_four_velocity")(C.byref(jet_c), a, r, th, _ptr(out))
        return out

    # -- display transform (image.cpp:22-191) ------------------------------------
    @staticmethod
    def _img(xyz):
        a = np.ascontiguousarray(xyz, dtype=np.float64)
        if a.ndim != 3 or a.shape[2] != 3:
            raise ValueError("image must be (height, width, 3)")
        return a

    def auto_exposure(self, xyz, key=1.0):
        a = self._img(xyz)
        px = a.ctypes.data_as(C.POINTER(abi.bh_xyz))
        if self.prefix == "orc_":
            return self._f("auto_exposure")(px, a.shape[0] * a.shape[1], key)
        return self._f("auto_exposure")(px, a.shape[1], a.shape[0], key)

    def add_glare(self, xyz, strength, radius_px):
        """The glared copy of the image."""
        a = self._img(xyz).copy()
        self._f("add_glare")(a.ctypes.data_as(C.POINTER(abi.bh_xyz)), a.shape[1], a.shape[0], strength, radius_px)
        return a

    def develop(self, xyz, exposure, tonemap=abi.TONEMAP_HDR, log_decades=16.0):
        a = self._img(xyz)
        out = np.empty((a.shape[0], a.shape[1], 3), dtype=np.uint8)
        px = a.ctypes.data_as(C.POINTER(abi.bh_xyz))
        u8 = out.ctypes.data_as(C.POINTER(C.c_uint8))
        if self.prefix == "orc_":
            self._f("develop")(px, a.shape[0] * a.shape[1], exposure, tonemap, log_decades, u8)
        else:
            self._f("develop")(px, a.shape[1], a.shape[0], exposure, tonemap, log_decades, u8)
        return out

    def scalar(self, name, *args):
        return self._f(name)(*args)


def oracle() -> Port:
    return Port(oracle_lib(), "orc_")


def reference():
    lib = ref_lib()
    return Port(lib, "ref_") if lib is not None else None
