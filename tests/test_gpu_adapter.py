"""Pixels through the drop-in adapter bh::render_gpu, on the GPU.

The adapter (blackhole_b200/adapter/render_gpu.cpp, compiled against the
reference's headers into oracle/_ref/libbh_adapter_check.so) renders the
256x256 plain FP64 scene (a = 0.9, 60 deg, disc r_isco..30 M at 0.1
Eddington, M = 4.3e6 M_sun) as main.cpp's `--gpu` branch would, on the
reference's own sky and horizon stop: its image must equal bh_gpu_render's
bit for bit (it is the same call), and match the reference's own bh::render
of the same bh::RenderConfig to the FP64 parity tolerance.
"""
import ctypes as C

import numpy as np
import pytest

from blackhole_b200 import Renderer, RenderStats, abi, workloads
from test_adapter import adapter

pytestmark = pytest.mark.gpu


def test_adapter_renders_the_reference_frame():
    lib = adapter()
    cfg = workloads.kerr_fp64_256()
    cfg.sky_mode = abi.SKY_GALACTIC
    cfg.stop_mode = abi.STOP_REFERENCE
    c = cfg.to_c()
    n = cfg.width * cfg.height
    via = np.zeros((cfg.height, cfg.width, 3))
    st = abi.bh_render_stats()
    rc = lib.adc_render_gpu(C.byref(c), via.ctypes.data_as(C.POINTER(abi.bh_xyz)), C.byref(st), abi.PRECISION_FP64)
    lib.adc_release()
    assert rc == abi.OK, abi.STATUS_NAMES.get(rc, rc)
    assert st.rays == n and st.steps > 0 and st.seconds > 0
    with Renderer(0) as r:
        direct = r.render(cfg, RenderStats())
    assert np.array_equal(via, direct)
    ref = np.zeros_like(via)
    rs = abi.bh_render_stats()
    assert lib.adc_render_ref(C.byref(c), ref.ctypes.data_as(C.POINTER(abi.bh_xyz)), C.byref(rs)) == abi.OK
    assert rs.rays == n
    lit = ref[..., 1] > 0
    rel = np.abs(via[..., 1][lit] - ref[..., 1][lit]) / ref[..., 1][lit]
    assert np.quantile(rel, 0.99) <= 1e-6, np.quantile(rel, 0.99)
    assert (via[~lit] == 0).mean() > 0.99
    for got, want in ((st.captured, rs.captured), (st.disc_hits, rs.disc_hits), (st.escaped, rs.escaped)):
        assert abs(got - want) <= max(3, 0.001 * n)
    assert abs(st.steps - rs.steps) / rs.steps < 0.01


def test_adapter_mixed_precision_is_the_libraries_mixed_frame():
    lib = adapter()
    cfg = workloads.kerr_fp64_256()
    cfg.sky_mode = abi.SKY_GALACTIC      # bh::RenderConfig has the reference's sky and stop only
    cfg.stop_mode = abi.STOP_REFERENCE
    c = cfg.to_c()
    via = np.zeros((cfg.height, cfg.width, 3))
    st = abi.bh_render_stats()
    rc = lib.adc_render_gpu(C.byref(c), via.ctypes.data_as(C.POINTER(abi.bh_xyz)), C.byref(st), abi.PRECISION_MIXED)
    lib.adc_release()
    assert rc == abi.OK
    with Renderer(0) as r:
        cfg.precision = abi.PRECISION_MIXED
        assert np.array_equal(via, r.render(cfg))
