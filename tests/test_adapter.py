"""The drop-in adapter bh::render_gpu, compiled against the reference's headers.

blackhole_b200/adapter/render_gpu.cpp is what a maintainer adds to the
reference to give its main.cpp a `--gpu` flag (render.h:72 -> the C-ABI).
oracle/Makefile compiles it against the reference's own render.h and the
structs it includes (the build asserts the reference structs' sizes, so a
field added there stops it), with the reference's render.cpp, into
oracle/_ref/libbh_adapter_check.so.  Without a GPU these tests check that
every field of the reference's RenderConfig crosses to bh_render_config and
back unchanged, and that a render fails with BH_ERR_NO_DEVICE; the pixels
through the adapter are checked on the GPU (tests/test_gpu_adapter.py).
"""
import ctypes as C
import os

import pytest

from blackhole_b200 import abi, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER_SO = os.path.join(ROOT, "oracle", "_ref", "libbh_adapter_check.so")

# bh_render_config fields the reference's RenderConfig does not have (their
# values come from bh_render_config_default), or that are bookkeeping.
EXTENSIONS = ("struct_size", "abi_version", "reserved0", "star.reserved", "precision", "sky_mode", "stop_mode", "milky_way",
              "stop_epsilon", "mixed_rtol", "mixed_atol", "mixed_step_limit", "mixed_capture",
              "mixed_near_critical")
# int32 fields that are bool in the reference.
FLAGS = ("disc_enabled", "stars_enabled", "sun_enabled", "jet_enabled", "quiet",
         "hotspot.enabled", "star.enabled", "star.caps", "star.two_caps")


def adapter():
    if not os.path.exists(ADAPTER_SO):
        pytest.skip("the adapter harness oracle/_ref/libbh_adapter_check.so was not built here "
                    "(it needs the reference's sources)")
    lib = C.CDLL(ADAPTER_SO)
    P = C.POINTER(abi.bh_render_config)
    lib.adc_roundtrip.argtypes = [P, P, C.c_int]
    lib.adc_render_gpu.argtypes = [P, C.POINTER(abi.bh_xyz), C.POINTER(abi.bh_render_stats), C.c_int]
    lib.adc_render_ref.argtypes = [P, C.POINTER(abi.bh_xyz), C.POINTER(abi.bh_render_stats)]
    return lib


def _leaves(struct, prefix=""):
    """(dotted name, owner, field, index) of every scalar of a ctypes struct."""
    for name, typ in struct._fields_:
        v = getattr(struct, name)
        full = prefix + name
        if isinstance(v, C.Structure):
            yield from _leaves(v, full + ".")
        elif isinstance(v, C.Array):
            for i in range(len(v)):
                yield f"{full}[{i}]", v, None, i
        else:
            yield full, struct, name, None


def _get(owner, field, idx):
    return owner[idx] if field is None else getattr(owner, field)


def _set(owner, field, idx, val):
    if field is None:
        owner[idx] = val
    else:
        setattr(owner, field, val)


def test_every_reference_field_crosses_the_adapter_unchanged():
    lib = adapter()
    base = gpu.default_config_c()
    for flag_value in (0, 1):
        src = abi.bh_render_config.from_buffer_copy(base)
        k = 0
        for name, owner, field, idx in _leaves(src):
            if name.split("[")[0] in EXTENSIONS:
                continue
            k += 1
            if name in FLAGS:
                _set(owner, field, idx, flag_value)
            elif isinstance(_get(owner, field, idx), float):
                _set(owner, field, idx, 1.0 + 0.001 * k)      # a distinct value per field
            else:
                _set(owner, field, idx, 100 + k)
        out = abi.bh_render_config()
        assert lib.adc_roundtrip(C.byref(src), C.byref(out), abi.PRECISION_MIXED) == abi.OK
        for (name, o1, f1, i1), (_, o2, f2, i2) in zip(_leaves(src), _leaves(out)):
            if name == "precision":
                assert _get(o2, f2, i2) == abi.PRECISION_MIXED
            elif name.split("[")[0] in EXTENSIONS:
                d = dict((n, (o, f, i)) for n, o, f, i in _leaves(base))[name]
                assert _get(o2, f2, i2) == _get(*d), name      # the library's default
            else:
                assert _get(o2, f2, i2) == _get(o1, f1, i1), name


def test_render_without_a_gpu_reports_no_device():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present: the adapter renders (tests/test_gpu_adapter.py)")
    except ImportError:
        pass
    lib = adapter()
    c = gpu.default_config_c()
    c.width = c.height = 4
    px = (abi.bh_xyz * 16)()
    st = abi.bh_render_stats()
    assert lib.adc_render_gpu(C.byref(c), px, C.byref(st), abi.PRECISION_FP64) == abi.ERR_NO_DEVICE
