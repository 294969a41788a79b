"""The C-ABI library: loads without a GPU, exports every declared symbol, and
its struct layouts match the ctypes mirror."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from blackhole_b200 import abi, gpu
from blackhole_b200.config import RenderConfig

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bh_gpu.h")


def _declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bh_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = gpu.load_library()
    names = _declared()
    assert "bh_gpu_render" in names and len(names) >= 15
    nm = subprocess.run(["nm", "-D", "--defined-only", gpu.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (bh_\w+)", nm))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert hasattr(lib, n)


def test_abi_version():
    assert gpu.load_library().bh_gpu_abi_version() == abi.ABI_VERSION


STRUCTS = {
    "bh_render_config": abi.bh_render_config,
    "bh_render_stats": abi.bh_render_stats,
    "bh_ray_result": abi.bh_ray_result,
    "bh_camera": abi.bh_camera,
    "bh_sun": abi.bh_sun,
    "bh_hotspot": abi.bh_hotspot,
    "bh_neutron_star": abi.bh_neutron_star,
    "bh_launch_params": abi.bh_launch_params,
    "bh_xyz": abi.bh_xyz,
    "bh_trace_record": abi.bh_trace_record,
    "bh_jet": abi.bh_jet,
    "bh_grad4": abi.bh_grad4,
    "bh_display": abi.bh_display,
}


def test_struct_layouts_match_header():
    """Compile a probe against the header and compare sizeof/offsetof with ctypes."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, cls in STRUCTS.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c11", src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.strip().splitlines())
    for cname, cls in STRUCTS.items():
        assert int(got[cname]) == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, f"{cname}.{fname}"


def test_default_config_matches_reference_defaults():
    """bh_render_config_default == RenderConfig() (render.h:15-53)."""
    c = gpu.default_config_c()
    p = RenderConfig().to_c()
    for name, _ in abi.bh_render_config._fields_:
        a, b = getattr(c, name), getattr(p, name)
        if isinstance(a, C.Structure):
            for sub, _ in a._fields_:
                x, y = getattr(a, sub), getattr(b, sub)
                if hasattr(x, "__len__"):
                    assert list(x) == list(y), f"{name}.{sub}"
                else:
                    assert x == y, f"{name}.{sub}"
        else:
            assert a == b, name


def test_catalogue_entry_point_matches_oracle(orc):
    for mode in (abi.SKY_GALACTIC, abi.SKY_UNIFORM):
        a = gpu.star_catalogue(5000, 99, mode)
        b = orc.star_catalogue(5000, 99, mode)
        assert np.array_equal(a, b)


def test_blackbody_table_entry_point_matches_oracle(orc):
    assert np.array_equal(gpu.blackbody_table(), orc.blackbody_table())


def test_create_without_gpu_fails_loudly():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    with pytest.raises(gpu.BHError) as e:
        gpu.Renderer(0)
    assert e.value.code == abi.ERR_NO_DEVICE


def test_enum_values_match_header():
    """Every BH_* constant of the header against its Python mirror."""
    txt = open(HEADER).read()
    names = sorted(set(re.findall(r"\b(BH_[A-Z0-9_]+)\s*=", txt)) | set(re.findall(r"#define (BH_[A-Z0-9_]+) ", txt)))
    lines = ['#include <stdio.h>', f'#include "{HEADER}"', "int main(void){"]
    lines += [f'printf("{n} %d\\n", (int){n});' for n in names]
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "enums.c")
        exe = os.path.join(d, "enums")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c11", src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = {k: int(v) for k, v in (line.split() for line in out.strip().splitlines())}
    assert len(got) >= 35
    for name, value in got.items():
        py = name[3:]
        if py == "GPU_ABI_VERSION":
            py = "ABI_VERSION"
        if hasattr(abi, py):
            assert getattr(abi, py) == value, name
    for py in ("OK", "ERR_INVALID_ARG", "HIT_SKY", "PRECISION_MIXED", "SKY_UNIFORM", "STOP_RELATIVE",
               "TONEMAP_HDR", "EVAL_FRAME", "STEP_LIMIT_NONE", "CAPTURE_REFERENCE", "NEAR_CRITICAL_BINARY32", "NOALLOC_MAX_RAYS"):
        assert got["BH_" + py] == getattr(abi, py), py
