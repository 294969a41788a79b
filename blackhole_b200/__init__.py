"""B200-native geodesic render path of the Kerr ray tracer.

The package mirrors the reference's render surface (render.h): ``RenderConfig``,
``Camera``, ``RenderStats`` and ``render()``, with the work done by the
sm_100a kernels in ``lib/libbh_gpu.so`` behind the C-ABI of
``include/bh_gpu.h``.
"""
from . import abi
from .config import Camera, HotSpot, NeutronStar, RenderConfig, RenderStats, SunBody
from .gpu import BHError, Renderer, load_library, render

__all__ = [
    "abi", "Camera", "HotSpot", "NeutronStar", "RenderConfig", "RenderStats", "SunBody",
    "BHError", "Renderer", "load_library", "render",
]
