"""ctypes mirror of include/bh_gpu.h.

The field order and types here must match the C header exactly; the
library checks ``struct_size`` and ``abi_version`` on every call, and
tests/test_abi.py compares these layouts against the compiled header.
"""
from __future__ import annotations

import ctypes as C

ABI_VERSION = 3

# Status codes (bh_gpu.h).
OK = 0
ERR_INVALID_ARG = -1
ERR_CUDA = -2
ERR_BUDGET = -3
ERR_ABORTED = -4
ERR_NO_DEVICE = -5
ERR_UNSUPPORTED = -6
ERR_OUT_OF_MEMORY = -7

STATUS_NAMES = {
    OK: "BH_OK",
    ERR_INVALID_ARG: "BH_ERR_INVALID_ARG",
    ERR_CUDA: "BH_ERR_CUDA",
    ERR_BUDGET: "BH_ERR_BUDGET",
    ERR_ABORTED: "BH_ERR_ABORTED",
    ERR_NO_DEVICE: "BH_ERR_NO_DEVICE",
    ERR_UNSUPPORTED: "BH_ERR_UNSUPPORTED",
    ERR_OUT_OF_MEMORY: "BH_ERR_OUT_OF_MEMORY",
}

# Termination classes, in the order of Hit::What (render.cpp:37).
HIT_HORIZON, HIT_DISC, HIT_SUN, HIT_STAR, HIT_SKY, HIT_EXHAUSTED = range(6)
# Display tone curves, in img::ToneMap order (image.h:16).
TONEMAP_LINEAR, TONEMAP_REINHARD, TONEMAP_ACES, TONEMAP_LOG, TONEMAP_HDR = range(5)
EVAL_RHS, EVAL_DISC_TEMPERATURE, EVAL_BLACKBODY, EVAL_FRAME = range(4)
STEP_LIMIT_AUTO, STEP_LIMIT_REFERENCE, STEP_LIMIT_NONE = range(3)
CAPTURE_AUTO, CAPTURE_REFERENCE = range(2)
NEAR_CRITICAL_AUTO, NEAR_CRITICAL_BINARY32 = range(2)
TONEMAP_NAMES = ("linear", "reinhard", "aces", "log", "hdr")
HIT_NAMES = ("Horizon", "Disc", "Sun", "Star", "Sky", "Exhausted")

PRECISION_FP64 = 0
PRECISION_MIXED = 1
SKY_GALACTIC = 0
SKY_UNIFORM = 1
STOP_REFERENCE = 0
STOP_RELATIVE = 1


class bh_xyz(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class bh_camera(C.Structure):
    _fields_ = [
        ("r", C.c_double), ("theta", C.c_double), ("phi", C.c_double),
        ("fov", C.c_double), ("yaw", C.c_double), ("pitch", C.c_double), ("roll", C.c_double),
    ]


class bh_sun(C.Structure):
    _fields_ = [("centre", C.c_double * 3), ("radius", C.c_double), ("T_eff", C.c_double)]


class bh_hotspot(C.Structure):
    _fields_ = [
        ("enabled", C.c_int32), ("sense", C.c_int32),
        ("r", C.c_double), ("phi0", C.c_double), ("sigma", C.c_double),
        ("contrast", C.c_double), ("omega", C.c_double),
    ]


class bh_neutron_star(C.Structure):
    _fields_ = [
        ("enabled", C.c_int32), ("caps", C.c_int32),
        ("M_kg", C.c_double), ("R_m", C.c_double), ("R", C.c_double),
        ("T_eff", C.c_double), ("spin_hz", C.c_double), ("Omega", C.c_double),
        ("cap_tilt", C.c_double), ("cap_radius", C.c_double), ("cap_T", C.c_double),
        ("cap_phase0", C.c_double),
        ("two_caps", C.c_int32), ("reserved", C.c_int32),
    ]


JET_PARAMS = ("z_base", "z_top", "R_base", "k", "gamma_max", "z_sat", "alpha", "u_peak", "u_wid", "spine",
              "spine_wid", "zeta", "eps_rad", "phi_flux")
JET_CONFIGURED = ("a", "Omega_F", "P_jet", "L_rad", "j_nu0", "r_bound", "volume_rg3")


class bh_jet(C.Structure):
    _fields_ = [(k, C.c_double) for k in JET_PARAMS + JET_CONFIGURED]


class bh_render_config(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("abi_version", C.c_uint32),
        ("M_kg", C.c_double), ("spin", C.c_double),
        ("cam", bh_camera),
        ("width", C.c_int32), ("height", C.c_int32), ("sqrt_spp", C.c_int32),
        ("disc_enabled", C.c_int32),
        ("disc_r_out", C.c_double), ("eddington", C.c_double),
        ("disc_sense", C.c_int32), ("stars_enabled", C.c_int32),
        ("star_count", C.c_int32), ("sun_enabled", C.c_int32),
        ("seed", C.c_uint64),
        ("sun", bh_sun),
        ("hotspot", bh_hotspot),
        ("star", bh_neutron_star),
        ("jet_enabled", C.c_int32), ("reserved0", C.c_int32),
        ("observer_time", C.c_double),
        ("rtol", C.c_double), ("atol", C.c_double), ("r_escape", C.c_double),
        ("max_steps", C.c_int32),
        ("threads", C.c_int32), ("quiet", C.c_int32),
        ("precision", C.c_int32), ("sky_mode", C.c_int32), ("stop_mode", C.c_int32),
        ("milky_way", C.c_int32),
        ("stop_epsilon", C.c_double),
        ("mixed_rtol", C.c_double), ("mixed_atol", C.c_double),
        ("jet", bh_jet),
        ("mixed_step_limit", C.c_int32), ("mixed_capture", C.c_int32), ("mixed_near_critical", C.c_int32),
    ]


class bh_render_stats(C.Structure):
    _fields_ = [
        ("rays", C.c_longlong), ("steps", C.c_longlong), ("captured", C.c_longlong),
        ("disc_hits", C.c_longlong), ("sun_hits", C.c_longlong), ("star_hits", C.c_longlong),
        ("jet_rays", C.c_longlong), ("escaped", C.c_longlong), ("exhausted", C.c_longlong),
        ("max_norm_error", C.c_double), ("max_carter_drift", C.c_double),
        ("seconds", C.c_double), ("total_flux", C.c_double),
        ("attempts", C.c_longlong), ("kernel_ms", C.c_double), ("shade_ms", C.c_double),
        ("h2d_bytes", C.c_longlong), ("d2h_bytes", C.c_longlong),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class bh_ray_result(C.Structure):
    _fields_ = [
        ("what", C.c_int32), ("steps", C.c_int32),
        ("y", C.c_double * 8), ("g", C.c_double), ("dir", C.c_double * 3),
        ("xyz", bh_xyz),
        ("attempts", C.c_int32), ("reserved", C.c_int32),
        ("max_norm", C.c_double), ("max_q", C.c_double),
        ("jet", C.c_double),
    ]


class bh_launch_params(C.Structure):
    _fields_ = [
        ("block_size", C.c_int32), ("rays_per_thread", C.c_int32),
        ("refill", C.c_int32), ("blocks_per_sm", C.c_int32),
        ("reg_variant", C.c_int32),
    ]


class bh_trace_record(C.Structure):
    _fields_ = [
        ("y", C.c_double * 8), ("max_norm", C.c_double), ("max_q", C.c_double),
        ("what", C.c_int32), ("steps", C.c_int32), ("attempts", C.c_int32), ("reserved", C.c_int32),
    ]


NOALLOC_MAX_RAYS = 65536


class bh_display(C.Structure):
    _fields_ = [
        ("exposure", C.c_double), ("key", C.c_double), ("glare", C.c_double),
        ("glare_radius", C.c_double), ("log_decades", C.c_double),
        ("tonemap", C.c_int32), ("reserved", C.c_int32),
    ]


class bh_grad4(C.Structure):
    _fields_ = [
        ("loss", C.c_double), ("d_spin", C.c_double), ("d_inclination", C.c_double),
        ("d_eddington", C.c_double), ("d_r_out", C.c_double), ("kernel_ms", C.c_double),
        ("rays", C.c_longlong), ("steps", C.c_longlong), ("replayed_steps", C.c_longlong),
        ("disc_rays", C.c_longlong), ("sky_rays", C.c_longlong),
        ("max_checkpoint_interval", C.c_int32), ("reserved", C.c_int32),
        ("edge_spin", C.c_double), ("edge_inclination", C.c_double),
        ("edge_candidates", C.c_longlong), ("edge_cells", C.c_longlong), ("edge_steps", C.c_longlong),
        ("held_spin", C.c_double), ("held_inclination", C.c_double), ("high_order_rays", C.c_longlong),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


def trace_record_dtype():
    import numpy as np

    return np.dtype({
        "names": ["y", "max_norm", "max_q", "what", "steps", "attempts"],
        "formats": [(np.float64, 8), np.float64, np.float64, np.int32, np.int32, np.int32],
        "offsets": [0, 64, 72, 80, 84, 88],
        "itemsize": C.sizeof(bh_trace_record),
    })


def work_order(width: int, height: int, sqrt_spp: int):
    """Row-major sample index (pixel row-major, then sample) of each ray id in
    the library's work order (bands of four rows, column by column)."""
    import numpy as np

    s = max(1, sqrt_spp)
    ss = s * s
    p = np.arange(width * height, dtype=np.int64)
    band = p // (4 * width)
    rel = p - band * 4 * width
    bh = np.minimum(4, height - 4 * band)
    x = rel // bh
    y = 4 * band + rel % bh
    pix = y * width + x
    return (pix[:, None] * ss + np.arange(ss)[None, :]).reshape(-1)


# numpy dtype of bh_ray_result, for zero-copy views of result arrays.
def ray_result_dtype():
    import numpy as np

    return np.dtype(
        {
            "names": ["what", "steps", "y", "g", "dir", "xyz", "attempts", "max_norm", "max_q", "jet"],
            "formats": [np.int32, np.int32, (np.float64, 8), np.float64, (np.float64, 3), (np.float64, 3),
                        np.int32, np.float64, np.float64, np.float64],
            "offsets": [0, 4, 8, 72, 80, 104, 128, 136, 144, 152],
            "itemsize": C.sizeof(bh_ray_result),
        }
    )
