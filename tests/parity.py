"""Per-sample comparison helpers for the parity tests.

A GPU result and a checker result (golden vectors or the oracle) are compared
ray by ray: termination class, redshift g of disc hits, final sky direction of
escaped rays and the sample's luminance Y.  Rays whose class differs are
counted separately: at class boundaries (shadow edge, disc edges, the photon
ring) an ulp of difference anywhere in the path legitimately changes the
outcome, as the oracle itself shows under perturbation.
"""
from __future__ import annotations

import numpy as np

from blackhole_b200 import abi


def window_of(full: np.ndarray, width: int, height: int, spp: int, x0: int, y0: int, w: int, h: int):
    """Per-sample results of a full frame (row-major pixel, then sample)
    restricted to a window, in the oracle's order."""
    ss = spp * spp
    a = full.reshape(height, width, ss)
    return a[y0:y0 + h, x0:x0 + w].reshape(-1)


def _has(x, key: str) -> bool:
    """Whether a structured array or a mapping (npz) has the field `key`."""
    names = getattr(getattr(x, "dtype", None), "names", None)
    return key in names if names is not None else key in x


def compare(gpu: np.ndarray, chk: dict) -> dict:
    """Error statistics of GPU samples against checker samples (same order)."""
    wg = gpu["what"].astype(np.int32)
    wc = np.asarray(chk["what"]).astype(np.int32)
    same = wg == wc
    out = {"n": int(len(wg)), "class_agree": float(same.mean()) if len(wg) else 1.0}

    disc = same & (wc == abi.HIT_DISC) & (np.asarray(chk["g"]) > 0)
    if disc.any():
        gc = np.asarray(chk["g"])[disc]
        out["g_rel"] = np.abs(gpu["g"][disc] - gc) / np.abs(gc)
    else:
        out["g_rel"] = np.zeros(0)
    sky = same & (wc == abi.HIT_SKY)
    if sky.any():
        dg = gpu["dir"][sky]
        dc = np.asarray(chk["dir"])[sky]
        # angle from the chord, stable for tiny angles
        out["dir_rad"] = 2.0 * np.arcsin(np.clip(np.linalg.norm(dg - dc, axis=1) / 2.0, 0.0, 1.0))
    else:
        out["dir_rad"] = np.zeros(0)
    lit = same & (np.asarray(chk["xyz"])[:, 1] > 0)
    if lit.any():
        yc = np.asarray(chk["xyz"])[lit, 1]
        out["Y_rel"] = np.abs(gpu["xyz"][lit, 1] - yc) / np.abs(yc)
    else:
        out["Y_rel"] = np.zeros(0)
    if _has(chk, "jet") and _has(gpu, "jet"):
        jc_all = np.asarray(chk["jet"])
        jl = same & (jc_all > 0)
        out["jet_rel"] = (np.abs(gpu["jet"][jl] - jc_all[jl]) / jc_all[jl]) if jl.any() else np.zeros(0)
        # no jet light where the checker has none, and vice versa
        out["jet_missing"] = int((same & ((jc_all > 0) != (gpu["jet"] > 0))).sum())
    else:
        out["jet_rel"] = np.zeros(0)
        out["jet_missing"] = 0
    steps = same & (wc != abi.HIT_HORIZON)
    out["steps_diff"] = np.abs(gpu["steps"][steps].astype(np.int64) - np.asarray(chk["steps"])[steps])
    return out


def q(x: np.ndarray, p: float) -> float:
    return float(np.quantile(x, p)) if len(x) else 0.0


def summary(s: dict) -> str:
    parts = [f"n={s['n']} class_agree={s['class_agree']:.4f}"]
    for k in ("g_rel", "dir_rad", "Y_rel", "jet_rel"):
        v = s[k]
        if len(v):
            parts.append(f"{k}: n={len(v)} p50={q(v, .5):.2e} p99={q(v, .99):.2e} max={v.max():.2e}")
    if len(s["steps_diff"]):
        parts.append(f"steps_diff: mean={s['steps_diff'].mean():.2f} max={s['steps_diff'].max()}")
    return " | ".join(parts)
