"""Benchmark of the GPU geodesic render path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One step renders one 1024x1024 frame of the near edge-on scene (a = 0.998,
inclination 85 deg, disc r_isco..50 M at 0.3 Eddington, M = 10 M_sun, +-25 M
field of view from r = 1000 M, one sample per pixel, seeded 250,000-star
uniform sky): 1,048,576 rays, traced in mixed precision.  The same frame in
plain FP64 is timed beside it, and the per-pixel error of the mixed frame
against the FP64 frame is reported.

Timing: W untimed warm-up steps, then K steps each bracketed by CUDA events on
the stream the kernels run on, with a 256 MiB write between steps to flush the
126 MB L2; barrier + synchronize around the timed loop; the maximum over ranks
is reported.  Under torchrun each rank renders its own frame (camera azimuth
2 pi rank / N): weak scaling with no collective on the data path.

`--impl reference` times the reference's own CPU implementation (the
reference renderer compiled from its sources, oracle/_ref) on the box's host
cores, on rows of the same frame.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "rays/s at 1024² on 1 B200: mixed vs FP64 plain at stated g/dir error; grads/s"
WORKLOAD = ("edge_on_1024: a=0.998, inclination 85 deg, 1024x1024, 1 spp, +-25 M from r=1000 M, "
            "disc r_isco..50 M at 0.3 Eddington, M=10 M_sun, 250k-star uniform sky + 21.5 mag/arcsec^2 "
            "background, escape 1.1 r_obs, horizon stop r_+(1+1e-6), rtol 1e-8 / atol 1e-10 (FP64), "
            "1e-6 / 1e-8 (mixed); FP64 under the reference's step cap, mixed under a loose cap "
            "h <= 0.3 max(1, r - r_+) with a rotation-invariant azimuth error scale and the escaping "
            "step landed within the reference cap of r_escape (no Sun, neutron star or jet in view), "
            "ingoing rays inside the innermost photon "
            "orbit ended as captured, and near-critical rays (escaping after circling close to the photon "
            "shell) traced in binary64 by a kernel beside the binary32 one")
L2_FLUSH_BYTES = 256 << 20
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "trace_kernel_traffic.txt")
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    p.add_argument("--size", type=int, default=1024, help="frame side (default 1024)")
    p.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison leg")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batch", action="store_true", help="skip the 64-frame batch leg")
    p.add_argument("--no-photon-ring", action="store_true", help="skip the 4096^2 photon-ring leg")
    p.add_argument("--no-adjoint", action="store_true", help="skip the 512^2 adjoint leg")
    p.add_argument("--no-display", action="store_true", help="skip the on-device display leg")
    p.add_argument("--no-jets", action="store_true", help="skip the jet and animation legs")
    p.add_argument("--leg", default=None, choices=["adjoint", "display", "jets"],
                   help="run one workload once (for profiling) and exit")
    p.add_argument("--once", action="store_true",
                   help="render the frame once in mixed precision and once in FP64 and exit (for ncu captures)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def frame_config(size: int, rank: int, world: int, precision: int):
    from blackhole_b200 import workloads

    cfg = workloads.edge_on_1024(precision=precision)
    cfg.width = cfg.height = size
    cfg.cam.phi = 2.0 * math.pi * rank / max(1, world)
    return cfg


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# the GPU arm
# ---------------------------------------------------------------------------

def time_device(r, cfg, steps, warmup, torch, flush, barrier):
    """Average device time of one render (CUDA events on the render stream)."""
    from blackhole_b200 import abi

    # A dedicated (non-default) stream: the kernels, the L2 flush and the
    # events all go on it, so the events bracket exactly the render's work.
    stream = torch.cuda.Stream()
    dev = torch.empty((cfg.height, cfg.width, 3), dtype=torch.float64, device="cuda")
    c = cfg.to_c()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            r.render_device(c, dev.data_ptr(), stream.cuda_stream)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        for i in range(steps):
            flush.add_(1.0)
            starts[i].record(stream)
            r.render_device(c, dev.data_ptr(), stream.cuda_stream)
            ends[i].record(stream)
        torch.cuda.synchronize()
    barrier()
    times = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    st = abi.bh_render_stats()
    r.render_device(c, dev.data_ptr(), stream.cuda_stream, stats=st)
    torch.cuda.synchronize()
    return sum(times), times, st, dev


def roofline(kernel_ms: float, steps: int, attempts: int, precision: str, peak: float, peak_src: str):
    from blackhole_b200 import flops

    per = flops.FLOPS_PER_STEP[precision]
    algo = per["alu_flop"] * steps          # accepted steps are the unit of work
    achieved = algo / (kernel_ms * 1e-3) / 1e12
    traffic = None
    if os.path.exists(PROFILE_TRAFFIC):
        for ln in open(PROFILE_TRAFFIC):
            if ln.startswith(f"{precision}_bytes_per_launch:"):
                try:
                    traffic = float(ln.split(":", 1)[1].strip())
                except ValueError:
                    pass
    return {
        "bound": "fp32-alu" if precision == "mixed" else "fp64-alu",
        "achieved": round(achieved, 3),
        "peak": round(peak, 3),
        "unit": "TFLOP/s",
        "frac": round(achieved / peak, 4) if peak > 0 else None,
        "traffic": traffic,
        "peak_source": peak_src,
        "flop_per_step": per["alu_flop"],
        "f64_flop_per_step": per["f64_flop"],
        "accepted_steps": steps,
        "attempts": attempts,
        "kernel_ms": round(kernel_ms, 4),
        # The HBM side of the same launch: the measured DRAM bytes against the
        # measured copy bandwidth (the path is not memory-bound).
        "hbm": hbm_side(traffic, kernel_ms),
    }


def hbm_side(traffic, kernel_ms):
    if traffic is None or not os.path.exists(MEASURED_PEAKS):
        return None
    try:
        peak = float(json.load(open(MEASURED_PEAKS))["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return None
    gbs = traffic / (kernel_ms * 1e-3) / 1e9
    return {"achieved": round(gbs, 2), "peak": peak, "unit": "GB/s", "frac": round(gbs / peak, 5),
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}


# Conditioning probe of a sky ray's final direction: the FP64 frame again with
# the camera turned by COND_YAW.  At r = 1000 M that turn moves each ray's
# image-plane impact parameter by 1.5e-7 M, the size of the change binary32
# rounding makes to a ray's constants of motion (E, L_z, p_th at ~3e-8
# relative).  A ray whose FP64 direction moves by more than COND_LIMIT under it
# cannot be resolved to 1e-4 rad from any binary32 state.
COND_YAW = 1.5e-10
COND_LIMIT = 1e-5


def accuracy(r, size, rank, world, cfgs=None):
    """Per-ray error of the mixed frame against the FP64 frame (same rays),
    with the conditioning probe of the sky rays."""
    import copy

    from blackhole_b200 import abi

    if cfgs is None:
        cfgs = (frame_config(size, rank, world, abi.PRECISION_FP64),
                frame_config(size, rank, world, abi.PRECISION_MIXED))
    a = r.trace_rays(cfgs[0])
    b = r.trace_rays(cfgs[1])
    turned = copy.deepcopy(cfgs[0])
    turned.cam.yaw += COND_YAW
    return compare_rays(a, b, probe=r.trace_rays(turned))


def _angle(u, v):
    """Angle between unit vectors, from the chord (stable for tiny angles)."""
    return 2.0 * np.arcsin(np.clip(np.linalg.norm(u - v, axis=1) / 2.0, 0.0, 1.0))


def _dist(e, tol):
    return {"p50": float(np.quantile(e, .5)), "p99": float(np.quantile(e, .99)),
            "p999": float(np.quantile(e, .999)), "max": float(e.max()), "n": int(e.size),
            "n_above_target": int((e > tol).sum())}


def conditioning(fp64, probe):
    """How far each ray's FP64 result moves when the camera turns by COND_YAW:
    the sky direction's angle for sky rays, |dg|/g for disc rays (inf where
    the turn changes the class).  fp64 and probe are GPU FP64 frames of the
    same rays, the probe with the camera turned."""
    from blackhole_b200 import abi

    moved = np.full(len(fp64), np.inf)
    sky = (fp64["what"] == abi.HIT_SKY) & (probe["what"] == abi.HIT_SKY)
    moved[sky] = _angle(probe["dir"][sky], fp64["dir"][sky])
    disc = (fp64["what"] == abi.HIT_DISC) & (probe["what"] == abi.HIT_DISC) & (fp64["g"] > 0)
    moved[disc] = np.abs(probe["g"][disc] - fp64["g"][disc]) / fp64["g"][disc]
    return moved


def compare_rays(a, b, probe=None, moved=None, against="the FP64 GPU frame (per ray)"):
    """Per-ray error of `b` against `a` (same rays, same order): class
    agreement, the relative error of g over disc rays of equal class and the
    sky-direction angle over sky rays of equal class, each with its tail
    beyond the target (1e-3, 1e-4 rad).  `moved` (from `conditioning`) or
    `probe` (a turned FP64 frame against `a`) marks the ill-conditioned rays,
    whose FP64 result moves by more than COND_LIMIT under the turn."""
    from blackhole_b200 import abi

    if moved is None and probe is not None:
        moved = conditioning(a, probe)
    same = a["what"] == b["what"]
    out = {"class_agree": float(same.mean()), "against": against, "rays": int(len(a)),
           "class_mismatch": int((~same).sum())}
    if (~same).any():
        pairs = {}
        for wa, wb in zip(a["what"][~same], b["what"][~same]):
            k = f"{abi.HIT_NAMES[wa]}->{abi.HIT_NAMES[wb]}"
            pairs[k] = pairs.get(k, 0) + 1
        out["class_mismatch_pairs"] = pairs
    disc = same & (a["what"] == abi.HIT_DISC) & (a["g"] > 0)
    if disc.any():
        e = np.abs(b["g"][disc] - a["g"][disc]) / a["g"][disc]
        out["g_rel"] = _dist(e, 1e-3)
        out["g_rel"]["frac_le_1e-3"] = float((e <= 1e-3).mean())
        if moved is not None:
            ill = moved[disc] > COND_LIMIT
            out["g_rel"]["ill_conditioned_rays"] = int(ill.sum())
            if (~ill).any():
                out["g_rel"]["max_well_conditioned"] = float(e[~ill].max())
                out["g_rel"]["n_above_target_well_conditioned"] = int((e[~ill] > 1e-3).sum())
    sky = same & (a["what"] == abi.HIT_SKY)
    if sky.any():
        d = _angle(b["dir"][sky], a["dir"][sky])
        out["dir_rad"] = _dist(d, 1e-4)
        out["dir_rad"]["frac_le_1e-4"] = float((d <= 1e-4).mean())
        if moved is not None:
            ill = moved[sky] > COND_LIMIT
            well = d[~ill]
            out["dir_rad"]["conditioning"] = {
                "probe": "FP64 GPU frame with the camera turned by %.1e rad" % COND_YAW,
                "ill_conditioned_rays": int(ill.sum()),
                "their_fp64_move_min": float(moved[sky][ill].min()) if ill.any() else None,
                "their_error_max": float(d[ill].max()) if ill.any() else None,
                "max_well_conditioned": float(well.max()) if well.size else None,
                "n_above_target_well_conditioned": int((well > 1e-4).sum()),
                "frac_le_1e-4_well_conditioned": float((well <= 1e-4).mean()) if well.size else None}
    return out


def rows_of(full, cfg, rows):
    """The per-sample results of whole rows of a row-major frame."""
    ss = max(1, cfg.sqrt_spp) ** 2
    return full.reshape(cfg.height, cfg.width * ss)[np.asarray(rows)].reshape(-1)


def checker_pin(r, size):
    """The GPU frames against the CPU checkers, per ray.  The checkers are
    test infrastructure used here only to check (nothing measured runs them):
      - oracle/bh_oracle.c, the FP64 restatement pinned bit for bit to the
        reference, on every 4th row of the frame under the workload's own
        settings (uniform sky, r_+(1+1e-6) stop), which the reference lacks;
      - the reference itself (oracle/_ref) on every 8th row under its own
        settings (galactic sky, its horizon stop), where it is built.
    Both precisions of the GPU path are compared; the conditioning probe
    (FP64 GPU frame, camera turned by COND_YAW) marks ill-conditioned rays."""
    import copy

    import oracle
    from blackhole_b200 import abi

    threads = os.cpu_count() or 1
    out = {}

    def leg(cd, cm, rows, port, checker, settings):
        t0 = time.perf_counter()
        chk, _ = port.trace_rows(cd, rows, threads)
        secs = time.perf_counter() - t0
        a = rows_of(r.trace_rays(cd), cd, rows)
        b = rows_of(r.trace_rays(cm), cm, rows)
        turned = copy.deepcopy(cd)
        turned.cam.yaw += COND_YAW
        moved = conditioning(a, rows_of(r.trace_rays(turned), cd, rows))
        return {"checker": checker, "settings": settings,
                "sample": f"{len(rows)} rows of the {size}x{size} frame (every {rows[1] - rows[0]}th), "
                          f"{len(chk)} rays, {threads} threads, {secs:.1f} s",
                "fp64": compare_rays(chk, a, moved=moved, against=checker),
                "mixed": compare_rays(chk, b, moved=moved, against=checker),
                "mixed_vs_fp64_gpu": compare_rays(a, b, moved=moved)}

    cd = frame_config(size, 0, 1, abi.PRECISION_FP64)
    cm = frame_config(size, 0, 1, abi.PRECISION_MIXED)
    out["oracle"] = leg(cd, cm, list(range(0, size, 4)), oracle.oracle(),
                        "the FP64 oracle (oracle/bh_oracle.c)",
                        "the workload's: uniform sky, horizon stop r_+(1+1e-6)")
    ref = oracle.reference()
    if ref is not None:
        for c in (cd, cm):
            c.sky_mode = abi.SKY_GALACTIC
            c.stop_mode = abi.STOP_REFERENCE
        out["reference"] = leg(cd, cm, list(range(0, size, 8)), ref,
                               "the reference's own trace()+shade() (oracle/_ref)",
                               "the reference's: galactic sky, horizon stop r_+ + 1e-4 + 1e-3 (r_+ - r_-)")
    return out


def photon_ring_leg(r, torch, flush, barrier, world, rank, check=True):
    """4096^2 frame of +-8 M centred on the prograde equatorial point of the
    critical curve (a = 0.998, 75 deg): mixed and FP64 device time, the
    per-ray step-count distribution and the mixed-vs-FP64 error."""
    from blackhole_b200 import abi, workloads

    cm = workloads.photon_ring_4096(abi.PRECISION_MIXED)
    cd = workloads.photon_ring_4096(abi.PRECISION_FP64)
    for c in (cm, cd):
        c.cam.phi = 2.0 * math.pi * rank / max(1, world)
    t_m, _, st_m, _ = time_device(r, cm, 2, 1, torch, flush, barrier)
    t_d, _, st_d, _ = time_device(r, cd, 2, 1, torch, flush, barrier)
    out = {"workload": "photon_ring_4096: a=0.998, inclination 75 deg, 4096x4096, +-8 M centred (yaw) on "
                       "alpha=-2.18 M, disc r_isco..100 M at 0.5 Eddington, M=6.5e9 M_sun",
           "rays": cm.n_rays,
           "mixed": {"value": round(cm.n_rays * 2 / (t_m * 1e-3), 1), "unit": "rays/s", "ms": round(t_m / 2, 3),
                     "steps_per_ray": round(st_m.steps / st_m.rays, 2)},
           "fp64": {"value": round(cd.n_rays * 2 / (t_d * 1e-3), 1), "unit": "rays/s", "ms": round(t_d / 2, 3),
                    "steps_per_ray": round(st_d.steps / st_d.rays, 2)}}
    out["mixed_over_fp64"] = round(out["mixed"]["value"] / out["fp64"]["value"], 3)
    a = r.trace_rays(cd)
    b = r.trace_rays(cm)
    steps = a["steps"].ravel()
    out["fp64_steps"] = {"mean": float(steps.mean()), "p50": float(np.quantile(steps, .5)),
                         "p99": float(np.quantile(steps, .99)), "max": int(steps.max()),
                         "frac_gt_2000": float((steps > 2000).mean())}
    out["classes"] = {abi.HIT_NAMES[k]: int(v) for k, v in enumerate(np.bincount(a["what"].ravel(), minlength=6))}
    out["accuracy"] = compare_rays(a, b)
    if rank == 0 and check:
        # A strip of 16 rows through the frame's centre, which the critical
        # curve crosses, against the FP64 oracle (the checker, timed apart).
        import oracle

        rows = list(range(cd.height // 2 - 8, cd.height // 2 + 8))
        t0 = time.perf_counter()
        chk, _ = oracle.oracle().trace_rows(cd, rows, os.cpu_count() or 1)
        secs = time.perf_counter() - t0
        sa, sb = rows_of(a, cd, rows), rows_of(b, cm, rows)
        checker = "the FP64 oracle (oracle/bh_oracle.c)"
        out["accuracy_vs_oracle"] = {
            "sample": f"rows {rows[0]}..{rows[-1]} ({len(chk)} rays) through the critical curve, {secs:.1f} s",
            "fp64": compare_rays(chk, sa, against=checker), "mixed": compare_rays(chk, sb, against=checker),
            "fp64_steps_in_strip": {"mean": float(sa["steps"].mean()), "max": int(sa["steps"].max())}}
    return out


def cpu_baseline(size: int, max_seconds: float = 20.0):
    """The reference CPU path on a bounded sample of the frame's rows."""
    import oracle
    from blackhole_b200 import abi

    cfg = frame_config(size, 0, 1, abi.PRECISION_FP64)
    ref = oracle.reference()
    threads = os.cpu_count() or 1
    if ref is not None:
        # The reference has one sky and one stop rule: run its own.
        cfg.sky_mode = abi.SKY_GALACTIC
        cfg.stop_mode = abi.STOP_REFERENCE
        rows = list(range(0, cfg.height, 2))
        t0 = time.perf_counter()
        _, st, setup = ref.render_rows(cfg, rows, threads)
        wall = time.perf_counter() - t0 - setup
        # the same path on one thread, over every 32nd row (a few seconds)
        rows1 = list(range(0, cfg.height, 32))
        _, st1, _ = ref.render_rows(cfg, rows1, 1)
        return {"value": st.rays / st.seconds, "unit": "rays/s", "cores": threads, "kind": "reference",
                "sample": f"{len(rows)} of {cfg.height} rows ({st.rays} rays) of the {size}x{size} frame, "
                          f"reference sky and horizon stop (its only ones), trace+shade on {threads} threads, "
                          f"{st.seconds:.2f} s excluding {setup:.2f} s scene set-up",
                "seconds": st.seconds,
                "one_thread": {"value": round(st1.rays / st1.seconds, 1), "unit": "rays/s",
                               "sample": f"{len(rows1)} rows ({st1.rays} rays), 1 thread, "
                                         f"{st1.seconds:.2f} s"}}
    port = oracle.oracle()
    w = 64
    t0 = time.perf_counter()
    _, st = port.trace_rays(cfg, (size - w) // 2, (size - w) // 2, w, 8)
    dt = time.perf_counter() - t0
    return {"value": st.rays / dt, "unit": "rays/s", "cores": 1, "kind": "port",
            "sample": f"{st.rays} rays of a {w}x8 window at the frame centre, oracle port, 1 thread",
            "seconds": dt}


def batch_leg(r, rank, world, barrier, max_over_ranks, steps=2, warmup=1):
    """The 64-frame batch (uneven sizes 256^2..2048^2, 89.1 M rays) through
    bh_gpu_render_batch: one persistent launch over all frames, captured as a
    CUDA graph on the first call and replayed.  Frames are split across ranks
    by ray count; the job's rate is all rays over the slowest rank."""
    from blackhole_b200 import shard, workloads

    frames = workloads.batch_64_frames()
    mine = [frames[i] for i in shard.frames_for_rank(frames, rank, world)]
    rays = sum(c.n_rays for c in frames)
    import torch

    # output buffers in pinned host memory, allocated once and reused (as a
    # film loop would), like the single-frame end-to-end leg's
    outs = [torch.empty((c.height, c.width, 3), dtype=torch.float64, pin_memory=True).numpy() for c in mine]
    for _ in range(warmup):
        r.render_batch(mine, outs=outs)
    barrier()
    dev_ms, wall = 0.0, 0.0
    st = []
    for _ in range(steps):
        t0 = time.perf_counter()
        r.render_batch(mine, st, outs=outs)
        wall += time.perf_counter() - t0
        dev_ms += st[0].kernel_ms if st else 0.0
    dev_ms = max_over_ranks(dev_ms)
    wall = max_over_ranks(wall)
    return {"workload": "batch_64_frames: spins {0,0.5,0.9,0.998} x inclinations {15,45,70,85} deg x "
                        "{256,512,1024,2048}^2, r_obs uniform 500..2000 M, mixed precision",
            "frames": len(frames), "rays_per_step": rays, "steps": steps, "warmup": warmup,
            "value": round(rays * steps / (dev_ms * 1e-3), 1) if dev_ms > 0 else None, "unit": "rays/s",
            "ms_per_step": round(dev_ms / steps, 3),
            "timing": "device time of the captured graph (staging copies, trace, shade, stats), max over ranks",
            "e2e": {"value": round(rays * steps / wall, 1), "unit": "rays/s",
                    "api": "bh_gpu_render_batch into pinned host arrays reused across calls, wall clock"},
            "steps_per_ray": round(sum(s.steps for s in st) / max(1, sum(s.rays for s in st)), 2)}


def jets_leg(r, torch, flush, barrier):
    """The reference's `quasar` preset with its Blandford-Znajek jets at
    1024x576: mixed and FP64 device time, rays with jet light, and the mixed
    path's error in the jet integral against FP64."""
    from blackhole_b200 import abi, workloads

    cm = workloads.quasar_jets(1024, 576, abi.PRECISION_MIXED)
    cd = workloads.quasar_jets(1024, 576, abi.PRECISION_FP64)
    t_m, _, st_m, _ = time_device(r, cm, 2, 1, torch, flush, barrier)
    t_d, _, st_d, _ = time_device(r, cd, 2, 1, torch, flush, barrier)
    a = r.trace_rays(cd)
    b = r.trace_rays(cm)
    same = (a["what"] == b["what"]) & (a["jet"] > 0)
    rel = np.abs(b["jet"][same] - a["jet"][same]) / a["jet"][same]
    return {"workload": "quasar_jets: reference `quasar` preset (a=0.998, 84 deg, r_cam 80 M, fov 0.90, "
                        "disc to 20 M at 0.5 Eddington, jets to z=130 M, Gamma_max 10), 1024x576, 1 spp",
            "rays": cm.n_rays,
            "mixed": {"value": round(cm.n_rays * 2 / (t_m * 1e-3), 1), "unit": "rays/s", "ms": round(t_m / 2, 3),
                      "jet_rays": st_m.jet_rays, "steps_per_ray": round(st_m.steps / st_m.rays, 2)},
            "fp64": {"value": round(cd.n_rays * 2 / (t_d * 1e-3), 1), "unit": "rays/s", "ms": round(t_d / 2, 3),
                     "jet_rays": st_d.jet_rays, "steps_per_ray": round(st_d.steps / st_d.rays, 2)},
            "mixed_jet_rel_err": {"p50": float(np.quantile(rel, .5)), "p99": float(np.quantile(rel, .99)),
                                  "max": float(rel.max()), "n": int(same.sum())} if same.any() else None}


def animation_leg(r, frames=48, width=512, height=288):
    """A hot-spot film made the CLI's way: exposure metered on a probe of the
    middle frame, then all frames traced in one launch and developed on the
    device (bh_gpu_render_batch_rgb); wall clock from the configs to the
    8-bit frames in host memory, after one warm-up pass of the same film."""
    from blackhole_b200 import workloads

    film = workloads.hotspot_orbit(frames=frames, width=width, height=height)
    # warm-up: the same film once (buffers sized, the batch graph captured)
    r.render_batch_rgb(film, exposure=1.0)
    t0 = time.perf_counter()
    _, e = r.render_rgb(workloads.exposure_probe(film[len(film) // 2]), meter_only=True)
    _, used = r.render_batch_rgb(film, exposure=e)
    wall = time.perf_counter() - t0
    rays = sum(c.n_rays for c in film)
    return {"workload": f"hotspot_orbit: {frames} frames {width}x{height}, a=0.9, 80 deg, r_cam 60 M, hot spot "
                        "at 8 M over one orbit, HDR curve, exposure locked from a probe",
            "value": round(frames / wall, 2), "unit": "frames/s", "rays_per_s": round(rays / wall, 1),
            "seconds": round(wall, 3), "exposure": e}


def adjoint_leg(r, steps=3, warmup=1):
    """Gradients per second of the discrete adjoint on the 512^2 gradient
    workload: one gradient = the binary64 render, the loss against the target
    frame and d(loss)/d(spin, inclination, Eddington ratio, r_out), the
    disc-edge term included."""
    from blackhole_b200 import workloads

    cfg = workloads.adjoint_512()
    target = r.render(workloads.adjoint_512(target=True))[..., 1].astype(np.float32)
    for _ in range(warmup):
        r.adjoint(cfg, target)
    dev_ms, gs = [], None
    t0 = time.perf_counter()
    for _ in range(steps):
        gs = r.adjoint(cfg, target)
        dev_ms.append(gs["kernel_ms"])
    wall = time.perf_counter() - t0
    ms = sum(dev_ms) / len(dev_ms)
    return {"workload": "adjoint_512: a=0.7, inclination 50 deg, 0.2 Eddington, r_out 25 M, 512x512, binary64; "
                        "target rendered at a=0.75, 53 deg, 0.22, 27 M; checkpoints every 16 accepted steps",
            "value": round(1e3 / ms, 2), "unit": "grads/s", "ms_per_grad": round(ms, 3),
            "timing": "device time of render + adjoint + reductions (CUDA events), mean of "
                      f"{steps} after {warmup} warm-up",
            "e2e": {"value": round(steps / wall, 2), "unit": "grads/s",
                    "api": "bh_gpu_adjoint from host target to host gradient, wall clock"},
            "loss": gs["loss"], "grad": [gs["d_spin"], gs["d_inclination"], gs["d_eddington"], gs["d_r_out"]],
            "steps_per_ray": round(gs["steps"] / gs["rays"], 2),
            "replay_over_forward": round(gs["replayed_steps"] / max(1, gs["steps"]), 3),
            "disc_rays": gs["disc_rays"], "sky_rays": gs["sky_rays"],
            "edge": {"candidates": gs["edge_candidates"], "cells": gs["edge_cells"],
                     "steps_over_forward": round(gs["edge_steps"] / max(1, gs["steps"]), 3),
                     "d_spin": gs["edge_spin"], "d_inclination": gs["edge_inclination"]},
            "held_out": {"rays": gs["high_order_rays"], "d_spin": gs["held_spin"],
                         "d_inclination": gs["held_inclination"]}}


def ring_adjoint_leg(r, steps=2):
    """Gradients per second with respect to (spin, inclination) on the
    1024^2 central crop of the photon-ring frame (binary64), against the
    crop rendered at a = 0.99, 76 deg."""
    from blackhole_b200 import workloads

    cfg = workloads.photon_ring_crop(1024)
    target = r.render(workloads.photon_ring_crop(1024, target=True))[..., 1].astype(np.float32)
    r.adjoint(cfg, target)
    ms, g = [], None
    for _ in range(steps):
        g = r.adjoint(cfg, target)
        ms.append(g["kernel_ms"])
    m = sum(ms) / len(ms)
    return {"workload": "photon_ring_crop: central 1024^2 of the photon-ring frame (a=0.998, 75 deg, "
                        "critical-curve centre), binary64; target at a=0.99, 76 deg",
            "value": round(1e3 / m, 2), "unit": "grads/s", "ms_per_grad": round(m, 3),
            "grad": [g["d_spin"], g["d_inclination"]], "loss": g["loss"],
            "steps_per_ray": round(g["steps"] / g["rays"], 2),
            "edge": {"candidates": g["edge_candidates"], "cells": g["edge_cells"]},
            "held_out": {"rays": g["high_order_rays"], "d_spin": g["held_spin"],
                         "d_inclination": g["held_inclination"]}}


def autotune_leg():
    """The launch-shape autotuner on the 64-frame batch: the search runs on
    every fourth frame of it (16 frames), then the whole batch is timed with
    the shape it keeps.  A fresh context, so no other leg sees the shape."""
    from blackhole_b200 import Renderer, workloads

    frames = workloads.batch_64_frames()
    with Renderer(0) as r:
        default = r.get_launch(frames[0].precision)
        r.render_batch(frames[::4])
        best, ms = r.autotune_batch(frames[::4])
        st = []
        r.render_batch(frames, st)
        r.render_batch(frames, st)
        rays = sum(c.n_rays for c in frames)
        return {"searched_on": "every 4th frame of batch_64_frames (16 frames)", "default": default,
                "best": best, "best_ms_on_subset": round(ms, 3),
                "batch_with_best": {"value": round(rays / (st[0].kernel_ms * 1e-3), 1), "unit": "rays/s",
                                    "ms": round(st[0].kernel_ms, 3)}}


def same_config_leg(r, size, rank, world, steps, warmup, torch, flush, barrier, max_over_ranks):
    """The same frame on the reference's own sky and horizon stop (the only
    ones it has; the reference arm times it on them), mixed and FP64: device
    time and end to end through bh_gpu_render into pinned host memory, so the
    speed-up over the reference arm can be read like for like."""
    from blackhole_b200 import abi

    res = {"settings": "galactic-band 250k-star sky (m <= 12) with the Milky Way background, horizon stop "
                       "r_+ + 1e-4 + 1e-3 (r_+ - r_-): the reference arm's settings"}
    for name, prec in (("mixed", abi.PRECISION_MIXED), ("fp64", abi.PRECISION_FP64)):
        cfg = frame_config(size, rank, world, prec)
        cfg.sky_mode = abi.SKY_GALACTIC
        cfg.stop_mode = abi.STOP_REFERENCE
        k = steps if prec == abi.PRECISION_MIXED else max(2, steps // 2)
        t, _, st, _ = time_device(r, cfg, k, max(1, warmup), torch, flush, barrier)
        t = max_over_ranks(t)
        entry = {"value": round(world * cfg.n_rays * k / (t * 1e-3), 1), "unit": "rays/s",
                 "ms_per_step": round(t / k, 4), "steps_per_ray": round(st.steps / max(1, st.rays), 2)}
        host = torch.empty((cfg.height, cfg.width, 3), dtype=torch.float64, pin_memory=True).numpy()
        for _ in range(max(1, warmup)):
            r.render_into(cfg, host)
        barrier()
        t0 = time.perf_counter()
        for _ in range(k):
            r.render_into(cfg, host)
        t_e = max_over_ranks(time.perf_counter() - t0)
        barrier()
        entry["e2e"] = {"value": round(world * cfg.n_rays * k / t_e, 1), "unit": "rays/s",
                        "api": "bh_gpu_render (C-ABI) into pinned host memory, wall clock"}
        res[name] = entry
    return res


def gpu_arm(args):
    import torch
    import torch.distributed as dist

    from blackhole_b200 import Renderer, abi, gpu

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    r = Renderer(local)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    size = args.size
    cfg_m = frame_config(size, rank, world, abi.PRECISION_MIXED)
    rays = cfg_m.n_rays

    with ClockSampler(local) as clk:
        t_mixed, times_m, st_m, _ = time_device(r, cfg_m, args.steps, args.warmup, torch, flush, barrier)
    t_mixed = max_over_ranks(t_mixed)
    value = world * rays * args.steps / (t_mixed * 1e-3)

    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "rays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_mixed / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 state/stages + f64 Delta/Sigma/error-norm/roots/diagnostics",
        "data": "synthetic (seeded camera rays and star catalogue)",
        "config": {"workload": WORKLOAD, "precision": "mixed", "rays_per_step": rays, "frame": f"{size}x{size}",
                   "partition": "one frame per GPU, camera azimuth 2 pi rank/N",
                   "l2": "256 MiB write between timed steps (L2 flushed)"},
    }

    # FP64 plain path, same frame.
    if not args.no_fp64:
        cfg_d = frame_config(size, rank, world, abi.PRECISION_FP64)
        t_fp64, _, st_d, _ = time_device(r, cfg_d, max(2, args.steps // 2), 1, torch, flush, barrier)
        t_fp64 = max_over_ranks(t_fp64)
        v64 = world * rays * max(2, args.steps // 2) / (t_fp64 * 1e-3)
        out["fp64"] = {"value": round(v64, 1), "unit": "rays/s",
                       "ms_per_step": round(t_fp64 / max(2, args.steps // 2), 4),
                       "steps_per_ray": round(st_d.steps / st_d.rays, 2),
                       "attempts_per_ray": round(st_d.attempts / st_d.rays, 2)}
        out["mixed_over_fp64"] = round(value / v64, 3)

        # The mixed path under the reference's step cap and with every
        # captured ray traced to the stop radius: the same step sequence
        # rule as the FP64 path, for comparison.
        cfg_c = frame_config(size, rank, world, abi.PRECISION_MIXED)
        cfg_c.mixed_step_limit = abi.STEP_LIMIT_REFERENCE
        cfg_c.mixed_capture = abi.CAPTURE_REFERENCE
        t_c, _, st_c, _ = time_device(r, cfg_c, max(2, args.steps // 2), 1, torch, flush, barrier)
        t_c = max_over_ranks(t_c)
        out["mixed_reference_cap"] = {
            "value": round(world * rays * max(2, args.steps // 2) / (t_c * 1e-3), 1), "unit": "rays/s",
            "ms_per_step": round(t_c / max(2, args.steps // 2), 4),
            "steps_per_ray": round(st_c.steps / st_c.rays, 2),
            "attempts_per_ray": round(st_c.attempts / st_c.rays, 2),
            "roofline_frac": roofline(st_c.kernel_ms, st_c.steps, st_c.attempts, "mixed",
                                      gpu.fma_peak_tflops(local, abi.PRECISION_MIXED), "")["frac"]}

        # The mixed path with every ray in binary32 (BH_NEAR_CRITICAL_BINARY32):
        # what tracing the near-critical rays in binary64 beside it costs, and
        # what it buys in direction error.
        cfg_b = frame_config(size, rank, world, abi.PRECISION_MIXED)
        cfg_b.mixed_near_critical = abi.NEAR_CRITICAL_BINARY32
        t_b, _, st_b, _ = time_device(r, cfg_b, max(2, args.steps // 2), 1, torch, flush, barrier)
        t_b = max_over_ranks(t_b)
        out["mixed_all_binary32"] = {
            "value": round(world * rays * max(2, args.steps // 2) / (t_b * 1e-3), 1), "unit": "rays/s",
            "ms_per_step": round(t_b / max(2, args.steps // 2), 4),
            "steps_per_ray": round(st_b.steps / st_b.rays, 2)}
        try:
            acc_b = accuracy(r, size, rank, world, cfgs=(cfg_d, cfg_b))
            out["mixed_all_binary32"]["dir_rad"] = acc_b.get("dir_rad")
            out["mixed_all_binary32"]["g_rel_max"] = acc_b.get("g_rel", {}).get("max")
        except Exception as e:  # noqa: BLE001 - a failed side measurement is reported, not fatal
            out["mixed_all_binary32"]["accuracy_error"] = repr(e)

    out["steps_per_ray"] = round(st_m.steps / st_m.rays, 2)
    out["attempts_per_ray"] = round(st_m.attempts / st_m.rays, 2)
    out["classes"] = {"captured": st_m.captured, "disc": st_m.disc_hits, "sky": st_m.escaped,
                      "exhausted": st_m.exhausted}
    out["diagnostics"] = {"max_norm_error": st_m.max_norm_error, "max_carter_drift": st_m.max_carter_drift}

    # Roofline of the dominant kernel (the trace kernel).
    peak32 = gpu.fma_peak_tflops(local, abi.PRECISION_MIXED)
    peak64 = gpu.fma_peak_tflops(local, abi.PRECISION_FP64)
    out["roofline"] = roofline(st_m.kernel_ms, st_m.steps, st_m.attempts, "mixed", peak32,
                               "FP32 FMA throughput measured in this run (bh_gpu_fma_peak)")
    if "fp64" in out:
        out["fp64"]["roofline"] = roofline(st_d.kernel_ms, st_d.steps, st_d.attempts, "fp64", peak64,
                                           "FP64 FMA throughput measured in this run (bh_gpu_fma_peak)")
    out["kernel_share"] = {"trace_ms": round(st_m.kernel_ms, 4), "shade_ms": round(st_m.shade_ms, 4)}

    if rank == 0:
        try:
            out["accuracy"] = accuracy(r, size, rank, world)
        except Exception as e:  # reported, not hidden
            out["accuracy"] = {"error": repr(e)}

    # End to end through the public API: host output buffer, synchronous call.
    from blackhole_b200 import RenderStats

    host = torch.empty((size, size, 3), dtype=torch.float64, pin_memory=True).numpy()
    st_e = RenderStats()
    for _ in range(max(1, args.warmup)):
        r.render_into(cfg_m, host)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s = abi.bh_render_stats()
        r.render_into(cfg_m, host, s)
        st_e.h2d_bytes, st_e.d2h_bytes = s.h2d_bytes, s.d2h_bytes
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    barrier()
    out["e2e"] = {"value": round(world * rays * args.steps / t_e2e, 1), "unit": "rays/s",
                  "h2d_bytes_per_step": int(st_e.h2d_bytes), "d2h_bytes_per_step": int(st_e.d2h_bytes),
                  "api": "bh_gpu_render (C-ABI) into pinned host memory, wall clock"}

    # Display leg: the same frame developed on the device (HDR curve, metered
    # exposure) so that only 8-bit sRGB crosses to the host.
    if not args.no_display:
        try:
            for _ in range(max(1, args.warmup)):
                r.render_rgb(cfg_m)
            barrier()
            t0 = time.perf_counter()
            st_d = RenderStats()
            for _ in range(args.steps):
                st_d = RenderStats()
                rgb, e = r.render_rgb(cfg_m, stats=st_d)
            t_rgb = max_over_ranks(time.perf_counter() - t0)
            barrier()
            out["display"] = {"value": round(world * rays * args.steps / t_rgb, 1), "unit": "rays/s",
                              "api": "bh_gpu_render_rgb (render + auto exposure + HDR tone curve + sRGB on "
                                     "the device), 8-bit image into host memory, wall clock",
                              "d2h_bytes_per_step": int(st_d.d2h_bytes), "exposure": e}
        except Exception as e:  # reported, not hidden
            out["display"] = {"error": repr(e)}

    if not args.no_fp64:
        try:
            out["same_config_as_reference"] = same_config_leg(r, size, rank, world, args.steps, args.warmup,
                                                              torch, flush, barrier, max_over_ranks)
        except Exception as e:  # reported, not hidden
            out["same_config_as_reference"] = {"error": repr(e)}

    # Kernels of ours launched in the timed region per mixed step: the
    # near-critical classification, the binary64 near-critical trace, two
    # binary32 traces (the main grid and the blocks started after the binary64
    # one), the binary64 resume trace, shade, 2 reduce.
    out["gpu_launches"] = 8 * args.steps
    out["clocks"] = clk.summary()

    if not args.no_jets:
        try:
            out["jets"] = jets_leg(r, torch, flush, barrier)
        except Exception as e:  # reported, not hidden
            out["jets"] = {"error": repr(e)}
        try:
            out["animation"] = animation_leg(r)
        except Exception as e:  # reported, not hidden
            out["animation"] = {"error": repr(e)}

    if not args.no_adjoint:
        try:
            out["adjoint"] = adjoint_leg(r)
        except Exception as e:  # reported, not hidden
            out["adjoint"] = {"error": repr(e)}
        try:
            out["photon_ring_adjoint"] = ring_adjoint_leg(r)
        except Exception as e:  # reported, not hidden
            out["photon_ring_adjoint"] = {"error": repr(e)}

    if not args.no_photon_ring:
        try:
            out["photon_ring"] = photon_ring_leg(r, torch, flush, barrier, world, rank,
                                                 check=world == 1 and not args.no_cpu_baseline)
        except Exception as e:  # reported, not hidden
            out["photon_ring"] = {"error": repr(e)}

    if not args.no_batch:
        try:
            out["batch"] = batch_leg(r, rank, world, barrier, max_over_ranks)
        except Exception as e:  # reported, not hidden
            out["batch"] = {"error": repr(e)}
        if world == 1:
            try:
                out["autotune"] = autotune_leg()
            except Exception as e:  # reported, not hidden
                out["autotune"] = {"error": repr(e)}

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline(size)
        except Exception as e:
            out["cpu_baseline"] = {"value": None, "error": repr(e)}
        try:
            out["accuracy_vs_checkers"] = checker_pin(r, size)
        except Exception as e:  # reported, not hidden
            out["accuracy_vs_checkers"] = {"error": repr(e)}

    if rank == 0:
        print(json.dumps(out), flush=True)
    r.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    from blackhole_b200 import abi

    cfg = frame_config(args.size, 0, 1, abi.PRECISION_FP64)
    ref = oracle.reference()
    threads = os.cpu_count() or 1
    kind = "reference"
    if ref is None:
        kind = "port"
        threads = 1
    else:
        cfg.sky_mode = abi.SKY_GALACTIC
        cfg.stop_mode = abi.STOP_REFERENCE
    # Each step: a bounded sample of rows (disjoint row sets cycle through the frame).
    rows_per_step = 64
    stride = max(1, cfg.height // rows_per_step)

    def step(i):
        rows = [(k * stride + i * 7) % cfg.height for k in range(rows_per_step)]
        if ref is not None:
            _, st, _ = ref.render_rows(cfg, rows, threads)
            return st.rays, st.seconds
        port = oracle.oracle()
        t0 = time.perf_counter()
        _, st = port.trace_rays(cfg, 0, rows[0], cfg.width, 1)
        return st.rays, time.perf_counter() - t0

    for i in range(args.warmup):
        step(i)
    n, secs = 0, 0.0
    for i in range(args.steps):
        a, b = step(args.warmup + i)
        n += a
        secs += b
    value = n / secs
    sample = (f"{rows_per_step} rows of the {args.size}x{args.size} frame per step "
              f"({rows_per_step * cfg.width} rays), reference sky and horizon stop (its only ones)"
              if ref is not None else f"one row of the frame per step, oracle port")
    out = {
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": "rays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * secs / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded camera rays and star catalogue)",
        "config": {"workload": WORKLOAD, "precision": "fp64 (the reference's only)", "frame": f"{args.size}x{args.size}"},
        "cpu_baseline": {"value": round(value, 1), "unit": "rays/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(value, 1), "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def once(args):
    """One render per precision: the launch list of a profiler capture is
    trace (mixed), trace (binary64 resume), shade, 2 x reduce, then trace
    (FP64), shade, 2 x reduce."""
    from blackhole_b200 import Renderer, RenderStats, abi

    with Renderer(0) as r:
        for prec in (abi.PRECISION_MIXED, abi.PRECISION_FP64):
            st = RenderStats()
            r.render(frame_config(args.size, 0, 1, prec), st)
            print(json.dumps({"precision": prec, "kernel_ms": st.kernel_ms, "steps": st.steps,
                              "attempts": st.attempts, "rays": st.rays}), flush=True)


def leg_once(args):
    """One invocation of one workload, for a profiler's launch list or a
    single-kernel capture: `adjoint` (bh_gpu_adjoint at --size^2 on the
    gradient workload), `display` (bh_gpu_develop of the --size^2 edge-on
    frame, HDR, metered), `jets` (the quasar preset at --size x 9/16 --size,
    mixed then FP64)."""
    from blackhole_b200 import Renderer, RenderStats, abi, workloads

    with Renderer(0) as r:
        if args.leg == "adjoint":
            cfg = workloads.adjoint_512()
            cfg.width = cfg.height = args.size
            t = workloads.adjoint_512(target=True)
            t.width = t.height = args.size
            target = r.render(t)[..., 1].astype(np.float32)
            g = r.adjoint(cfg, target)
            print(json.dumps({k: g[k] for k in ("loss", "d_spin", "kernel_ms", "steps", "replayed_steps")}))
        elif args.leg == "display":
            xyz = r.render(frame_config(args.size, 0, 1, abi.PRECISION_MIXED))
            rgb, e = r.develop(xyz, glare=0.3)
            print(json.dumps({"exposure": e, "mean": float(rgb.mean())}))
        elif args.leg == "jets":
            for prec in (abi.PRECISION_MIXED, abi.PRECISION_FP64):
                st = RenderStats()
                r.render(workloads.quasar_jets(args.size, args.size * 9 // 16, prec), st)
                print(json.dumps({"precision": prec, "kernel_ms": st.kernel_ms, "jet_rays": st.jet_rays}))
        else:
            raise SystemExit(f"unknown leg {args.leg!r}")


def main():
    args = parse()
    if args.leg:
        leg_once(args)
    elif args.once:
        once(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
