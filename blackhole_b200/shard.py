"""Frame sharding across ranks (one process per GPU).

Rays never interact, so a multi-GPU render needs no data-path collective: each
rank renders whole frames.  ``frames_for_rank`` partitions a list of frames
into contiguous blocks of nearly equal ray count (the work unit), and
``reduce_stats`` combines the per-rank ``RenderStats`` the way the reference
combines its per-thread stats (render.cpp:481-494): counters summed, drift
maxima maximised, ``seconds`` the maximum over ranks.  ``reduce_grads`` sums
the adjoint's loss and four gradients over ranks that each differentiated
their own frames (the loss of a set of frames is the sum of theirs).  All run
over any torch.distributed process group (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

from .config import RenderStats

SUM_FIELDS = ("rays", "steps", "captured", "disc_hits", "sun_hits", "star_hits", "jet_rays",
              "escaped", "exhausted", "total_flux", "attempts", "h2d_bytes", "d2h_bytes")
MAX_FIELDS = ("max_norm_error", "max_carter_drift", "seconds", "kernel_ms", "shade_ms")


def frames_for_rank(cfgs: list, rank: int, world: int) -> list:
    """Indices of the frames rank `rank` of `world` renders: contiguous blocks
    split at the ray-count quantiles (every frame on exactly one rank)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    weights = [c.n_rays for c in cfgs]
    total = sum(weights)
    out, acc = [], 0
    for i, w in enumerate(weights):
        # the frame goes to the rank owning the midpoint of its ray range
        mid = acc + 0.5 * w
        owner = min(world - 1, int(world * mid / total)) if total > 0 else i % world
        if owner == rank:
            out.append(i)
        acc += w
    return out


def reduce_stats(stats: RenderStats, group=None, device=None) -> RenderStats:
    """All-reduce one rank's stats into the job's (sum / max), on every rank."""
    import torch
    import torch.distributed as dist

    s = torch.tensor([float(getattr(stats, f)) for f in SUM_FIELDS], dtype=torch.float64, device=device)
    m = torch.tensor([float(getattr(stats, f)) for f in MAX_FIELDS], dtype=torch.float64, device=device)
    dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
    out = RenderStats()
    for f, v in zip(SUM_FIELDS, s.tolist()):
        setattr(out, f, v if f == "total_flux" else int(round(v)))
    for f, v in zip(MAX_FIELDS, m.tolist()):
        setattr(out, f, v)
    return out


GRAD_FIELDS = ("loss", "d_spin", "d_inclination", "d_eddington", "d_r_out",
               "edge_spin", "edge_inclination", "held_spin", "held_inclination")
GRAD_COUNTS = ("rays", "steps", "replayed_steps", "disc_rays", "sky_rays", "edge_candidates", "edge_cells",
               "edge_steps", "high_order_rays")


def reduce_grads(grad: dict, group=None, device=None) -> dict:
    """Sum-all-reduce of one rank's adjoint result (loss, the four
    gradients and their edge and held-out parts; counters summed too), on
    every rank.  Fields absent from `grad` count as 0."""
    import torch
    import torch.distributed as dist

    keys = GRAD_FIELDS + GRAD_COUNTS
    t = torch.tensor([float(grad.get(k, 0.0)) for k in keys], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    out = dict(grad)
    for k, v in zip(keys, t.tolist()):
        out[k] = v if k in GRAD_FIELDS else int(round(v))
    return out
