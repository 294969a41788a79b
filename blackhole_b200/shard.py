"""Frame sharding across ranks (one process per GPU).

Rays never interact, so a multi-GPU render needs no data-path collective: each
rank renders whole frames.  ``frames_for_rank`` partitions a list of frames
into contiguous blocks of nearly equal ray count (the work unit), and
``reduce_stats`` combines the per-rank ``RenderStats`` the way the reference
combines its per-thread stats (render.cpp:481-494): counters summed, drift
maxima maximised, ``seconds`` the maximum over ranks.  ``reduce_grads`` sums
the adjoint's loss and four gradients over ranks that each differentiated
their own frames (the loss of a set of frames is the sum of theirs).
``gather_frames`` brings every rank's frames to one rank, in batch order, as
the reference's pool joins its rows into one image (render.cpp:474-494).  All
run over any torch.distributed process group (NCCL on GPUs, gloo on CPU).
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


def gather_frames(cfgs: list, mine: list, rank: int, world: int, dst: int = 0, group=None, device=None):
    """Gather the pixels of a batch sharded by ``frames_for_rank``.

    ``mine`` holds this rank's frames in the order ``frames_for_rank(cfgs,
    rank, world)`` lists them, each an array of height x width x 3 values
    (float64 XYZ, or the 8-bit sRGB of a developed frame).  Every rank but
    ``dst`` sends its frames to ``dst`` as one contiguous buffer (point to
    point: the frames' sizes differ, and every rank knows them from
    ``cfgs``).  Returns, on ``dst``, the list of all frames in batch order;
    None on the other ranks.  ``device``: where the buffers go through the
    process group (the rank's GPU under NCCL, None for gloo).
    """
    import numpy as np
    import torch
    import torch.distributed as dist

    if world == 1:
        return list(mine)
    parts = [frames_for_rank(cfgs, r, world) for r in range(world)]
    if len(mine) != len(parts[rank]):
        raise ValueError(f"rank {rank} holds {len(mine)} frames, frames_for_rank gives it {len(parts[rank])}")
    dtype = np.asarray(mine[0]).dtype if mine else np.dtype(np.float64)
    if dtype not in (np.float64, np.uint8):
        raise ValueError("frames are float64 XYZ or uint8 sRGB")
    tdt = torch.float64 if dtype == np.float64 else torch.uint8
    sizes = [cfgs[i].height * cfgs[i].width * 3 for i in range(len(cfgs))]
    if rank != dst:
        flat = np.concatenate([np.ascontiguousarray(f, dtype=dtype).reshape(-1) for f in mine]) if mine \
            else np.zeros(0, dtype=dtype)
        if flat.size:
            dist.send(torch.from_numpy(flat).to(device), dst=dst, group=group)
        return None
    out = [None] * len(cfgs)
    for k, i in enumerate(parts[dst]):
        out[i] = np.ascontiguousarray(mine[k], dtype=dtype).reshape(cfgs[i].height, cfgs[i].width, 3)
    for r in range(world):
        if r == dst or not parts[r]:
            continue
        n = sum(sizes[i] for i in parts[r])
        buf = torch.empty(n, dtype=tdt, device=device)
        dist.recv(buf, src=r, group=group)
        flat = buf.cpu().numpy()
        off = 0
        for i in parts[r]:
            out[i] = flat[off:off + sizes[i]].reshape(cfgs[i].height, cfgs[i].width, 3)
            off += sizes[i]
    return out
