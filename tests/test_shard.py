"""Multi-rank frame sharding and stats reduction, on CPU with gloo.

The render path shards by frame with no data-path collective; the cross-rank
steps are the stats reduction (sums and maxima), the timing max and the final
gather of every rank's frames to one rank.  Two gloo ranks on 127.0.0.1 run
the same code bench.py runs over NCCL.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

import numpy as np

from blackhole_b200 import shard, workloads
from blackhole_b200.config import RenderConfig, RenderStats


def test_partition_covers_every_frame_once_and_balances_rays():
    frames = workloads.batch_64_frames()
    for world in (1, 2, 3, 4, 8):
        parts = [shard.frames_for_rank(frames, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(frames)))
        rays = [sum(frames[i].n_rays for i in p) for p in parts]
        biggest = max(f.n_rays for f in frames)
        assert max(rays) - min(rays) <= 2 * biggest + 1


def test_partition_rejects_bad_ranks():
    with pytest.raises(ValueError):
        shard.frames_for_rank(workloads.batch_64_frames(), 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    st = RenderStats(rays=100 + rank, steps=1000 * (rank + 1), captured=rank, disc_hits=10, escaped=5,
                     max_norm_error=1e-9 * (rank + 1), max_carter_drift=[3e-6, 1e-6][rank],
                     seconds=0.5 + rank, total_flux=1.5 * (rank + 1), attempts=1001 * (rank + 1))
    tot = shard.reduce_stats(st)
    frames = workloads.batch_64_frames()
    mine = shard.frames_for_rank(frames, rank, world)
    g = shard.reduce_grads({"loss": 1.0 + rank, "d_spin": [0.5, -2.0][rank], "d_inclination": 3.0,
                            "d_eddington": 1e20 * (rank + 1), "d_r_out": -2.0 * (rank + 1), "rays": 10, "steps": 7,
                            "edge_spin": 0.25, "edge_cells": 3 + rank})
    q.put((rank, tot.as_tuple() if hasattr(tot, "as_tuple") else vars(tot), mine, g))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_stats_and_split_frames():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda t: t[0])
    for _, tot, _, g in res:
        assert g["loss"] == 3.0 and g["d_spin"] == -1.5 and g["d_inclination"] == 6.0
        assert g["d_eddington"] == pytest.approx(3e20) and g["rays"] == 20 and g["steps"] == 14
        assert g["d_r_out"] == -6.0 and g["edge_spin"] == 0.5 and g["edge_cells"] == 7
        assert g["held_spin"] == 0.0 and g["edge_steps"] == 0
        assert tot["rays"] == 201 and tot["steps"] == 3000 and tot["captured"] == 1
        assert tot["disc_hits"] == 20 and tot["escaped"] == 10 and tot["attempts"] == 3003
        assert tot["max_norm_error"] == pytest.approx(2e-9)
        assert tot["max_carter_drift"] == pytest.approx(3e-6)
        assert tot["seconds"] == pytest.approx(1.5) and tot["total_flux"] == pytest.approx(4.5)
    a, b = res[0][2], res[1][2]
    assert sorted(a + b) == list(range(64)) and not set(a) & set(b)


def _small_batch():
    """Seven frames of uneven size (the batch's shape, CPU-sized)."""
    dims = [(24, 16), (8, 8), (40, 30), (16, 9), (32, 32), (12, 20), (48, 27)]
    return [RenderConfig(width=w, height=h) for w, h in dims]


def _fake_frame(cfg, i, kind):
    """A frame's pixels as a deterministic function of frame and pixel: the
    stand-in for a render, so the test checks the gather's bookkeeping."""
    n = cfg.height * cfg.width * 3
    v = (np.arange(n, dtype=np.float64) * 1.25 + 1000.0 * i).reshape(cfg.height, cfg.width, 3)
    return v if kind == "xyz" else (v.astype(np.int64) % 251).astype(np.uint8)


def _gather_worker(rank, world, port, q, kind):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    cfgs = _small_batch()
    mine = [_fake_frame(cfgs[i], i, kind) for i in shard.frames_for_rank(cfgs, rank, world)]
    got = shard.gather_frames(cfgs, mine, rank, world)
    q.put((rank, got))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["xyz", "srgb8"])
def test_two_gloo_ranks_gather_frames_equal_one_rank_batch(kind):
    cfgs = _small_batch()
    single = shard.gather_frames(cfgs, [_fake_frame(c, i, kind) for i, c in enumerate(cfgs)], 0, 1)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, q, kind)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[1] is None
    assert len(res[0]) == len(cfgs)
    for a, b, c in zip(res[0], single, cfgs):
        assert a.shape == (c.height, c.width, 3) and a.dtype == b.dtype
        assert np.array_equal(a, b)


def test_gather_rejects_a_wrong_frame_count():
    cfgs = _small_batch()
    with pytest.raises(ValueError):
        shard.gather_frames(cfgs, [], 0, 2)
