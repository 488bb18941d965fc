"""Multi-GPU plumbing: one process per GPU, no data-path collective.

The path shards into independent units -- whole scenes of a batched build
(the BLAS set of bajo/bvh/gpu/triangle_bvh.mojo:469) and whole-pixel chunks
of a render (the chunk loop of bajo/rt/gpu/resources.mojo:217) -- so every
rank works alone and ranks only meet for a barrier and the max-over-ranks
timing.  The plain single-scene workload runs as replicas.

Process groups use NCCL over NVLink on GPUs and gloo on CPU (tests); ranks
read RANK / WORLD_SIZE / LOCAL_RANK / MASTER_* from the environment as
torchrun sets them.
"""
from __future__ import annotations

import os
from datetime import timedelta

import numpy as np


def world_from_env():
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str | None = None, timeout_s: float = 120.0):
    """Join the process group when WORLD_SIZE > 1 (NCCL with a GPU, gloo
    without); set this process's GPU.  Returns (world, rank, local)."""
    import torch
    world, rank, local = world_from_env()
    if world > 1:
        import torch.distributed as td
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        td.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def _device():
    import torch
    import torch.distributed as td
    return torch.device("cuda", torch.cuda.current_device()) if td.get_backend() == "nccl" else torch.device("cpu")


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as td
        td.barrier()


def max_over_ranks(world: int, x: float) -> float:
    """The largest value any rank reports (timings: the slowest rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as td
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(world: int, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as td
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    td.all_reduce(t, op=td.ReduceOp.SUM)
    return float(t.item())


def finish(world: int) -> None:
    if world > 1:
        import torch.distributed as td
        td.destroy_process_group()


# ---- sharding ---------------------------------------------------------------
def shard_scenes(counts, world: int, rank: int) -> np.ndarray:
    """Indices of the scenes this rank builds and traces.

    Greedy longest-processing-time assignment by predicted cost (triangle
    count), ties to the lower rank: every rank computes the same assignment
    from the same counts, so no exchange is needed.  Returned in ascending
    scene order."""
    counts = np.asarray(counts, dtype=np.int64)
    order = np.argsort(-counts, kind="stable")
    load = np.zeros(world, np.int64)
    owner = np.empty(counts.size, np.int64)
    for s in order:
        r = int(np.argmin(load))
        owner[s] = r
        load[r] += counts[s]
    return np.nonzero(owner == rank)[0]


def shard_pixels(n_pixels: int, world: int, rank: int) -> tuple[int, int]:
    """[begin, end) of this rank's contiguous pixel range (whole pixels, so
    every pixel's samples stay on one rank)."""
    per = n_pixels // world
    extra = n_pixels % world
    begin = rank * per + min(rank, extra)
    return begin, begin + per + (1 if rank < extra else 0)


def subset_offsets(seg_offsets, scenes) -> tuple[np.ndarray, np.ndarray]:
    """(item indices, new segment offsets) of the chosen scenes of a
    segmented vertex buffer, in the given scene order."""
    so = np.asarray(seg_offsets, dtype=np.int64)
    items, new = [], [0]
    for s in scenes:
        items.append(np.arange(so[s], so[s + 1]))
        new.append(new[-1] + int(so[s + 1] - so[s]))
    idx = np.concatenate(items) if items else np.zeros(0, np.int64)
    return idx, np.asarray(new, np.int64)
