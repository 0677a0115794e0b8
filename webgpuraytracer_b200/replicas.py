"""Replicated rendering across ranks (one process per GPU).

Progressive path tracing shards by samples: every rank renders the same view with its own seed
(an independent sample stream of the same estimator), so the data path needs no collective.
This module holds the plumbing around it: process-group set-up from the torchrun environment,
the max-over-ranks device time, and the one optional exchange -- merging the ranks' running
means into the image of all their samples (a sample-count-weighted all-reduce, done outside
any timed region).
"""
from __future__ import annotations

import os
from datetime import timedelta

import numpy as np


def env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment (1 process when unset)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def setup(backend: str = "nccl", timeout_s: float = 120.0) -> tuple[int, int, int]:
    """Joins the process group when WORLD_SIZE > 1 (NCCL binds this rank's GPU first)."""
    rank, world, local = env()
    if world > 1:
        import torch
        import torch.distributed as dist
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
    return rank, world, local


def _device():
    import torch
    import torch.distributed as dist
    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x: float, world: int) -> float:
    """The largest of every rank's x (the job's time is its slowest rank's)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def rank_seed(base: int, rank: int) -> int:
    """Per-rank value of SceneParams.seed: distinct sample streams on every rank."""
    return int(base) + int(rank)


def merge_accumulations(acc: np.ndarray, samples: int, world: int) -> tuple[np.ndarray, int]:
    """All ranks' running means (H, W, 4) of `samples` samples each merged into the mean of all
    their samples: sum(acc_r * n_r) / sum(n_r), in float64 on the host side of the exchange."""
    if world == 1:
        return acc, samples
    import torch
    import torch.distributed as dist
    dev = _device()
    t = torch.from_numpy(np.ascontiguousarray(acc, np.float64) * float(samples)).to(dev)
    n = torch.tensor([float(samples)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    total = int(round(float(n.item())))
    return (t / n).cpu().numpy(), total


def teardown(world: int):
    if world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()


def assign_lpt(work: list[float], world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of independent jobs (e.g. camera views weighted
    by width x height x spp) to `world` ranks: jobs in descending order of work, each to the rank
    with the least work so far (ties to the lower rank).  Returns the job indices per rank."""
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += work[i]
    return out


def gather_lists(values: list[float], world: int) -> list[float]:
    """Every rank's list of values, concatenated in rank order (on every rank)."""
    if world == 1:
        return list(values)
    import torch.distributed as dist
    parts: list = [None] * world
    dist.all_gather_object(parts, list(values))
    return [x for part in parts for x in part]
