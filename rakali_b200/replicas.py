"""Replicas: one independent simulation per rank (one process per GPU).

The structured step has no exchange between independent simulations, so a
multi-GPU run is N replicas of the single-GPU workload (weak scaling): no
collective on the data path.  The ranks meet only around the timed region: a
barrier before it, and the maximum of the per-rank device times after it (the
job is as slow as its slowest rank).  These helpers hold that logic so that it
can be exercised with the gloo backend on CPU.
"""
from __future__ import annotations

import os


def visible_gpu_index(local_rank: int, env=None) -> int:
    """Physical index of the GPU a local rank drives (CUDA_VISIBLE_DEVICES aware),
    for nvidia-smi queries; the CUDA device ordinal itself is `local_rank`."""
    vis = (os.environ if env is None else env).get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def max_over_ranks(x: float, dist, device: str = "cuda") -> float:
    """The maximum of a per-rank value over all ranks (identity without dist)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_value(world: int, units_per_rank: float, steps: int, ms: float) -> float:
    """Whole-job throughput: units all ranks processed per second of the slowest rank."""
    return world * units_per_rank * steps / (ms * 1e-3)


def replica_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s synthetic workload (independent replicas)."""
    return base + rank


__all__ = ["visible_gpu_index", "barrier", "max_over_ranks", "weak_value", "replica_seed"]
