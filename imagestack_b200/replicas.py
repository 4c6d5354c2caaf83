"""Host-side logic of running the lattice on several GPUs of one node.

A single image does not shard (its splat needs one key -> vertex map and its blur's
neighbours span the whole lattice), while independent images shard trivially, so several
GPUs run replicas: one process per GPU, each filtering its own images, with no collective
on the data path.  The only exchange is the timing: a job is as slow as its slowest rank.
"""
from __future__ import annotations


def rank_env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment; (1, 0, 0) alone."""
    import os
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def frame_seeds(rank: int, count: int, base_seed: int, stride: int = 17) -> list[int]:
    """Seeds of the `count` synthetic frames rank `rank` filters per step: distinct across
    ranks (rank r uses base + stride*r + k), so replicas never filter the same frame."""
    if count > stride:
        raise ValueError("more frames per rank than the seed stride separates")
    return [base_seed + stride * rank + k for k in range(count)]


def shard(n: int, rank: int, world: int) -> list[int]:
    """Indices of the independent images rank `rank` of `world` takes from a list of n:
    round robin, so sizes that vary along the list spread evenly."""
    if not (0 <= rank < world):
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    return list(range(rank, n, world))


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks of the default process group (the job's time is
    its slowest rank's); `value` itself when no group is initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
