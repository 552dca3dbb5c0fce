"""Multi-GPU host logic: replicas only.

The reference's path has no exchange step (one process, one GPU), so N GPUs
run N independent replicas, one process per GPU: each rank builds its own
cloud from its own seed (or takes its own share of the right-hand sides of a
batch) and no collective touches the data path.  The only collectives are
the timing ones: a barrier on each side of the timed region and the maximum
of the per-rank device times.  They work with the "nccl" backend on GPUs and
with "gloo" on CPU (tests).
"""
from __future__ import annotations

import os


def env_rank():
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base: int, rank: int) -> int:
    """Seed of rank's cloud: distinct per rank, rank 0 keeps the base seed."""
    return base + 1000 * rank


def shard(count: int, world: int, rank: int):
    """[start, stop) of rank's share of `count` independent items (right-hand
    sides): contiguous, sizes differ by at most one, the shares cover
    0..count-1 exactly once."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


class Timing:
    """Barrier and max-over-ranks for an initialised process group (or none)."""

    def __init__(self, dist=None, device=None):
        self.dist = dist
        self.device = device

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device or "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())
