"""Independent walker replicas, one per GPU (the multi-GPU mode of this path).

Walkers are independent within a sweep (the reference's docs/architecture.md
:182-191), and one B200 holds the whole population of the benchmarked runs,
so N GPUs run N independent DMC/VMC replicas — own seeds, own branch streams,
no exchange on the data path.  What crosses ranks is bookkeeping only: a
barrier around the timed region, the slowest rank's device time (max) and the
ranks' work (sum).  This module holds that logic so that it runs unchanged on
NCCL (one process per GPU) and on gloo (CPU tests, world size 2).
"""
from __future__ import annotations

from typing import Optional


def replica_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s replica: distinct streams for every rank
    (stream_seed mixes the seed through splitmix64, so neighbouring seeds
    give unrelated xoshiro256++ states)."""
    return int(base) + 7919 * int(rank)


class Replicas:
    """Rank bookkeeping over an initialised torch.distributed group (or none:
    one replica).  `device` is where reduction tensors live (a CUDA device for
    NCCL, the CPU for gloo)."""

    def __init__(self, dist=None, device=None):
        self.dist = dist if dist is not None and dist.is_available() and dist.is_initialized() else None
        self.device = device
        self.world = self.dist.get_world_size() if self.dist else 1
        self.rank = self.dist.get_rank() if self.dist else 0

    def barrier(self) -> None:
        if self.dist:
            self.dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if not self.dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        """The slowest rank's value (device times: the job ends with it)."""
        return self._reduce(x, self.dist.ReduceOp.MAX if self.dist else None)

    def sum(self, x: float) -> float:
        """The whole job's total (moves, evaluations, launches)."""
        return self._reduce(x, self.dist.ReduceOp.SUM if self.dist else None)

    def throughput(self, work: float, ms: float) -> Optional[float]:
        """Whole-job rate: every rank's work over the slowest rank's time."""
        total, slowest = self.sum(work), self.max(ms)
        return total / (slowest * 1e-3) if slowest > 0.0 else None
