"""Replica plumbing of the multi-GPU runs: one independent periodic box (or
batch) per rank and no data-path collective.  Ranks meet only for barriers
and for the max over ranks of a device-timed region, so a whole-job rate is
(units on all ranks) / (slowest rank's time).

The reference decomposes one box over MPI ranks; this path shards by box, the
way the batched and served forms shard (independent boxes to independent
GPUs).  Everything here is host logic and runs on any torch.distributed
backend (NCCL on the GPUs, gloo in the CPU tests).
"""

from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class RankInfo:
    rank: int
    world: int
    local_rank: int

    @property
    def is_root(self) -> bool:
        return self.rank == 0


def rank_info(default_world: int = 1, env=None) -> RankInfo:
    """RANK / WORLD_SIZE / LOCAL_RANK as torchrun sets them (defaults: a
    single process)."""
    env = os.environ if env is None else env

    def get(name, default):
        try:
            return int(env.get(name, default))
        except ValueError:
            return default

    return RankInfo(get("RANK", 0), get("WORLD_SIZE", default_world), get("LOCAL_RANK", 0))


class Replicas:
    """Process group of the replicas (None when world == 1).

    backend "nccl" on GPUs, "gloo" on CPU; a short timeout so that ranks which
    wait on a missing peer end with an error instead of hanging."""

    def __init__(self, info: RankInfo, backend: str = "nccl", timeout_s: float = 120.0,
                 device=None):
        self.info = info
        self.device = device
        self.dist = None
        if info.world > 1:
            import torch.distributed as dist
            if not dist.is_initialized():
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self, sync=None):
        """Barrier over ranks, then `sync()` (e.g. a device synchronise)."""
        if self.dist is not None:
            self.dist.barrier()
        if sync is not None:
            sync()

    def max(self, x: float) -> float:
        """Max of x over ranks (the slowest rank's time)."""
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None and self.dist.is_initialized():
            self.dist.destroy_process_group()
        self.dist = None


def whole_job_rate(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Units processed by all ranks per second of the slowest rank."""
    return world * units_per_rank / seconds_max
