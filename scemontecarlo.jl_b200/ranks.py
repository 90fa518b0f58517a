"""Replica-parallel runs over several GPUs (one process per GPU, torch.distributed).

The sweep does not shard a chain: every rank advances its own batch of replicas
(weak scaling), so the data path has no collective. Ranks meet only to time the
job: a barrier before and after the timed region, the slowest rank's device time
(MAX) and the attempts of all ranks (SUM)."""
from __future__ import annotations

import numpy as np


def rank_keys(base_seed: int, rank: int, count: int) -> list:
    """`count` 64-bit device keys for the replicas of `rank`, distinct across ranks
    (a numpy SeedSequence spawned per rank from the job's seed)."""
    ss = np.random.SeedSequence(int(base_seed)).spawn(rank + 1)[rank]
    return [int(x) for x in np.random.default_rng(ss).integers(0, 2 ** 63, size=count)]


def aggregate(local_ms: float, local_attempts: float, dist=None, device=None):
    """(job device time in ms = max over ranks, attempts summed over ranks)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(local_ms), float(local_attempts)
    import torch
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    a = torch.tensor([float(local_attempts)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(a, op=dist.ReduceOp.SUM)
    return float(t.item()), float(a.item())
