"""Replica runs across GPUs.

Rollouts never exchange data, so N GPUs run N independent replicas (one process per GPU,
each stepping its own rollouts) with no collective on the data path.  The only
cross-rank steps are host-side bookkeeping: the job's time is the maximum over ranks
(every rank must finish) and its work the sum over ranks.  Both are one all-reduce each
on the process group (NCCL on GPUs, gloo on CPU in the tests), taken by every rank in
the same order.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def job_totals(local_ms: float, local_units: float, device=None) -> tuple[float, float]:
    """(max over ranks of local_ms, sum over ranks of local_units); the local values when
    no process group is initialised."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(local_ms), float(local_units)
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    u = torch.tensor([float(local_units)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


def replica_seed(base: int, rank: int) -> int:
    """Seed of a rank's synthetic workload: distinct replicas, reproducible per rank."""
    return int(base) * 1000 + int(rank)
