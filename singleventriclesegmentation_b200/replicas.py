"""Host-side plumbing for running the solver on several GPUs as independent replicas.

Frame pairs and sequences are independent solves, so the path shards by units with no data
exchange (the reference runs one process per GPU over patient index ranges,
scripts/parallel_flow.sh:15-45). One process per GPU; torch.distributed is used only to agree on
the work split and to take the slowest rank's time.
"""
from __future__ import annotations

import os
from typing import List, Sequence, TypeVar

import torch
import torch.distributed as dist

T = TypeVar("T")


def env_rank():
    """(rank, local_rank, world_size) from the launcher's environment (torchrun)."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def shard(units: Sequence[T], rank: int, world: int) -> List[T]:
    """Contiguous block of `units` for `rank` (block sizes differ by at most one), the analogue of
    parallel_flow.sh's index ranges."""
    n = len(units)
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return list(units[start:stop])


def max_over_ranks(value: float, device=None) -> float:
    """The slowest rank's value (a no-op without an initialised process group)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
