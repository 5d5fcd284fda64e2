"""Several GPUs: independent replicas, one process per GPU.

Every workload here shards without a data-path collective: a world's step
does not span GPUs (each fits one), the scenes of the batched form and the
requests of the serving form are independent.  Each rank therefore runs its
own replica on its own seed or its own share of the requests, and the only
communication is timing: a barrier around the timed region and the maximum
of the ranks' device times, from which the whole-job throughput follows.
"""
from __future__ import annotations

from typing import List, Sequence, TypeVar

T = TypeVar("T")


def replica_seed(base: int, rank: int) -> int:
    """Seed of rank r's replica of a workload whose single-GPU seed is base."""
    return base + rank


def shard(items: Sequence[T], rank: int, world_size: int) -> List[T]:
    """Rank r's share of independent work items (scenes, requests): every
    world_size-th item starting at r, so shares differ by at most one item and
    keep the items' order."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("bad rank / world size")
    return list(items[rank::world_size])


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest of the ranks' values (all ranks call it; a no-op without
    an initialised process group)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    """The sum of the ranks' values (all ranks call it)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_throughput(units_per_rank: float, world_size: int, ms_max: float) -> float:
    """Whole-job units per second: every rank processed units_per_rank, the
    slowest took ms_max."""
    return units_per_rank * world_size / (ms_max / 1000.0)
