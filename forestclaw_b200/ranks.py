"""Rank plumbing of multi-GPU runs.

One process per GPU (torch.distributed; NCCL on GPUs, gloo on the CPU).  The
path shards without a data-path exchange: every rank advances its own forests
-- a replica of a single-forest workload, or its own slice of independent batch
instances -- so the only collectives are two scalars per measurement: the
maximum of the ranks' device times and the sum of their cell updates.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def rank_world() -> tuple[int, int]:
    """(rank, world size); (0, 1) without an initialised process group."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def instance_seed_base(rank: int, per_rank: int) -> int:
    """First instance seed of a rank that runs per_rank batch instances: ranks draw
    disjoint, consecutive seed ranges, so N ranks run N * per_rank distinct instances."""
    return rank * per_rank


def max_over_ranks(value: float, device: str | torch.device = "cpu") -> float:
    rank, world = rank_world()
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device: str | torch.device = "cpu") -> float:
    rank, world = rank_world()
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def aggregate(total_ms: float, cells: float, device: str | torch.device = "cpu") -> tuple[float, float, float]:
    """Whole-job throughput of a timed region: (max device ms over ranks, cell updates
    of all ranks, cell updates per second).  Every rank calls it in the same order."""
    ms = max_over_ranks(total_ms, device)
    c = sum_over_ranks(cells, device)
    return ms, c, c / (ms * 1e-3) if ms > 0 else 0.0
