"""Replica bookkeeping of the multi-GPU benchmark.

The benchmark workloads fit one GPU, so `bench.py --gpus N` runs N independent replicas:
each rank mines its own copy of the database and no collective touches the data path
(transaction sharding, tensorfim_b200.shard, is for databases beyond one GPU's memory).  The only collective is the timing reduction: the job takes as long as its slowest
rank, and its throughput is the supports all ranks counted over that time (weak scaling).
Works on any torch.distributed backend (NCCL with CUDA tensors on the GPU box, gloo on CPU
in the tests).
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def world_size() -> int:
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def max_over_ranks(x: float, device: str | torch.device = "cpu") -> float:
    """The largest `x` over all ranks (every rank gets the same value)."""
    if world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(supports_per_replica: float, ms_slowest: float, world: int | None = None) -> float:
    """Supports per second of the whole job: every replica counts the same database."""
    w = world_size() if world is None else world
    return w * float(supports_per_replica) / (ms_slowest / 1000.0)
