"""Replica runs over several GPUs of one node.

One SpMV of one matrix has no exchange step, so the multi-GPU form of the
path is N independent replicas, one process per GPU (torchrun): every rank
builds the same matrix and times the same steps, and the job's figure is the
bytes all ranks processed over the slowest rank's time.  These helpers hold
that host logic; they work with any torch.distributed backend (NCCL on the
GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import os


def rank_info() -> tuple[int, int, int]:
    """(rank, local rank, world size) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def max_over_ranks(value: float, device=None) -> float:
    """The largest of every rank's value (the value itself without a process
    group).  device: where the reduction tensor lives (a CUDA device for NCCL;
    None = CPU, for gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(bytes_per_step_per_rank: float, slowest_seconds_per_step: float, world: int) -> float:
    """Whole-job throughput in GB/s: every rank's bytes over the slowest
    rank's time per step (weak scaling: each rank does a full step)."""
    if slowest_seconds_per_step <= 0:
        raise ValueError("time per step must be positive")
    return world * bytes_per_step_per_rank / slowest_seconds_per_step / 1e9
