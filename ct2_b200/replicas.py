"""Replica bookkeeping for multi-GPU runs of the gravity step.

The step has no exchange between GPUs (each rank integrates its own periodic
box), so a multi-GPU run is N independent replicas.  These helpers turn the
per-rank device times into the whole-job figures: the slowest rank's time
bounds the job, and the job's throughput is all ranks' particles over that
time.  They work with any torch.distributed backend (NCCL on GPUs, gloo on
CPU for tests).
"""
from __future__ import annotations


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks (identity when not distributed)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_throughput(particles_local: int, ms_local: float, device=None):
    """(particles/s of the whole job, max ms over ranks): every rank's
    particles divided by the slowest rank's time."""
    ms = max_over_ranks(ms_local, device)
    total = sum_over_ranks(particles_local, device)
    return total / (ms * 1e-3), ms
