"""Replica plumbing for running one time-stepping job per GPU.

The Taylor-Green workload fits one GPU and the reference's step has no data
exchange once everything is on one device, so N GPUs run N independent
replicas (weak scaling): no collective on the data path.  Across ranks there is
only the bookkeeping of a benchmark: a barrier before and after the timed
region, the slowest rank's time, and the aggregate rate.  This module holds that
bookkeeping, independent of the device (NCCL on GPUs, gloo on CPUs), so it can
be exercised without GPUs.
"""
from __future__ import annotations

import os
from datetime import timedelta


def dist_env():
    """(rank, world_size, local_rank) from the torchrun environment; 1 rank without it."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(world: int, backend: str, timeout_s: float = 120.0) -> None:
    """Join the process group (rendezvous from MASTER_ADDR / MASTER_PORT) when world > 1."""
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))


def shutdown(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def barrier(world: int, sync=None) -> None:
    """Device synchronisation (sync, e.g. torch.cuda.synchronize), then a barrier over ranks."""
    if sync is not None:
        sync()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int, device: str = "cpu") -> float:
    """The largest x over all ranks (the slowest replica's time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Whole-job rate: the units every rank processed over the slowest rank's time."""
    return world * units_per_rank / max_seconds
