"""One process per GPU, independent replicas: the host-side rules of a multi-GPU run.

The sketch path has no exchange step: a graph stream lives on one GPU, and the batched and served
workloads split by tenant.  Ranks therefore share nothing on the data path; they meet only to line up
the timed region (a barrier) and to take the slowest rank's time (all-reduce MAX), and the whole-job
rate is the units every rank processed divided by that time.
"""
from __future__ import annotations

import os


def env_rank() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torch.distributed launcher's environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def replica_seed(base: int, rank: int) -> int:
    """Stream and sketch seeds of a replica: each rank ingests its own stream."""
    return (base + rank) & (2**64 - 1)


def tenant_shard(num_tenants: int, rank: int, world: int) -> list[int]:
    """Tenants a rank owns when a multi-tenant workload is split over ranks (round robin)."""
    return list(range(rank, num_tenants, world))


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """The slowest rank's value (all ranks get it)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, dist=None, device=None) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(units_all_ranks: float, ms_max: float) -> float:
    """Units per second of the whole job, timed by its slowest rank."""
    return units_all_ranks / (ms_max / 1e3)
