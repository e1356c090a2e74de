"""Multi-GPU replicas: one process per GPU, independent work, no data-path collective.

The R^k path shards by independent units: ions, serving requests, and whole
(k, kappa-block) tables. Each rank runs the full engine on its own units.
The only collectives are scalar reductions of timings and counts, outside
the timed work, and a barrier on each side of the timed region.

* ``init``: the process group from the torchrun environment (RANK,
  WORLD_SIZE, LOCAL_RANK, MASTER_ADDR/PORT). NCCL is used when CUDA is
  present, gloo otherwise, with a short timeout so that ranks waiting for a
  dead peer end with an error.
* ``reduce_max`` / ``reduce_sum``: scalar reductions; the job time is the
  max over ranks.
* ``shard``: assigns units to ranks by estimated cost, longest first onto
  the least-loaded rank, so that ranks finish together.
"""
from __future__ import annotations

import os
from datetime import timedelta

import torch

__all__ = ["init", "reduce_max", "reduce_sum", "barrier", "shard", "finalize", "replica_seed"]


def init(backend: str | None = None, timeout_s: float = 120.0) -> tuple[int, int, int]:
    """(rank, world, local_rank); initialises the process group when world > 1."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return rank, world, local


def _reduce(x: float, world: int, op) -> float:
    if world == 1:
        return float(x)
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=op)
    return float(t.item())


def reduce_max(x: float, world: int) -> float:
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.MAX)


def reduce_sum(x: float, world: int) -> float:
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.SUM)


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def finalize(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def replica_seed(base: int, rank: int) -> int:
    """Seed of a rank's own replica of a seeded workload."""
    return int(base) + int(rank)


def shard(costs, world: int) -> list[list[int]]:
    """Indices of units per rank: longest first onto the least-loaded rank."""
    loads = [0.0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda j: -float(costs[j])):
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(o) for o in out]
