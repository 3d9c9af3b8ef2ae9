"""Multi-GPU plumbing for the data-parallel workloads (one process per GPU, torch.distributed).

The ERI microbenchmark and the batched-molecule workload shard into independent units (quartets,
molecules) with no data-path exchange: every rank evaluates its own units (weak scaling: a fixed amount
per rank), and the only collective is the max-over-ranks of the timed region.  A direct J/K build of ONE
molecule shards its quartet list (the library's qcg_set_shard: each rank evaluates a contiguous 1/world
slice of every class's screened quartets) and needs one sum-reduction of J and K; sharded_fock_jk does
both, reduce_jk the NCCL all-reduce.
"""
from __future__ import annotations

import os
from typing import List, Sequence

import numpy as np


def dist_env():
    """(rank, world_size, local_rank) from the torchrun environment; (0, 1, 0) when absent."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def shard_range(n: int, rank: int, world: int):
    """Contiguous, balanced [lo, hi) share of n units for one rank."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_weighted(costs: Sequence[float], world: int) -> List[List[int]]:
    """Greedy longest-processing-time assignment of weighted units (e.g. molecules) to ranks."""
    order = np.argsort(-np.asarray(costs, dtype=float), kind="stable")
    load = np.zeros(world)
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        out[r].append(int(i))
        load[r] += costs[i]
    for lst in out:
        lst.sort()
    return out


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (the timed region's duration) over all ranks; identity without a group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_jk(J, K):
    """Sum partial J and K (torch tensors, same shape on every rank) over all ranks in place."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(J)
        dist.all_reduce(K)
    return J, K


def sharded_fock_jk(engine, dD: int, dJ: int, dK: int, J, K, rank: int = None, world: int = None,
                    deterministic: bool = False):
    """One J/K build split over the ranks of the process group: this rank's slice into the device buffers
    dJ/dK (the data pointers of the torch tensors J and K), then the sum over ranks in place.  rank/world
    default to the process group's; deterministic=True accumulates each slice in exact integer pairs."""
    import torch.distributed as dist
    if rank is None or world is None:
        on = dist.is_available() and dist.is_initialized()
        rank, world = (dist.get_rank(), dist.get_world_size()) if on else (0, 1)
    engine.set_shard(rank, world)
    st = engine.fock_jk_device(dD, dJ, dK, deterministic=deterministic)
    reduce_jk(J, K)
    return st
