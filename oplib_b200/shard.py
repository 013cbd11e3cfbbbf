"""Work partitioning across GPUs (one process per GPU, torch.distributed for the plumbing).

* Monte Carlo: paths are a function of (seed, path id) only -- path p draws from
  MT19937 init_genrand(seed + p) -- so contiguous path-id ranges shard with no data
  exchange; the only collective is one all-reduce of the per-rank payoff sums (2 doubles).
* Batched lattices: lattices are independent; they are bin-packed by cost n^3 with the
  longest-processing-time rule and each rank solves its own set; quotes are gathered once.
* A single lattice does not shard (replicas only).
The reference runs its devices one after another with no inter-GPU data
(benchmarks/glv/Program.cs:56-59); nothing here crosses GPUs on the data path.
"""
from __future__ import annotations

import heapq

import torch


def path_range(npaths: int, rank: int, world: int) -> tuple[int, int]:
    """(first path id, count) of this rank's contiguous share of npaths paths."""
    base, extra = divmod(npaths, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def lpt_partition(costs, world: int) -> list[list[int]]:
    """Longest-processing-time assignment of items with the given costs to `world` bins:
    items in decreasing cost, each to the currently lightest bin (ties: lowest rank)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    bins: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        bins[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(b) for b in bins]


def allreduce_sums(sums: torch.Tensor) -> torch.Tensor:
    """Sum of the per-rank payoff sums (in place when a process group is initialised)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(sums, op=dist.ReduceOp.SUM)
    return sums


def gather_quotes(local: torch.Tensor, assignment: list[list[int]], nlat: int) -> torch.Tensor:
    """Reassemble per-rank quotes [len(assignment[rank]), ...] into [nlat, ...] on every rank."""
    import torch.distributed as dist
    world = len(assignment)
    if not (dist.is_available() and dist.is_initialized()) or world == 1:
        out = torch.empty((nlat,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
        out[assignment[0]] = local
        return out
    rank = dist.get_rank()
    width = max(len(a) for a in assignment)
    pad = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: len(assignment[rank])] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    out = torch.empty((nlat,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    for r in range(world):
        out[assignment[r]] = parts[r][: len(assignment[r])]
    return out
