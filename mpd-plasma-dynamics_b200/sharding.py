"""Batched steady solves over several GPUs of one node.

One process per GPU (``torch.distributed``: NCCL between GPUs, gloo for the
CPU tests).  The solves of a sweep are independent, so the work shards by
solve: each rank runs its share as one batch (``BatchSolver``) on its own
device and nothing crosses GPUs while solving.  The only collectives are the
maximum of the ranks' device times and the gather of the per-solve results on
rank 0 at the end.

Shares are balanced by estimated cost (cells x estimated steps to converge),
largest first onto the least-loaded rank; the assignment is deterministic, so
every rank computes it locally without communicating.

The reference runs one solve per MPI job (src/main.cpp); there is no
counterpart to batching or to this sharding in it.
"""
from __future__ import annotations

import dataclasses
import heapq
from typing import Callable, Sequence

import numpy as np

from .batch import estimated_steps


def solve_cost(cfg, max_steps: int) -> float:
    """Cell updates a cold solve of cfg's shape is expected to take."""
    return float(cfg.L_max * (cfg.M_max + 1) * estimated_steps(cfg, max_steps))


def shard(costs: Sequence[float], world: int) -> list[list[int]]:
    """Indices of the solves each of `world` ranks runs: longest processing
    time first onto the least-loaded rank (ties: lower index, lower rank).
    Every index appears in exactly one share; each share is in increasing
    order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shares]


def _dist():
    import torch.distributed as dist
    return dist


def _device_for(group=None):
    import torch
    dist = _dist()
    return torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")


def max_over_ranks(x: float, group=None) -> float:
    """The maximum of x over the ranks of the group (every rank gets it)."""
    import torch
    dist = _dist()
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_on_root(obj, group=None):
    """Rank 0: the list of every rank's obj in rank order; others: None."""
    dist = _dist()
    rank = dist.get_rank(group)
    out = [None] * dist.get_world_size(group) if rank == 0 else None
    dist.gather_object(obj, out, dst=0, group=group)
    return out


@dataclasses.dataclass
class ShardedResult:
    runs: list                 # per solve, in the sweep's order
    solve_ms: np.ndarray       # per solve: its batch's first step -> its last step
    device_ms: float           # the slowest rank's batch
    shares: list[list[int]]    # the solves each rank ran


def run_sharded(costs: Sequence[float], run_share: Callable, group=None) -> ShardedResult | None:
    """Run a sweep sharded over the group's ranks.  run_share(indices) runs
    this rank's solves and returns (runs, solve_ms, device_ms) for them, in
    the order given.  Rank 0 gets the merged result, the others None; every
    rank takes the same collective steps."""
    dist = _dist()
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    shares = shard(costs, world)
    mine = shares[rank]
    runs, solve_ms, device_ms = run_share(mine) if mine else ([], np.zeros(0), 0.0)
    if len(runs) != len(mine) or len(solve_ms) != len(mine):
        raise RuntimeError("run_share returned results for a different number of solves")
    slowest = max_over_ranks(device_ms, group)
    parts = gather_on_root((mine, list(runs), list(np.asarray(solve_ms, dtype=float))), group)
    if rank != 0:
        return None
    n = len(costs)
    all_runs: list = [None] * n
    all_ms = np.zeros(n)
    for idx, r, ms in parts:
        for j, i in enumerate(idx):
            all_runs[i] = r[j]
            all_ms[i] = ms[j]
    return ShardedResult(all_runs, all_ms, slowest, shares)
