"""Multi-GPU helpers: one process per GPU, independent systems sharded across
ranks (no data-path collective), timing reduced as the maximum over ranks.

The batched and serving forms solve independent systems, so N GPUs take
disjoint shards of the system list and the only cross-rank traffic is the
reduction of the timings and counters for the report (torch.distributed:
NCCL on GPUs, gloo on CPU).  A single long system is replicated per rank
(replicas only): splitting one scan across GPUs would need an exchange of
shard totals, which is not built.
"""
from __future__ import annotations

from typing import Callable, List, Sequence, TypeVar

T = TypeVar("T")


def shard(items: Sequence[T], rank: int, world: int, cost: Callable[[T], float] = None) -> List[int]:
    """Indices of the items rank `rank` of `world` solves.

    Largest-cost-first assignment to the least-loaded rank (deterministic:
    every rank computes the same assignment without communicating); ties keep
    the original order.  With no cost function every item costs 1."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank / world out of range")
    costs = [float(cost(x)) if cost else 1.0 for x in items]
    order = sorted(range(len(items)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    owner = [0] * len(items)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(items)) if owner[i] == rank]


def system_cost(case) -> float:
    """Work estimate of one solve: scan dimension squared times steps."""
    return float(case.scan_dim) ** 2 * float(case.T)


def reduce_report(dist, device, elapsed_ms: float, state_steps: float):
    """Max elapsed time and summed state*steps over ranks (the whole-job
    throughput is the sum of work over the slowest rank's time)."""
    import torch

    t = torch.tensor([elapsed_ms], dtype=torch.float64, device=device)
    w = torch.tensor([state_steps], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    ms, work = float(t.item()), float(w.item())
    return ms, work, (work / (ms / 1e3) if ms > 0 else 0.0)
