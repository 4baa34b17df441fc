"""Multi-GPU helpers: one process per GPU, independent systems sharded across
ranks (no data-path collective), timing reduced as the maximum over ranks.

The batched and serving forms solve independent systems, so N GPUs take
disjoint shards of the system list and the only cross-rank traffic is the
reduction of the timings and counters for the report (torch.distributed:
NCCL on GPUs, gloo on CPU).

One long solve can also be split over the ranks by time (the reference's
only multi-device mechanism: a share of the horizon per device, each
device's up-sweep, the devices' totals carried across, each device's
down-sweep; Sources/RungeKutta4thOrder.cpp:96-125,
Sources/GPUFixedStepIterative.cpp:296-337).  `time_shard_layout` is the
split; `solve_time_partitioned` runs a rank's shard through the library's
shard plans with one all-gather of the shards' chunk aggregates between the
two phases; `emulate_time_partition` runs every shard on one device.
"""
from __future__ import annotations

from typing import Callable, List, Sequence, TypeVar

import numpy as np

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


def time_shard_layout(n_blocks: int, shards: int):
    """The split of n_blocks blocks over `shards` ranks, as the library makes
    it (solver.cpp, Plan::setup_shard): every shard but the last holds
    S = c 16^k blocks, with c in [16, 256) once a rank's share reaches 256
    blocks (else k = 0 and c the share), so the chunked carry's first k levels
    stay inside a shard and the shards' level-k chunk aggregates, c per shard,
    line up as one sequence.  Returns (k, c, [(first block, end block)])."""
    if shards < 1 or n_blocks < 1:
        raise ValueError("need at least one shard and one block")
    per = -(-n_blocks // shards)
    k, p16 = 0, 1
    while p16 * 256 <= per:
        p16 *= 16
        k += 1
    c = -(-per // p16)
    S = p16 * c
    ranges = [(r * S, min((r + 1) * S, n_blocks)) for r in range(shards)]
    if ranges[-1][0] >= n_blocks:
        raise ValueError("more shards than the horizon's blocks fill")
    return k, c, ranges


def solve_time_partitioned(pb, dist, device, A, B, Cm, D, x0, u_index, t0, t_end, h, solver=0, precision=0,
                           stream=None):
    """This rank's shard of one solve split by time over the process group.

    Each rank makes its shard plan, runs the up phase into its items, the
    group all-gathers the items (NCCL over NVLink: shards x items x NP
    doubles), and the rank finishes its steps.  Returns (plan, y) with y the
    rank's rows on the device (plan.num_outputs x plan.channels, rows per the
    plan's shard_info); plan.output() gives the host copy and time slice."""
    import torch

    rank, world = dist.get_rank(), dist.get_world_size()
    plan = pb.Plan(A, B, Cm, D, x0, u_index, t0, t_end, h, solver=solver, precision=precision, shard=rank,
                   shards=world)
    _, _, c, np_, shards = plan.shard_info
    if shards != world:
        raise RuntimeError("shard plan does not match the process group")
    top = torch.zeros(c * np_, dtype=torch.float64, device=device)
    gathered = torch.empty(world * c * np_, dtype=torch.float64, device=device)
    y = torch.empty((plan.num_outputs, plan.channels), dtype=torch.float64, device=device)
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream(device).cuda_stream
    plan.shard_up(top.data_ptr(), s)
    torch.cuda.synchronize(device)
    dist.all_gather_into_tensor(gathered, top)
    torch.cuda.synchronize(device)
    plan.shard_down(gathered.data_ptr(), y.data_ptr(), s)
    torch.cuda.synchronize(device)
    return plan, y


def emulate_time_partition(pb, A, B, Cm, D, x0, u_index, t0, t_end, h, shards, solver=0, precision=0):
    """Every shard of a time-partitioned solve on the current device, one
    after another (the all-gather is a device copy into one buffer): the
    whole horizon's y, assembled on the host from the shards' rows."""
    import torch

    plans = [pb.Plan(A, B, Cm, D, x0, u_index, t0, t_end, h, solver=solver, precision=precision, shard=r,
                     shards=shards) for r in range(shards)]
    infos = [p.shard_info for p in plans]
    c, np_ = infos[0][2], infos[0][3]
    gathered = torch.zeros(shards * c * np_, dtype=torch.float64, device="cuda")
    for r, p in enumerate(plans):
        p.shard_up(gathered[r * c * np_:(r + 1) * c * np_].data_ptr())
    torch.cuda.synchronize()
    parts = []
    for r, p in enumerate(plans):
        y = torch.empty((p.num_outputs, p.channels), dtype=torch.float64, device="cuda")
        p.shard_down(gathered.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        parts.append(y.cpu().numpy())
    ybase = 3 if solver == 1 else 0
    y = np.concatenate([parts[0]] + [q[ybase:] for q in parts[1:]], axis=0)
    for p in plans:
        p.close()
    return y, infos
