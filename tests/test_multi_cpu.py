"""The N>1 path on CPU: world_size 2 with the gloo backend.

Ranks shard independent systems without communicating (every rank computes
the same assignment), solve their shard (here with the CPU oracle, standing
in for the GPU solve), and reduce the report: max time, summed work.  The
union of the shards must be the whole set, disjoint, balanced by cost, and
the gathered results must equal a single-rank run.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from parode_b200 import multi
from parode_b200 import workloads as wl


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _cases():
    return [wl.small(300 + k, k % 2, 2 + (k * 5) % 9, 1, 1, 40 + 17 * k, h=1e-2) for k in range(10)]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from oracle import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cases = _cases()
        mine = multi.shard(cases, rank, world, multi.system_cost)
        ys = {}
        work = 0.0
        for i in mine:
            c = cases[i]
            y = oracle.simulate_affine(oracle.System(c.A, c.B, c.C, c.D, c.x0),
                                       oracle.Input.sinusoid(c.u.a, c.u.f, c.u.phi), c.solver, c.t0, c.t_end, c.h)
            ys[i] = y
            work += c.n * y.shape[0]
        ms, total, rate = multi.reduce_report(dist, torch.device("cpu"), 10.0 + rank, work)
        gathered = [None] * world
        dist.all_gather_object(gathered, ys)
        out[rank] = (mine, ms, total, gathered if rank == 0 else None)
    finally:
        dist.destroy_process_group()


def test_shard_is_a_balanced_partition():
    cases = _cases()
    parts = [multi.shard(cases, r, 3, multi.system_cost) for r in range(3)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(cases)))
    loads = [sum(multi.system_cost(cases[i]) for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(multi.system_cost(c) for c in cases)
    with pytest.raises(ValueError):
        multi.shard(cases, 3, 3)


def test_world2_gloo_shards_and_reduces():
    from oracle import oracle

    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    mine0, ms0, total0, gathered = out[0]
    mine1, ms1, total1, _ = out[1]
    assert sorted(mine0 + mine1) == list(range(10)) and not set(mine0) & set(mine1)
    assert ms0 == ms1 == 11.0  # the slower rank's time, on every rank
    assert total0 == total1
    cases = _cases()
    merged = {}
    for part in gathered:
        merged.update(part)
    for i, c in enumerate(cases):
        ref = oracle.simulate_affine(oracle.System(c.A, c.B, c.C, c.D, c.x0),
                                     oracle.Input.sinusoid(c.u.a, c.u.f, c.u.phi), c.solver, c.t0, c.t_end, c.h)
        assert np.array_equal(merged[i], ref)
    assert total0 == sum(c.n * merged[i].shape[0] for i, c in enumerate(cases))
