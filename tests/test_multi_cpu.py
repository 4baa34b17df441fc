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


# ---- time partition of one solve ------------------------------------------
# The split the library's shard plans make (multi.time_shard_layout) and the
# exchange between its two phases, with the device's chunked carry restated in
# numpy: each rank up-sweeps its blocks' aggregates k levels from a zero state,
# the ranks all-gather their level-k items (gloo), every rank scans the
# gathered sequence seeded with x0 and down-sweeps its own levels.  The block
# states must equal the sequential recurrence X_{b+1} = Q X_b + G_b.

def _chunk_up(items, Q):
    """Level above: aggregates of chunks of 16 (a short last chunk padded with
    zero items at its end, as on the device)."""
    d = items.shape[1]
    out = []
    for c0 in range(0, len(items), 16):
        x = np.zeros(d)
        for j in range(16):
            g = items[c0 + j] if c0 + j < len(items) else np.zeros(d)
            x = Q @ x + g
        out.append(x)
    return np.array(out).reshape(-1, d)


def _chunk_down(items, Q, carries):
    """Items of a level rewritten to the states entering them, from the
    states entering their chunks."""
    out = np.empty_like(items)
    for c, x in enumerate(carries):
        for j in range(16):
            i = 16 * c + j
            if i >= len(items):
                break
            out[i] = x
            x = Q @ x + items[i]
    return out


def _exclusive_scan(items, Q, x0):
    out = np.empty_like(items)
    x = x0.copy()
    for i, g in enumerate(items):
        out[i] = x
        x = Q @ x + g
    return out


def _time_problem(n_blocks, d=6, seed=11):
    rng = np.random.default_rng(seed)
    M = rng.standard_normal((d, d))
    Q = 0.9 * M / np.max(np.abs(np.linalg.eigvals(M)))
    return Q, rng.standard_normal((n_blocks, d)), rng.standard_normal(d)


def _time_worker(rank, world, port, n_blocks, out):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        Q, G, x0 = _time_problem(n_blocks)
        k, c, ranges = multi.time_shard_layout(n_blocks, world)
        b0, b1 = ranges[rank]
        # up: k levels inside the shard
        levels = [G[b0:b1]]
        for lev in range(k):
            levels.append(_chunk_up(levels[-1], np.linalg.matrix_power(Q, 16 ** lev)))
        top = np.zeros((c, Q.shape[0]))
        top[:len(levels[k])] = levels[k]
        gathered = [torch.zeros(c * Q.shape[0], dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, torch.from_numpy(top.reshape(-1)))
        seq = np.concatenate([g.numpy().reshape(c, -1) for g in gathered])
        prefixes = _exclusive_scan(seq, np.linalg.matrix_power(Q, 16 ** k), x0)
        carries = prefixes[rank * c:rank * c + len(levels[k])]
        for lev in range(k - 1, -1, -1):
            carries = _chunk_down(levels[lev], np.linalg.matrix_power(Q, 16 ** lev), carries)
        out[rank] = (b0, b1, carries)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_blocks,world", [(3 * 4096 + 77, 2), (700, 2), (37, 2), (5000, 3)])
def test_time_partition_decomposition_gloo(n_blocks, world):
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_time_worker, args=(r, world, port, n_blocks, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs)
    Q, G, x0 = _time_problem(n_blocks)
    ref = _exclusive_scan(G, Q, x0)
    covered = 0
    for r in range(world):
        b0, b1, states = out[r]
        assert b0 == covered and states.shape[0] == b1 - b0
        np.testing.assert_allclose(states, ref[b0:b1], rtol=1e-11, atol=1e-11)
        covered = b1
    assert covered == n_blocks


def test_time_shard_layout_rules():
    for n_blocks in (1, 15, 16, 17, 255, 256, 4096, 65536, 100003):
        for shards in (1, 2, 3, 4, 8):
            if shards > n_blocks:
                continue
            per = -(-n_blocks // shards)
            if per < 256 and -(-n_blocks // per) < shards:
                # equal shares of `per` blocks fill fewer shards: refused
                with pytest.raises(ValueError):
                    multi.time_shard_layout(n_blocks, shards)
                continue
            k, c, ranges = multi.time_shard_layout(n_blocks, shards)
            S = c * 16 ** k
            assert ranges[0][0] == 0 and ranges[-1][1] == n_blocks
            assert all(b - a == S for a, b in ranges[:-1]) and 0 < ranges[-1][1] - ranges[-1][0] <= S
            assert c < 256 and (k == 0 or c >= 16)
