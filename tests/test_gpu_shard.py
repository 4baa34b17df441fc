"""Time partition of one solve (ParODE_PlanCreateShard / ShardUp / ShardDown).

Every shard of the split runs on this one device, one after another, with the
all-gather between the two phases done as a device copy
(parode_b200.multi.emulate_time_partition); the assembled y must equal the
unsplit solve and the FP64 oracle: per-channel relative error <= 1e-12 (FP64
form) or <= 1e-6 (mixed form).  The shard geometry must be the documented
layout (multi.time_shard_layout), each shard's time vector the horizon's
slice, and execute() is refused on a shard plan.
"""
import numpy as np
import pytest

from oracle import oracle
from parode_b200 import multi
from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _oracle(c):
    return oracle.simulate_affine(oracle.System(c.A, c.B, c.C, c.D, c.x0),
                                  oracle.Input.sinusoid(c.u.a, c.u.f, c.u.phi), c.solver, c.t0, c.t_end, c.h)


CASES = [  # solver, n, m, p, T, shards, precision
    (0, 16, 2, 2, 20000, 2, 0), (0, 32, 4, 4, 50000, 3, 1), (1, 8, 2, 2, 30000, 4, 0), (1, 16, 2, 2, 12345, 2, 1),
    (0, 64, 8, 8, 1 << 18, 4, 1), (0, 8, 1, 1, 3000, 3, 0), (1, 4, 1, 1, 700, 3, 1),
]


@pytest.mark.parametrize("solver,n,m,p,T,shards,precision", CASES)
def test_time_partition_matches_whole_solve(pb, solver, n, m, p, T, shards, precision):
    c = wl.small(8100 + n + T, solver, n, m, p, T, h=1e-3)
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    y, infos = multi.emulate_time_partition(pb, c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, shards,
                                            solver=solver, precision=precision)
    pb.set_option(pb.OPT_PATH, pb.PATH_BLOCKED_RESPONSE)  # the path the shards run
    try:
        whole = pb.Plan(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=solver, precision=precision)
    finally:
        pb.set_option(pb.OPT_PATH, 0)
    whole.execute()
    t_whole, y_whole = whole.output()
    B = whole.response_shape[0]
    nblocks = whole.response_shape[3]
    whole.close()
    # the documented layout
    k, cc, ranges = multi.time_shard_layout(nblocks, shards)
    for r, info in enumerate(infos):
        b0, b1 = ranges[r]
        assert info[0] == b0 * B and info[2] == cc and info[4] == shards, (r, info)
        assert info[0] + info[1] == min(b1 * B, y_whole.shape[0] - (3 if solver == 1 else 0)), (r, info)
    assert y.shape == y_whole.shape
    tol = 1e-12 if precision == 0 else 1e-6
    e_whole = oracle.rel_err(y, y_whole)
    e_oracle = oracle.rel_err(y, _oracle(c))
    print(f"{shards} shards solver={solver} n={n} T={T} precision={precision}: vs whole {e_whole:.2e}, "
          f"vs oracle {e_oracle:.2e} (k={k}, c={cc})")
    assert e_oracle <= tol, e_oracle
    assert e_whole <= tol, e_whole


def test_shard_time_slice_and_refused_execute(pb):
    c = wl.small(8200, 1, 8, 2, 2, 5000, h=1e-3)
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    t_all = oracle.time_vector(1, c.t0, c.t_end, c.h).astype(np.float64)
    plan = pb.Plan(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=1, shard=1, shards=2)
    begin, steps = plan.shard_info[:2]
    with pytest.raises(pb.ParODEError):
        plan.execute()
    import torch

    _, _, cc, np_, shards = plan.shard_info
    top = torch.zeros(cc * np_, dtype=torch.float64, device="cuda")
    plan.shard_up(top.data_ptr())
    gathered = torch.zeros(shards * cc * np_, dtype=torch.float64, device="cuda")
    plan.shard_down(gathered.data_ptr())
    t, _ = plan.output()
    plan.close()
    assert np.array_equal(t[3:], t_all[3 + begin:3 + begin + steps])
    assert np.array_equal(t[:3], t_all[:3])


def test_shard_needs_the_response_path(pb):
    c = wl.small(8300, 0, 80, 4, 4, 2000, h=1e-3)  # scan dimension 80 > 64
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    with pytest.raises(pb.ParODEError):
        pb.Plan(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=0, shard=0, shards=2)


@pytest.mark.parametrize("precision", [0, 1])
def test_time_partition_with_a_user_input_function(pb, precision):
    """An NVRTC-compiled UFunc: every shard samples it at the whole horizon's
    sample times (the sample index offset), so the split equals the unsplit
    solve bit for bit."""
    src = ("fType UFunc(fType t, int nInputIndex) {\n"
           "    return sin(3.0 * t + nInputIndex) + 0.5 * cos(7.0 * t);\n"
           "}\n")
    u = pb.register_input(src)
    c = wl.small(8400, 0, 16, 2, 2, 40000, h=1e-3)
    y, _ = multi.emulate_time_partition(pb, c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, 3, solver=0,
                                        precision=precision)
    pb.set_option(pb.OPT_PATH, pb.PATH_BLOCKED_RESPONSE)
    try:
        whole = pb.Plan(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=0, precision=precision)
    finally:
        pb.set_option(pb.OPT_PATH, 0)
    whole.execute()
    _, y_whole = whole.output()
    whole.close()
    assert np.array_equal(y, y_whole)
