"""Repeated executes replay the launch list as a CUDA graph (captured at the
second execute into the same output buffer): every replay must give the
eager execute's result bit for bit, for single plans (response and in-block
sweep leaves, FP64 and mixed) and for batches; a new output buffer or stage
profiling goes back to launch-by-launch execution, still bit for bit.
"""
import numpy as np
import pytest
import torch

from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _spec(pb, c):
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    return {"A": c.A, "B": c.B, "C": c.C, "D": c.D, "x0": c.x0, "u": u, "t0": c.t0, "t_end": c.t_end, "h": c.h,
            "solver": c.solver}


@pytest.mark.parametrize("solver,n,T,precision,path", [(0, 64, 50000, 1, 0), (1, 16, 20000, 0, 0),
                                                       (0, 32, 30000, 1, 4), (1, 40, 8000, 1, 0)])
def test_plan_graph_replay_is_bit_exact(pb, solver, n, T, precision, path):
    c = wl.small(9100 + n + T, solver, n, max(1, n // 8), max(1, n // 8), T, h=1e-3)
    s = _spec(pb, c)
    pb.set_option(pb.OPT_PATH, path)
    try:
        plan = pb.Plan(c.A, c.B, c.C, c.D, c.x0, s["u"], c.t0, c.t_end, c.h, solver=solver, precision=precision)
    finally:
        pb.set_option(pb.OPT_PATH, 0)
    y = torch.empty((plan.num_outputs, plan.channels), dtype=torch.float64, device="cuda")
    outs = []
    for _ in range(4):  # eager, capture + replay, replay, replay
        y.fill_(float("nan"))
        plan.execute(y.data_ptr())
        torch.cuda.synchronize()
        outs.append(y.cpu().numpy().copy())
    y2 = torch.empty_like(y)  # another buffer: eager again
    plan.execute(y2.data_ptr())
    torch.cuda.synchronize()
    outs.append(y2.cpu().numpy())
    plan.set_profiling(True)  # profiled: eager
    y.fill_(float("nan"))
    plan.execute(y.data_ptr())
    torch.cuda.synchronize()
    outs.append(y.cpu().numpy())
    plan.close()
    for k, o in enumerate(outs[1:], 1):
        assert np.array_equal(o, outs[0]), k


def test_batch_graph_replay_is_bit_exact(pb):
    cases = [wl.small(9200 + k, k % 2, 4 + 11 * k, 1 + k % 3, 1 + k % 2, 1500 + 700 * k, h=1e-3) for k in range(9)]
    b = pb.Batch([_spec(pb, c) for c in cases], precision=pb.MIXED)
    outs = []
    for _ in range(4):
        b.execute()
        torch.cuda.synchronize()
        outs.append([b.output(i)[1] for i in range(len(cases))])
    b.close()
    for k in range(1, 4):
        for i in range(len(cases)):
            assert np.array_equal(outs[k][i], outs[0][i]), (k, i)
