"""The one-shot calls (SimulateODE, ParODE_SimulateODE_d) run the output stage
of the block-response path over four block ranges and copy each range's rows
to the host while the later ranges are formed.  Their results must equal a
device plan's execute + get_output bit for bit (RK4 and ABM, ragged horizons,
FP64, mixed and single-pass TF32), and the float call must equal that output
rounded to float.
"""
import numpy as np
import pytest

from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("solver,n,T,precision", [(0, 64, 50001, 1), (1, 16, 30001, 1), (0, 32, 40000, 0),
                                                  (1, 8, 20003, 0), (0, 64, 65536, 2), (0, 8, 4099, 1)])
def test_pipelined_calls_equal_plan(pb, solver, n, T, precision):
    c = wl.small(9700 + n + T, solver, n, max(1, n // 8), max(1, n // 8), T, h=1e-3)
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    prev_path = pb.get_option(pb.OPT_PATH)
    pb.set_option(pb.OPT_PATH, pb.PATH_BLOCKED_RESPONSE)
    try:
        _check_case(pb, c, u, solver, precision)
    finally:
        pb.set_option(pb.OPT_PATH, prev_path)


def _check_case(pb, c, u, solver, precision):
    plan = pb.Plan(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=solver, precision=precision)
    assert plan.path == pb.PATH_BLOCKED_RESPONSE
    plan.execute()
    tp, yp = plan.output()
    t, y = pb.simulate(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=solver, precision=precision)
    assert np.array_equal(t, tp)
    assert np.array_equal(y, yp)

    # the float ABI: the system rounded to float, y rounded on the device
    f = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    plan32 = pb.Plan(f(c.A), f(c.B), f(c.C), f(c.D), f(c.x0), u, c.t0, c.t_end, c.h, solver=solver,
                     precision=precision)
    plan32.execute()
    _, y64 = plan32.output()
    prev = pb.get_option(pb.OPT_PRECISION)
    pb.set_option(pb.OPT_PRECISION, precision)
    try:
        t32, y32, err = pb.simulate_f32(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=solver)
    finally:
        pb.set_option(pb.OPT_PRECISION, prev)
    assert err == 0
    assert np.array_equal(t32, tp.astype(np.float32))
    assert np.array_equal(y32, y64.astype(np.float32))
