"""The reference C ABI's float output (SimulateODE with fType = float arrays):
y is rounded to float on the device and copied straight into the caller's
array, the time vector is written as float on the host.  Both must equal the
FP64 extension's results for the same float-rounded system, rounded to float,
bit for bit (RK4 and ABM, FP64 and mixed precision modes), also into
caller-owned arrays.
"""
import numpy as np
import pytest

from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("solver,n,T,precision", [(0, 16, 4097, 0), (1, 8, 3001, 0), (0, 64, 50000, 1),
                                                  (1, 16, 20000, 1)])
def test_float_abi_equals_rounded_fp64(pb, solver, n, T, precision):
    c = wl.small(9500 + n + T, solver, n, max(1, n // 8), max(1, n // 8), T, h=1e-3)
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    # the float ABI rounds the system to float first: solve the same rounded
    # system through the FP64 extension
    f = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    prev = pb.get_option(pb.OPT_PRECISION)
    pb.set_option(pb.OPT_PRECISION, precision)
    try:
        t32, y32, err = pb.simulate_f32(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=solver)
        Tn = pb.num_outputs(solver, c.t0, c.t_end, c.h)
        tp = np.empty(Tn, dtype=np.float32)
        yp = np.empty((Tn, y32.shape[1]), dtype=np.float32)
        t32b, y32b, err2 = pb.simulate_f32(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=solver,
                                           t_out=tp, y_out=yp)
    finally:
        pb.set_option(pb.OPT_PRECISION, prev)
    assert err == 0 and err2 == 0
    t64, y64 = pb.simulate(f(c.A), f(c.B), f(c.C), f(c.D), f(c.x0), u, c.t0, c.t_end, c.h, solver=solver,
                           precision=precision)
    assert np.array_equal(t32, t64.astype(np.float32))
    assert np.array_equal(y32, y64.astype(np.float32))
    assert np.shares_memory(t32b, tp) and np.shares_memory(y32b, yp)  # views of the caller's arrays
    assert np.array_equal(tp, t32) and np.array_equal(yp, y32)
