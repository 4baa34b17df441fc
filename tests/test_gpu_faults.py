"""Failure detection without a GPU fault: injected on the host, reported as
error codes, and the library keeps working afterwards.

  - PARODE_OPT_FAULT_ALLOC makes the k-th device allocation fail as if the
    device were out of memory: the single solve, the batch and the served
    request each report -4 (NotEnoughResources), and the next call succeeds.
  - PARODE_OPT_FAULT_WITHHOLD makes the mixed-precision tensor-core kernel
    withhold the arrive of one pipeline stage in its first CTA: every wait on
    that stage gives up after its bound (about a second), the kernel records
    the time-out in its status word and returns, the solve reports -10
    (DeviceError), and a following solve on the same device is correct.
Nothing here traps, faults or hangs the GPU.
"""
import time

import numpy as np
import pytest

from oracle import oracle
from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _oracle_y(c):
    return oracle.simulate_affine(oracle.System(c.A, c.B, c.C, c.D, c.x0),
                                  oracle.Input.sinusoid(c.u.a, c.u.f, c.u.phi), c.solver, c.t0, c.t_end, c.h)


def _solve(pb, c, precision=0):
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    return pb.simulate(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver, precision=precision)[1]


@pytest.mark.parametrize("precision", [0, 1])
def test_injected_allocation_failure_in_a_solve(pb, precision):
    """Every allocation site of the solve in turn (the plan's buffers are one
    carved allocation; the mixed form's tensor-core set-up adds more): each
    failure reports -4 and the plan gives back what it took, until k passes
    the last site and the solve runs."""
    c = wl.small(61, 0, 24, 3, 3, 3000, h=1e-3)
    k = 0
    y = None
    try:
        while k < 64:
            pb.set_option(pb.OPT_FAULT_ALLOC, k)
            try:
                y = _solve(pb, c, precision)
            except pb.ParODEError as e:
                assert e.code == -4, (k, e.code)
                k += 1
                continue
            break
    finally:
        pb.set_option(pb.OPT_FAULT_ALLOC, -1)
    assert 1 <= k < 64, k
    tol = 1e-12 if precision == 0 else 1e-6
    assert oracle.rel_err(y, _oracle_y(c)) <= tol
    assert oracle.rel_err(_solve(pb, c, precision), _oracle_y(c)) <= tol


def test_injected_allocation_failure_in_a_batch(pb):
    cases = [wl.small(70 + i, i % 2, 6 + 5 * i, 2, 2, 900 + 300 * i, h=1e-3) for i in range(4)]
    specs = []
    for c in cases:
        u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
        specs.append({"A": c.A, "B": c.B, "C": c.C, "D": c.D, "x0": c.x0, "u": u, "t0": c.t0, "t_end": c.t_end,
                      "h": c.h, "solver": c.solver})
    pb.set_option(pb.OPT_FAULT_ALLOC, 0)
    try:
        with pytest.raises(pb.ParODEError) as e:
            pb.Batch(specs)
        assert e.value.code == -4
    finally:
        pb.set_option(pb.OPT_FAULT_ALLOC, -1)
    b = pb.Batch(specs)
    b.execute()
    for i, c in enumerate(cases):
        assert oracle.rel_err(b.output(i)[1], _oracle_y(c)) <= 1e-12
    b.close()


def test_injected_allocation_failure_in_a_served_request(pb):
    c = wl.small(81, 1, 10, 2, 2, 2000, h=1e-3)
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    server = pb.Server(precision=0, hbm_budget_bytes=4e9, max_batch=1, max_inflight=1)
    try:
        pb.set_option(pb.OPT_FAULT_ALLOC, 0)
        rid = server.submit(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver)
        with pytest.raises(pb.ParODEError) as e:
            server.wait(rid, timeout_s=60)
        assert e.value.code == -4
        pb.set_option(pb.OPT_FAULT_ALLOC, -1)
        rid = server.submit(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver)
        _, y, _ = server.wait(rid, timeout_s=60)
        assert oracle.rel_err(y, _oracle_y(c)) <= 1e-12
        st = server.stats()
        assert st["failed"] == 1 and st["completed"] == 1
    finally:
        pb.set_option(pb.OPT_FAULT_ALLOC, -1)
        server.close()


def test_withheld_arrive_times_out_and_device_stays_usable(pb):
    # RK4 n=64 with inputs: the mixed form runs the tensor-core response kernel
    c = wl.small(91, 0, 64, 8, 8, 20000, h=1e-3)
    pb.set_option(pb.OPT_FAULT_WITHHOLD, 1)
    try:
        t0 = time.monotonic()
        with pytest.raises(pb.ParODEError) as e:
            _solve(pb, c, precision=1)
        elapsed = time.monotonic() - t0
        assert e.value.code == -10
        assert elapsed < 30.0  # the waits are bounded (about a second each)
    finally:
        pb.set_option(pb.OPT_FAULT_WITHHOLD, 0)
    assert oracle.rel_err(_solve(pb, c, precision=1), _oracle_y(c)) <= 1e-6
