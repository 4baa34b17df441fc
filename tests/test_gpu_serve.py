"""GPU tests of the serving loop (ParODE_Server*): continuous batching.

Requests are submitted with Poisson gaps while earlier ones run; every result
must equal the same solve done alone (the single-system entry point) and the
FP64 oracle, to the plain-scan gate (1e-12) in FP64 and to the mixed bound
(1e-6) in the mixed form.  The HBM budget must bound the device bytes in
flight, and a request larger than the budget must be refused.
"""
import time

import numpy as np
import pytest

from oracle import oracle
from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_MIXED = 1e-6


def _oracle_y(case):
    sysd = oracle.System(case.A, case.B, case.C, case.D, case.x0)
    inp = oracle.Input.sinusoid(case.u.a, case.u.f, case.u.phi)
    return oracle.simulate_affine(sysd, inp, case.solver, case.t0, case.t_end, case.h)


def _run_mix(pb, server, reqs, speedup=1.0):
    ids = []
    t0 = time.monotonic()
    for arrival, c in reqs:
        delay = t0 + arrival / speedup - time.monotonic()
        if delay > 0:
            time.sleep(delay)
        u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
        ids.append((server.submit(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver), c))
    return [(c, server.wait(rid, timeout_s=120)) for rid, c in ids]


@pytest.mark.parametrize("precision", [0, 1])
def test_serve_mix_equals_alone(pb, precision):
    reqs = wl.cfg5(24, rate=2000.0, seed=4242, n_range=(4, 40), T_range=(50, 4000))
    server = pb.Server(precision=precision, hbm_budget_bytes=8e9, max_batch=6, max_inflight=3)
    results = _run_mix(pb, server, reqs)
    tol = TOL_FP64 if precision == 0 else TOL_MIXED
    for c, (t, y, lat) in results:
        ref = _oracle_y(c)
        assert y.shape == ref.shape
        assert oracle.rel_err(y, ref) <= tol, (c.name, oracle.rel_err(y, ref))
        u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
        _, alone = pb.simulate(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver,
                               precision=precision)
        assert oracle.rel_err(y, alone) <= tol, c.name
        assert lat > 0
    st = server.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["batches"] >= 2  # requests arrived while others ran
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    server.close()


def test_serve_budget_bounds_inflight_bytes(pb):
    reqs = wl.cfg5(10, rate=5000.0, seed=99, n_range=(20, 60), T_range=(2000, 6000))
    budget = 64e6
    server = pb.Server(precision=0, hbm_budget_bytes=budget, max_batch=8, max_inflight=4)
    results = _run_mix(pb, server, reqs, speedup=1e9)
    for c, (t, y, lat) in results:
        assert oracle.rel_err(y, _oracle_y(c)) <= TOL_FP64
    st = server.stats()
    assert st["completed"] == len(reqs)
    assert 0 < st["peak_bytes"] <= budget
    server.close()


def test_serve_rejects_request_above_budget(pb):
    c = wl.small(5, 0, 64, 4, 4, 200000, h=1e-4)
    server = pb.Server(precision=0, hbm_budget_bytes=1e6)
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    with pytest.raises(pb.ParODEError) as e:
        server.submit(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h)
    assert e.value.code == -4
    server.close()
