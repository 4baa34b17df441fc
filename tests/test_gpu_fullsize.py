"""GPU parity at the benchmark configurations' full sizes, against the FP64 oracle O1.

  cfg3  ABM4 n=128 (scan dimension 512), m=p=16, h=5e-4, T=2^18: FP64 and mixed
  ABM at the T=2^20 bound of the mixed form (scan dimensions 64 and 128)
  cfg4  all 4096 systems of the batched workload, FP64 and mixed
  cfg5  serving requests across the serving ranges (n up to 256, T up to 10^6,
        RK4 / ABM 50/50), through the server and alone

Gates (per output channel max_k |y - y_oracle| / max_k |y_oracle|, maximum over
channels): 1e-12 for the FP64 form, 1e-6 for the mixed form.  Each test prints
its worst relative error (pytest -s shows it).  The oracle runs the systems of a
set on all host threads (oracle.simulate_affine_many).
"""
import math

import numpy as np
import pytest

from oracle import oracle
from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_MIXED = 1e-6


def _job(c):
    return (oracle.System(c.A, c.B, c.C, c.D, c.x0), oracle.Input.sinusoid(c.u.a, c.u.f, c.u.phi), c.solver, c.t0,
            c.t_end, c.h)


def _spec(pb, c):
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    return {"A": c.A, "B": c.B, "C": c.C, "D": c.D, "x0": c.x0, "u": u, "t0": c.t0, "t_end": c.t_end, "h": c.h,
            "solver": c.solver}


def _solve(pb, c, precision):
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    _, y = pb.simulate(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver, precision=precision)
    return y


@pytest.fixture(scope="module")
def cfg3_ref():
    c = wl.cfg3()
    return c, oracle.simulate_affine_many([_job(c)])[0]


@pytest.mark.parametrize("precision,tol", [(0, TOL_FP64), (1, TOL_MIXED)])
def test_cfg3_full_size(pb, cfg3_ref, precision, tol):
    c, ref = cfg3_ref
    y = _solve(pb, c, precision)
    assert y.shape == ref.shape == (c.T, c.p)  # the horizon rule gives T outputs for ABM too
    err = oracle.rel_err(y, ref)
    print(f"cfg3 ABM n=128 T=2^18 precision={precision}: rel err {err:.3e}")
    assert err <= tol, err


ABM_2_20 = [(16, 2, 2), (32, 4, 4)]  # (n, m, p): scan dimensions 64 and 128


@pytest.fixture(scope="module")
def abm_2_20_refs():
    cases = [wl.lti(wl.Rng(4100 + n), f"abm{n}", 1, n, m, p, -1.0, 0.4, 5e-4, 1 << 20, max_re=-0.2)
             for n, m, p in ABM_2_20]
    return cases, oracle.simulate_affine_many([_job(c) for c in cases])


@pytest.mark.parametrize("k", range(len(ABM_2_20)))
@pytest.mark.parametrize("precision,tol", [(1, TOL_MIXED), (0, TOL_FP64)])
def test_abm_at_2_20(pb, abm_2_20_refs, k, precision, tol):
    cases, refs = abm_2_20_refs
    c, ref = cases[k], refs[k]
    y = _solve(pb, c, precision)
    err = oracle.rel_err(y, ref)
    print(f"ABM n={c.n} T=2^20 precision={precision}: rel err {err:.3e}")
    assert err <= tol, err


@pytest.fixture(scope="module")
def cfg4_refs():
    cases = wl.cfg4()
    return cases, oracle.simulate_affine_many([_job(c) for c in cases])


@pytest.mark.parametrize("precision,tol", [(1, TOL_MIXED), (0, TOL_FP64)])
def test_cfg4_every_system(pb, cfg4_refs, precision, tol):
    """All 4096 systems of the batched workload in one batch."""
    cases, refs = cfg4_refs
    batch = pb.Batch([_spec(pb, c) for c in cases], precision=precision)
    batch.execute()
    worst, where = 0.0, -1
    for i, c in enumerate(cases):
        _, y = batch.output(i)
        assert y.shape == refs[i].shape, i
        e = oracle.rel_err(y, refs[i])
        if e > worst or math.isnan(e):
            worst, where = e, i
    batch.close()
    c = cases[where]
    print(f"cfg4 4096 systems precision={precision}: worst rel err {worst:.3e} (system {where}: "
          f"{'RK4' if c.solver == 0 else 'ABM'} n={c.n} T={c.T})")
    assert worst <= tol, (where, worst)


def _cfg5_cases():
    """Requests spanning the serving ranges: n in [8, 256], T in [10^3, 10^6],
    RK4 / ABM alternating, m = p = max(1, n / 8), A = -(1 + U) I + 0.5 G / sqrt(n),
    h = 1e-3 (the serving workload's generator)."""
    shapes = [(0, 256, 20000), (1, 256, 6000), (0, 8, 1000000), (1, 8, 1000000), (0, 40, 300000),
              (1, 64, 80000), (0, 128, 60000), (1, 20, 400000), (0, 90, 1000), (1, 150, 3000)]
    out = []
    for k, (solver, n, T) in enumerate(shapes):
        rng = wl.Rng(5200 + k)
        m = p = max(1, n // 8)
        diag = -(1.0 + float(rng.uniform(1)[0]))
        out.append(wl.lti(rng, f"serve{k}", solver, n, m, p, diag, 0.5, 1e-3, T))
    return out


@pytest.fixture(scope="module")
def cfg5_refs():
    cases = _cfg5_cases()
    return cases, oracle.simulate_affine_many([_job(c) for c in cases])


@pytest.mark.parametrize("precision,tol", [(1, TOL_MIXED), (0, TOL_FP64)])
def test_cfg5_range_requests_served(pb, cfg5_refs, precision, tol):
    """Submitted together to the server (so they share batches), each result
    matches the oracle and the same solve run alone."""
    cases, refs = cfg5_refs
    server = pb.Server(precision=precision, hbm_budget_bytes=150e9, max_batch=4, max_inflight=4)
    ids = [server.submit(s["A"], s["B"], s["C"], s["D"], s["x0"], s["u"], s["t0"], s["t_end"], s["h"],
                         solver=s["solver"]) for s in (_spec(pb, c) for c in cases)]
    worst = worst_alone = 0.0
    for rid, c, ref in zip(ids, cases, refs):
        _, y, _lat = server.wait(rid, timeout_s=600)
        assert y.shape == ref.shape, c.name
        e = oracle.rel_err(y, ref)
        alone = _solve(pb, c, precision)
        ea = oracle.rel_err(y, alone)
        print(f"  {c.name}: {'RK4' if c.solver == 0 else 'ABM'} n={c.n} T={c.T}: vs oracle {e:.3e}, "
              f"vs alone {ea:.3e}")
        worst, worst_alone = max(worst, e), max(worst_alone, ea)
        assert e <= tol, (c.name, e)
        assert ea <= tol, (c.name, ea)
    st = server.stats()
    server.close()
    print(f"cfg5-range requests precision={precision}: worst rel err {worst:.3e} vs oracle, "
          f"{worst_alone:.3e} vs alone, {int(st['batches'])} batches")
    assert st["completed"] == len(cases) and st["failed"] == 0
