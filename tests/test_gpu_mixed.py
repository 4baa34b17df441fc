"""GPU parity of the mixed-precision form against the CPU FP64 oracle: the
3xTF32 tcgen05 leaf (in-block sweeps, path 4) or the block-response GEMMs on
tcgen05 (aggregates and output windows, path 3), with the power table, the
carry and the initial-state part of the outputs in FP64.

Tolerance: per-channel relative error <= 1e-6 (max_k |y - y_oracle| /
max_k |y_oracle|), the bound the mixed form is specified to meet at T = 2^20.
"""
import numpy as np
import pytest

from oracle import oracle
from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-6


def _run(pb, case, precision, path=0):
    pb.set_option(pb.OPT_PATH, path)
    u = pb.register_sinusoid(case.u.a, case.u.f, case.u.phi)
    plan = pb.Plan(case.A, case.B, case.C, case.D, case.x0, u, case.t0, case.t_end, case.h, solver=case.solver,
                   precision=precision)
    plan.execute()
    _, y = plan.output()
    used = plan.precision
    plan.close()
    pb.set_option(pb.OPT_PATH, 0)
    return y, used


def _oracle(case):
    sysd = oracle.System(case.A, case.B, case.C, case.D, case.x0)
    inp = oracle.Input.sinusoid(case.u.a, case.u.f, case.u.phi)
    return oracle.simulate_affine(sysd, inp, case.solver, case.t0, case.t_end, case.h)


@pytest.mark.parametrize("solver,n,m,p,T", [(0, 16, 2, 2, 5000), (0, 24, 3, 4, 3000), (0, 32, 4, 4, 20000),
                                            (0, 48, 6, 6, 7777), (0, 64, 8, 8, 4096), (1, 4, 1, 1, 3000),
                                            (1, 8, 2, 2, 5000), (1, 16, 2, 2, 10000)])
@pytest.mark.parametrize("path", [0, 3, 4])
def test_mixed_parity(pb, solver, n, m, p, T, path):
    case = wl.small(500 + n + 3 * T + solver, solver, n, m, p, T, h=1e-3)
    y, used = _run(pb, case, pb.MIXED, path)
    assert used == pb.MIXED, "the tensor-core leaves should cover scan dimensions 16..64"
    err = oracle.rel_err(y, _oracle(case))
    assert err <= TOL_MIXED, err


@pytest.mark.parametrize("path", [0, 4])
def test_mixed_cfg2_full_size(pb, path):
    """The benchmark workload (RK4 n=64, T=2^20) in the mixed form."""
    case = wl.cfg2()
    y, used = _run(pb, case, pb.MIXED, path)
    assert used == pb.MIXED
    err = oracle.rel_err(y, _oracle(case))
    assert err <= TOL_MIXED, err


def test_mixed_falls_back_to_fp64_outside_its_shapes(pb):
    # scan dimension 8 (RK4 n=8): the tensor-core leaf needs N >= 16
    case = wl.small(9, 0, 8, 2, 2, 500, h=1e-2)
    y, used = _run(pb, case, pb.MIXED)
    assert used == pb.FP64
    assert oracle.rel_err(y, _oracle(case)) <= 1e-12
