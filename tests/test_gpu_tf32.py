"""GPU parity of the single-pass TF32 form (PARODE_PRECISION_TF32) against the
CPU FP64 oracle.

The block-response GEMMs (aggregates and output windows) run one TF32
product per term, both operands rounded to TF32 (2^-11 relative), with FP32
accumulation drained into FP64 every eight K slices; the carry and the
initial-state part of the outputs stay FP64.  Off the block-response path the
plan runs the mixed form and reports it; a batch always runs the mixed form.

Tolerance: per-channel relative error <= 2e-3 (max_k |y - y_oracle| /
max_k |y_oracle|): the operands' TF32 rounding left in.  Each test prints its
error (pytest -s).
"""
import pytest

from oracle import oracle
from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL_TF32 = 2e-3


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


@pytest.mark.parametrize("solver,n,m,p,T", [(0, 16, 2, 2, 5000), (0, 32, 4, 4, 20000), (0, 64, 8, 8, 4096),
                                            (1, 8, 2, 2, 5000), (1, 16, 2, 2, 10000)])
def test_tf32_parity(pb, solver, n, m, p, T):
    case = wl.small(900 + n + 3 * T + solver, solver, n, m, p, T, h=1e-3)
    y, used = _run(pb, case, pb.TF32, path=3)
    assert used == pb.TF32
    ref = _oracle(case)
    err = oracle.rel_err(y, ref)
    y3, _ = _run(pb, case, pb.MIXED, path=3)
    err3 = oracle.rel_err(y3, ref)
    print(f"TF32 solver={solver} n={n} T={T}: rel err {err:.3e} (mixed {err3:.3e})")
    assert err <= TOL_TF32, err
    assert err3 <= err or err3 <= 1e-6, (err3, err)


def test_tf32_cfg2_full_size(pb):
    """The benchmark workload (RK4 n=64, T=2^20) in the single-pass form."""
    case = wl.cfg2()
    y, used = _run(pb, case, pb.TF32)
    assert used == pb.TF32
    err = oracle.rel_err(y, _oracle(case))
    print(f"TF32 cfg2 T=2^20: rel err {err:.3e}")
    assert err <= TOL_TF32, err


def test_tf32_off_the_response_path_runs_mixed(pb):
    """The in-block sweep leaf has no single-pass form: the plan runs 3xTF32
    and reports MIXED; its result meets the mixed bound."""
    case = wl.small(931, 0, 32, 4, 4, 3000, h=1e-3)
    y, used = _run(pb, case, pb.TF32, path=4)
    assert used == pb.MIXED
    assert oracle.rel_err(y, _oracle(case)) <= 1e-6


def test_tf32_batch_runs_mixed(pb):
    case = wl.small(932, 0, 16, 2, 2, 4000, h=1e-3)
    u = pb.register_sinusoid(case.u.a, case.u.f, case.u.phi)
    spec = {"A": case.A, "B": case.B, "C": case.C, "D": case.D, "x0": case.x0, "u": u, "t0": case.t0,
            "t_end": case.t_end, "h": case.h, "solver": case.solver}
    b = pb.Batch([spec], precision=pb.TF32)
    b.execute()
    _, y = b.output(0)
    assert b.precision(0) in (pb.MIXED, pb.FP64)
    b.close()
    assert oracle.rel_err(y, _oracle(case)) <= 1e-6
