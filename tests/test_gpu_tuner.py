"""The measured block-length tuner of the block-response leaf (ParODE_TuneResponseBlock).

For a class of systems it times the candidate block lengths on the device and
records the fastest; a solve of a system of that class then runs with it, and
still matches the FP64 oracle to the gate of its precision form.
"""
import pytest

from oracle import oracle
from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _oracle(c):
    return oracle.simulate_affine(oracle.System(c.A, c.B, c.C, c.D, c.x0),
                                  oracle.Input.sinusoid(c.u.a, c.u.f, c.u.phi), c.solver, c.t0, c.t_end, c.h)


@pytest.mark.parametrize("solver,n,m,p,T,precision", [(0, 64, 8, 8, 1 << 16, 1), (1, 24, 3, 3, 20000, 0),
                                                      (0, 40, 5, 5, 30000, 0)])
def test_tuned_block_length_is_used_and_correct(pb, solver, n, m, p, T, precision):
    try:
        R, best, model = pb.tune_response_block(solver, n, m, p, T, precision)
        assert 2 <= R <= 7
        assert 0 < best <= model * 1.0001
        c = wl.small(7100 + n, solver, n, m, p, T, h=1e-3)
        u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
        plan = pb.Plan(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver, precision=precision)
        assert plan.path == pb.PATH_BLOCKED_RESPONSE
        assert plan.response_shape[0] == 1 << R
        plan.execute()
        _, y = plan.output()
        plan.close()
        assert oracle.rel_err(y, _oracle(c)) <= (1e-12 if precision == 0 else 1e-6)
    finally:
        pb.tune_clear()
