"""GPU parity of the batched form (ParODE_Batch*) against the CPU FP64 oracle.

Every system of a batch must match its own sequential FP64 recurrence (O1)
to the plain-scan gate, 1e-12 per-channel relative error, whatever the mix of
scan dimensions (blocked buckets NP = 8..64 and level-synchronous systems),
integrators, horizons and absent matrices in the batch.
"""
import numpy as np
import pytest

from oracle import oracle
from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def _oracle_y(case, B=True, Cm=True, D=True):
    sysd = oracle.System(case.A, case.B if B else None, case.C if Cm else None, case.D if D else None, case.x0)
    inp = oracle.Input.sinusoid(case.u.a, case.u.f, case.u.phi)
    return oracle.simulate_affine(sysd, inp, case.solver, case.t0, case.t_end, case.h)


def _spec(pb, case, B=True, Cm=True, D=True):
    u = pb.register_sinusoid(case.u.a, case.u.f, case.u.phi)
    return {"A": case.A, "B": case.B if B else None, "C": case.C if Cm else None, "D": case.D if D else None,
            "x0": case.x0, "u": u, "t0": case.t0, "t_end": case.t_end, "h": case.h, "solver": case.solver}


MIX = [  # (solver, n, m, p, T, B, C, D)
    (0, 3, 1, 2, 700, True, True, True),      # NP 8
    (0, 13, 2, 2, 2500, True, True, True),    # NP 16
    (0, 40, 4, 5, 3000, True, True, True),    # NP 64
    (1, 2, 1, 1, 900, True, True, True),      # ABM, N_s 8
    (1, 10, 2, 3, 1500, True, True, True),    # ABM, N_s 40
    (1, 20, 3, 2, 1200, True, True, True),    # ABM, N_s 80: level-synchronous
    (0, 70, 5, 4, 1000, True, True, True),    # RK4 n 70: level-synchronous
    (0, 6, 2, 2, 333, False, True, True),     # no B
    (0, 9, 2, 2, 444, True, False, False),    # y = x
    (1, 5, 2, 2, 555, True, False, True),     # ABM, no C
    (0, 1, 1, 1, 1, True, True, True),        # one step
    (1, 1, 1, 1, 4, True, True, True),        # ABM, one scan step
    (0, 33, 3, 3, 4097, True, True, True),    # NP 64, ragged tiles
    (1, 30, 2, 2, 2049, True, True, False),   # ABM N_s 120, level-synchronous
]


def _mix_cases():
    out = []
    for k, (solver, n, m, p, T, B, Cm, D) in enumerate(MIX):
        case = wl.small(7000 + 13 * k, solver, n, m, p, T, h=1e-3)
        out.append((case, B, Cm, D))
    return out


@pytest.mark.parametrize("path", [0, 1, 3])
def test_batch_mixed_sizes_match_oracle(pb, path):
    pb.set_option(pb.OPT_PATH, path)
    cases = _mix_cases()
    batch = pb.Batch([_spec(pb, c, B, Cm, D) for c, B, Cm, D in cases], precision=pb.FP64)
    batch.execute()
    for i, (c, B, Cm, D) in enumerate(cases):
        _, y = batch.output(i)
        ref = _oracle_y(c, B, Cm, D)
        assert y.shape == ref.shape, (i, y.shape, ref.shape)
        err = oracle.rel_err(y, ref)
        assert err <= TOL_FP64, (i, MIX[i], err)
    # paths: 1 level-synchronous (forced), 3 block response (forced: every
    # system here has inputs); automatic: scan dimension <= 64 blocked or
    # block response, larger level-synchronous or block response
    paths = [batch.path(i) for i in range(len(cases))]
    for i, (c, *_rest) in enumerate(cases):
        if path in (1, 3):
            assert paths[i] == path, (i, paths[i])
        else:
            assert paths[i] in ((2, 3) if c.scan_dim <= 64 else (1, 3)), (i, paths[i])
    pb.set_option(pb.OPT_PATH, 0)
    batch.close()


def test_batch_repeat_and_launch_count(pb):
    pb.set_option(pb.OPT_PATH, 0)
    cases = _mix_cases()
    batch = pb.Batch([_spec(pb, c, B, Cm, D) for c, B, Cm, D in cases], precision=pb.FP64)
    batch.execute()
    first = [batch.output(i)[1].copy() for i in range(len(cases))]
    batch.execute()
    for i in range(len(cases)):
        assert np.array_equal(first[i], batch.output(i)[1])
    # a fixed number of launches, independent of the number of systems
    assert batch.launch_count < 120, batch.launch_count
    batch.close()


def test_batch_equals_single_solves(pb):
    pb.set_option(pb.OPT_PATH, 0)
    cases = _mix_cases()[:6]
    batch = pb.Batch([_spec(pb, c) for c, *_ in cases], precision=pb.FP64)
    batch.execute()
    for i, (c, *_r) in enumerate(cases):
        u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
        _, ys = pb.simulate(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver)
        _, yb = batch.output(i)
        assert oracle.rel_err(yb, ys) <= TOL_FP64
    batch.close()


def test_batch_cfg4_subset(pb):
    """The first 48 systems of the 4096-system batched workload, FP64."""
    pb.set_option(pb.OPT_PATH, 0)
    cases = wl.cfg4()[:48]
    batch = pb.Batch([_spec(pb, c) for c in cases], precision=pb.FP64)
    batch.execute()
    worst = 0.0
    for i, c in enumerate(cases):
        _, y = batch.output(i)
        worst = max(worst, oracle.rel_err(y, _oracle_y(c)))
    assert worst <= TOL_FP64, worst
    batch.close()


TOL_MIXED = 1e-6

MIXED_LS = [  # level-synchronous systems (scan dimension > 64): tensor-core levels below the top four
    (0, 72, 6, 4, 5000), (0, 96, 8, 8, 20000), (1, 20, 3, 3, 3000), (1, 33, 4, 4, 9000), (1, 96, 12, 12, 4000),
    (0, 130, 8, 6, 1500), (1, 64, 8, 8, 2500),
]


@pytest.mark.parametrize("path", [1, 3])
def test_batch_mixed_level_synchronous(pb, path):
    """Mixed form: the level-synchronous scan over steps (path 1) or over the
    blocks of the response leaf (path 3), lower levels on the tensor cores."""
    pb.set_option(pb.OPT_PATH, path)
    cases = [wl.small(9100 + 7 * k, s, n, m, p, T, h=1e-3) for k, (s, n, m, p, T) in enumerate(MIXED_LS)]
    batch = pb.Batch([_spec(pb, c) for c in cases], precision=pb.MIXED)
    batch.execute()
    pb.set_option(pb.OPT_PATH, 0)
    for i, c in enumerate(cases):
        assert batch.path(i) == path and batch.precision(i) == pb.MIXED, i
        _, y = batch.output(i)
        err = oracle.rel_err(y, _oracle_y(c))
        assert err <= TOL_MIXED, (i, MIXED_LS[i], err)
    batch.close()


RESPONSE = [  # (solver, n, m, p, T, B, C, D): block-response systems, FP64
    (1, 128, 16, 16, 3000, True, True, True),   # ABM N_s 512 (the n=128 workload's shape)
    (0, 200, 12, 9, 2100, True, True, True),    # RK4 N_s 200
    (1, 24, 3, 5, 777, False, True, True),      # no B: D only
    (0, 17, 1, 1, 65, True, False, False),      # y = x, T below two blocks
    (1, 7, 2, 3, 4, True, True, True),          # ABM, one scan step
    (0, 64, 8, 8, 5000, True, True, True),      # the n=64 RK4 workload's shape
]


def test_batch_response_leaf_matches_oracle(pb):
    pb.set_option(pb.OPT_PATH, 3)
    cases = [(wl.small(9300 + 11 * k, s, n, m, p, T, h=1e-3), B, Cm, D)
             for k, (s, n, m, p, T, B, Cm, D) in enumerate(RESPONSE)]
    batch = pb.Batch([_spec(pb, c, B, Cm, D) for c, B, Cm, D in cases], precision=pb.FP64)
    batch.execute()
    batch.execute()  # repeat: the block scan's padding is rewritten every execute
    pb.set_option(pb.OPT_PATH, 0)
    for i, (c, B, Cm, D) in enumerate(cases):
        assert batch.path(i) == 3, i
        _, y = batch.output(i)
        err = oracle.rel_err(y, _oracle_y(c, B, Cm, D))
        assert err <= TOL_FP64, (i, RESPONSE[i], err)
    batch.close()


def test_batch_rejects_bad_system(pb):
    c = wl.small(1, 0, 4, 1, 1, 10)
    bad = _spec(pb, c)
    bad["solver"] = 7
    with pytest.raises(pb.ParODEError):
        pb.Batch([_spec(pb, c), bad])


def test_pool_keep_reuses_memory_bit_for_bit(pb):
    """With the stream-ordered pool keeping freed memory, a batch set up again
    on the memory of the first gives the same outputs bit for bit."""
    cases = _mix_cases()
    specs = [_spec(pb, c, B, Cm, D) for c, B, Cm, D in cases]
    pb.set_option(pb.OPT_POOL_KEEP, 1 << 30)
    try:
        assert pb.get_option(pb.OPT_POOL_KEEP) == 1 << 30
        outs = []
        for _ in range(2):
            b = pb.Batch(specs, precision=pb.MIXED)
            b.execute()
            outs.append([b.output(i)[1] for i in range(len(cases))])
            b.close()
    finally:
        pb.set_option(pb.OPT_POOL_KEEP, 0)
    for i in range(len(cases)):
        assert np.array_equal(outs[0][i], outs[1][i]), i


@pytest.mark.parametrize("precision", [0, 1])
def test_host_and_device_discretisation_agree_bit_for_bit(pb, precision):
    """The batch's discretisation on the host threads and on the device take
    every operation in the same order: Phi, Bbar, their distance to the exact
    part (which sizes the mixed form's levels) and so every output agree bit
    for bit, over RK4 and ABM, blocked, response and level-synchronous
    systems and absent matrices."""
    cases = _mix_cases()
    specs = [_spec(pb, c, B, Cm, D) for c, B, Cm, D in cases]
    outs = {}
    try:
        for where in (pb.DISCRETISE_HOST, pb.DISCRETISE_DEVICE):
            pb.set_option(pb.OPT_DISCRETISE, where)
            b = pb.Batch(specs, precision=precision)
            b.execute()
            outs[where] = [b.output(i)[1] for i in range(len(cases))]
            b.close()
    finally:
        pb.set_option(pb.OPT_DISCRETISE, pb.DISCRETISE_AUTO)
    for i in range(len(cases)):
        assert np.array_equal(outs[pb.DISCRETISE_HOST][i], outs[pb.DISCRETISE_DEVICE][i]), i
