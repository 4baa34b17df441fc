"""CPU tests of the oracle: pinned against the reference tests' own fixtures
and criterion, and against independent restatements of the same maths."""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle
from parode_b200 import workloads as wl

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_fixtures.json")


@pytest.fixture(scope="module")
def fixtures():
    with open(GOLDEN) as fh:
        return json.load(fh)["fixtures"]


def _fx_system(fx):
    return oracle.System(np.array(fx["A"]), np.array(fx["B"]), np.array(fx["C"]), np.array(fx["D"]), np.array(fx["x0"]))


def _fx_input(kind):
    if kind == "sin_cos":
        return lambda t, i: math.sin(t) if i == 0 else (math.cos(t) if i == 1 else 0.0)
    if kind == "sin_cos_4":
        return lambda t, i: math.sin(t) if i in (0, 2) else (math.cos(t) if i in (1, 3) else 0.0)
    return lambda t, i: t if i < 2 else 0.0


def test_reference_criterion_o1_vs_o2(fixtures):
    """O1 (FP64 affine recurrence) passes every reference test's own criterion
    sqrt(sum err^2) < 0.1 against the reference test loops (O2, float)."""
    for fx in fixtures:
        sysd = _fx_system(fx)
        inp = oracle.Input.callable(_fx_input(fx["input"]), float_time=True)
        for c in fx["cases"]:
            y1 = oracle.simulate_affine(sysd, inp, c["solver"], 0.0, c["t_end"], fx["h"])
            y2 = np.array(c["y_o2_f32"])
            start, stop = (1, None) if c["solver"] == 0 else (4, c["n_out"] - 1)
            assert y1.shape == y2.shape
            assert oracle.l2_err(y1, y2, start, stop) < 0.1, (fx["name"], c["solver"], c["steps"])
            # and it reproduces the committed O1 vectors bit for bit
            assert np.array_equal(y1, np.array(c["y_o1"])), (fx["name"], c["solver"], c["steps"])


def test_reference_stepper_golden(fixtures):
    """O2 reproduces the committed golden outputs of the reference test loops."""
    for fx in fixtures:
        sysd = _fx_system(fx)
        inp = oracle.Input.callable(_fx_input(fx["input"]), float_time=True)
        for c in fx["cases"]:
            y2 = oracle.stepper(sysd, inp, c["solver"], 0.0, fx["h"], c["n_out"], use_float=True)
            assert np.array_equal(y2, np.array(c["y_o2_f32"]))


def test_step_counts_and_time_vector(fixtures):
    # the float accumulation and the truncating count rule of the reference
    for fx in fixtures:
        for c in fx["cases"]:
            nt, ns = oracle.num_outputs(c["solver"], 0.0, c["t_end"], fx["h"])
            assert nt == c["n_out"]
            assert ns == (nt if c["solver"] == 0 else nt - 3)
            tv = oracle.time_vector(c["solver"], 0.0, c["t_end"], fx["h"])
            assert np.array_equal(tv.astype(float), np.array(c["time"]))
    # (tEnd - t0)/h = 95.999... truncates: ABM with 100 requested steps yields 99
    assert oracle.num_outputs(1, 0.0, 99 * 0.1, 0.1)[0] == 99
    assert oracle.num_outputs(0, 0.0, 99 * 0.1, 0.1)[0] == 100
    assert oracle.num_outputs(0, 1.0, 0.5, 0.1)[0] == -1


def test_rk4_discretisation_is_rk4_step():
    """Phi, Bbar reproduce one classical RK4 step exactly (up to rounding)."""
    case = wl.small(11, 0, 6, 3, 2, 10, h=0.05)
    Phi, Bbar = oracle.discretise(0, case.A, case.B, case.h)
    x = case.x0.copy()
    u = [np.array([case.u(0.0 + q * case.h / 2, i) for i in range(case.m)]) for q in range(3)]
    f = lambda x, u: case.A @ x + case.B @ u
    h = case.h
    k1 = f(x, u[0]); k2 = f(x + h / 2 * k1, u[1]); k3 = f(x + h / 2 * k2, u[1]); k4 = f(x + h * k3, u[2])
    ref = x + h / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
    got = Phi @ x + Bbar @ np.concatenate(u)
    assert np.allclose(got, ref, rtol=1e-13, atol=1e-13)


def test_abm_discretisation_is_pece():
    """The companion map reproduces the AB4/AM4 PECE step."""
    case = wl.small(12, 1, 5, 2, 2, 10, h=0.02)
    Phi, Bbar = oracle.discretise(1, case.A, case.B, case.h)
    n, h = case.n, case.h
    xs = [np.random.default_rng(q).standard_normal(n) for q in range(4)]
    us = [np.random.default_rng(10 + q).standard_normal(case.m) for q in range(5)]
    f = lambda x, u: case.A @ x + case.B @ u
    fs = [f(xs[q], us[q]) for q in range(4)]
    pred = xs[3] + h / 24 * (55 * fs[3] - 59 * fs[2] + 37 * fs[1] - 9 * fs[0])
    corr = xs[3] + h / 24 * (9 * f(pred, us[4]) + 19 * fs[3] - 5 * fs[2] + fs[1])
    X = np.concatenate(xs)
    Xn = Phi @ X
    Xn[3 * n:] += Bbar @ np.concatenate(us)
    assert np.allclose(Xn[3 * n:], corr, rtol=1e-12, atol=1e-12)
    assert np.array_equal(Xn[:3 * n], X[n:])


@pytest.mark.parametrize("solver", [0, 1])
def test_o1_matches_fp64_stepper(solver):
    """O1 and the FP64 restatement of the reference test loops agree to
    rounding (they are the same maths evaluated in different orders)."""
    case = wl.small(21 + solver, solver, 7, 3, 4, 300, h=0.01)
    sysd = oracle.System(case.A, case.B, case.C, case.D, case.x0)
    inp = oracle.Input.sinusoid(case.u.a, case.u.f, case.u.phi)
    y1 = oracle.simulate_affine(sysd, inp, solver, 0.0, case.t_end, case.h)
    y2 = oracle.stepper(sysd, inp, solver, 0.0, case.h, y1.shape[0], use_float=False)
    assert oracle.rel_err(y2, y1) < 1e-12


@pytest.mark.parametrize("solver", [0, 1])
@pytest.mark.parametrize("batch", [0, 64])
def test_o3_reference_pipeline_float(solver, batch):
    """O3 (the reference's FP32 Blelloch pipeline with host carry between
    power-of-two batches) stays within FP32 accuracy of O1."""
    case = wl.small(31 + solver, solver, 6, 2, 3, 700, h=0.01)
    sysd = oracle.System(case.A, case.B, case.C, case.D, case.x0)
    inp = oracle.Input.sinusoid(case.u.a, case.u.f, case.u.phi)
    y1 = oracle.simulate_affine(sysd, inp, solver, 0.0, case.t_end, case.h)
    y3 = oracle.refscan_f32(sysd, inp, solver, 0.0, case.t_end, case.h, batch=batch)
    assert y3.shape == y1.shape
    assert oracle.rel_err(y3, y1) < 1e-4


def test_output_selection_and_absent_matrices():
    case = wl.small(41, 0, 4, 2, 3, 50)
    inp = oracle.Input.sinusoid(case.u.a, case.u.f, case.u.phi)
    both = oracle.simulate_affine(oracle.System(case.A, case.B, case.C, case.D, case.x0), inp, 0, 0.0, case.t_end, case.h)
    conly = oracle.simulate_affine(oracle.System(case.A, case.B, case.C, None, case.x0), inp, 0, 0.0, case.t_end, case.h)
    donly = oracle.simulate_affine(oracle.System(case.A, case.B, None, case.D, case.x0), inp, 0, 0.0, case.t_end, case.h)
    xonly = oracle.simulate_affine(oracle.System(case.A, case.B, None, None, case.x0), inp, 0, 0.0, case.t_end, case.h)
    assert xonly.shape[1] == case.n
    assert np.allclose(conly + donly, both, rtol=1e-12, atol=1e-12)
    assert np.allclose(conly, xonly @ case.C.T, rtol=1e-12, atol=1e-12)


def test_rel_err_definition():
    yref = np.array([[1.0, 0.0], [2.0, 0.0], [-4.0, 0.0]])
    y = yref + np.array([[0.0, 0.0], [0.4, 0.0], [0.0, 3e-3]])
    # channel 0: 0.4/4; channel 1 has no signal: absolute error
    assert oracle.rel_err(y, yref) == pytest.approx(0.1)
