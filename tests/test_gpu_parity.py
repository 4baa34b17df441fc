"""GPU parity of the FP64 scan against the CPU oracle (O1), through the C ABI.

Gate for the plain FP64 scan: per-channel relative error <= 1e-12
(max_k |y - y_oracle| / max_k |y_oracle|).  Float entry points (the
reference C ABI, fType = float) are held to the reference tests' own
criterion sqrt(sum err^2) < 0.1 and to a float-level relative bound.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle
from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_fixtures.json")


def _oracle_y(case, solver=None, Cm="C", D="D", B="B"):
    s = case.solver if solver is None else solver
    sysd = oracle.System(case.A, None if B is None else case.B, None if Cm is None else case.C,
                         None if D is None else case.D, case.x0)
    inp = oracle.Input.sinusoid(case.u.a, case.u.f, case.u.phi)
    return oracle.simulate_affine(sysd, inp, s, case.t0, case.t_end, case.h)


def _gpu_y(pb, case, path, precision=0, Cm="C", D="D", B="B"):
    pb.set_option(pb.OPT_PATH, path)
    u = pb.register_sinusoid(case.u.a, case.u.f, case.u.phi)
    _, y = pb.simulate(case.A, None if B is None else case.B, None if Cm is None else case.C,
                       None if D is None else case.D, case.x0, u, case.t0, case.t_end, case.h, solver=case.solver,
                       precision=precision)
    return y


# level-synchronous; blocked (scan dimension <= 64) with the leaf chosen by
# cost, with the block-response GEMM leaf, with the in-block sweep leaf
PATHS = [1, 2, 3, 4]


def _skip_unsupported(path, case):
    if path >= 2 and case.scan_dim > 64:
        pytest.skip("blocked path covers scan dimensions up to 64")


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("solver", [0, 1])
@pytest.mark.parametrize("n,m,p,T", [(1, 1, 1, 1), (1, 1, 1, 2), (2, 1, 1, 3), (3, 2, 2, 17), (5, 2, 3, 100),
                                     (8, 2, 2, 257), (13, 3, 2, 1000), (16, 4, 4, 1024), (31, 4, 3, 513),
                                     (64, 8, 8, 2048)])
def test_fp64_parity_sizes(pb, path, solver, n, m, p, T):
    if solver == 1 and T < 4:
        T = T + 4  # the ABM start-up needs three steps before the scan
    case = wl.small(1000 + 7 * n + T, solver, n, m, p, T, h=0.01)
    _skip_unsupported(path, case)
    y = _gpu_y(pb, case, path)
    yo = _oracle_y(case)
    assert y.shape == yo.shape
    assert oracle.rel_err(y, yo) <= TOL_FP64


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("solver", [0, 1])
def test_fp64_absent_matrices(pb, path, solver):
    case = wl.small(77 + solver, solver, 6, 2, 3, 200, h=0.02)
    _skip_unsupported(path, case)
    for Cm, D, B in [("C", None, "B"), (None, "D", "B"), (None, None, "B"), ("C", "D", None), (None, None, None)]:
        if path == 3 and B is None and D is None:
            continue  # the response leaf maps input samples: nothing to map without inputs
        y = _gpu_y(pb, case, path, Cm=Cm, D=D, B=B)
        yo = _oracle_y(case, Cm=Cm, D=D, B=B)
        assert y.shape == yo.shape
        assert oracle.rel_err(y, yo) <= TOL_FP64, (Cm, D, B)


@pytest.mark.parametrize("path", PATHS)
def test_cfg1_full(pb, path):
    case = wl.cfg1()
    y = _gpu_y(pb, case, path)
    yo = _oracle_y(case)
    assert y.shape == (4096, 2)
    assert oracle.rel_err(y, yo) <= TOL_FP64


@pytest.mark.parametrize("path", PATHS)
def test_cfg2_full_size(pb, path):
    """RK4, n=64, T=2^20 (the benchmark workload), full size."""
    case = wl.cfg2()
    y = _gpu_y(pb, case, path)
    yo = _oracle_y(case)
    assert oracle.rel_err(y, yo) <= TOL_FP64


def test_plan_reuse_and_launch_count(pb):
    case = wl.small(5, 0, 12, 3, 2, 3000, h=0.01)
    u = pb.register_sinusoid(case.u.a, case.u.f, case.u.phi)
    plan = pb.Plan(case.A, case.B, case.C, case.D, case.x0, u, case.t0, case.t_end, case.h, solver=0)
    plan.execute()
    _, y1 = plan.output()
    plan.execute()
    _, y2 = plan.output()
    assert np.array_equal(y1, y2)
    assert plan.launch_count > 0
    assert oracle.rel_err(y1, _oracle_y(case)) <= TOL_FP64
    plan.close()


@pytest.mark.parametrize("solver,n,m,p,T", [(1, 40, 4, 3, 2500), (0, 100, 6, 5, 3000)])
def test_large_scan_plan_runs_as_one_system_batch(pb, solver, n, m, p, T):
    """Scan dimensions above 64: the plan runs the batch engine's one-system
    form (response leaf, scan over blocks); repeated executes, a caller
    device buffer on a caller stream, and the host copy all agree."""
    import torch

    pb.set_option(pb.OPT_PATH, 0)
    case = wl.small(7100 + n, solver, n, m, p, T, h=1e-3)
    u = pb.register_sinusoid(case.u.a, case.u.f, case.u.phi)
    plan = pb.Plan(case.A, case.B, case.C, case.D, case.x0, u, case.t0, case.t_end, case.h, solver=solver)
    assert plan.path == 3 and plan.response_shape[0] > 0, (plan.path, plan.response_shape)
    plan.execute()
    _, y1 = plan.output()
    ydev = torch.zeros((plan.num_outputs, plan.channels), dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    plan.execute(ydev.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    _, y2 = plan.output()
    assert np.array_equal(y1, y2)
    assert np.array_equal(ydev.cpu().numpy(), y1)
    assert oracle.rel_err(y1, _oracle_y(case)) <= TOL_FP64
    plan.close()



@pytest.mark.parametrize("solver,n,m,p,T", [(0, 96, 4, 4, 4000), (1, 40, 3, 3, 3000)])
def test_executions_option_changes_block_length_not_result(pb, solver, n, m, p, T):
    """PARODE_OPT_EXECUTIONS: with the table build spread over many solves the
    block-response leaf takes longer blocks; FP64 and mixed results match the
    oracle either way."""
    pb.set_option(pb.OPT_PATH, 0)
    case = wl.small(7300 + n, solver, n, m, p, T, h=1e-3)
    u = pb.register_sinusoid(case.u.a, case.u.f, case.u.phi)
    ref = _oracle_y(case)
    blocks = {}
    try:
        for ex in (1, 1000):
            pb.set_option(pb.OPT_EXECUTIONS, ex)
            for prec, tol in ((pb.FP64, TOL_FP64), (pb.MIXED, 1e-6)):
                plan = pb.Plan(case.A, case.B, case.C, case.D, case.x0, u, case.t0, case.t_end, case.h,
                               solver=solver, precision=prec)
                assert plan.path == 3, plan.path
                blocks[(ex, prec)] = plan.response_shape[0]
                plan.execute()
                _, y = plan.output()
                err = oracle.rel_err(y, ref)
                assert err <= tol, (ex, prec, err)
                plan.close()
    finally:
        pb.set_option(pb.OPT_EXECUTIONS, 1)
    assert blocks[(1, pb.FP64)] < blocks[(1000, pb.FP64)], blocks


def _fx_input(kind):
    if kind == "sin_cos":
        return lambda t, i: math.sin(t) if i == 0 else (math.cos(t) if i == 1 else 0.0)
    if kind == "sin_cos_4":
        return lambda t, i: math.sin(t) if i in (0, 2) else (math.cos(t) if i in (1, 3) else 0.0)
    return lambda t, i: t if i < 2 else 0.0


def test_reference_fixtures_through_c_abi(pb):
    """The reference's own test programs, replayed through SimulateODE (float
    ABI, NVRTC-compiled UFunc): their criterion, and float-level agreement
    with the FP64 oracle fed the same float-time inputs."""
    pb.set_option(pb.OPT_PATH, 0)
    with open(GOLDEN) as fh:
        fixtures = json.load(fh)["fixtures"]
    for fx in fixtures:
        u = pb.register_input(fx["ufunc"])
        sysd = oracle.System(np.array(fx["A"]), np.array(fx["B"]), np.array(fx["C"]), np.array(fx["D"]),
                             np.array(fx["x0"]))
        inp = oracle.Input.callable(_fx_input(fx["input"]), float_time=True)
        for c in fx["cases"]:
            t, y, err = pb.simulate_f32(np.array(fx["A"]), np.array(fx["B"]), np.array(fx["C"]), np.array(fx["D"]),
                                        np.array(fx["x0"]), u, 0.0, c["t_end"], fx["h"], solver=c["solver"])
            assert err == 0
            assert y.shape[0] == c["n_out"]
            assert np.array_equal(t.astype(float), np.array(c["time"]))
            y2 = np.array(c["y_o2_f32"])
            start, stop = (1, None) if c["solver"] == 0 else (4, c["n_out"] - 1)
            assert oracle.l2_err(y, y2, start, stop) < 0.1, (fx["name"], c["solver"], c["steps"])
            yo = oracle.simulate_affine(sysd, inp, c["solver"], 0.0, c["t_end"], fx["h"])
            assert oracle.rel_err(y, yo) < 1e-5, (fx["name"], c["solver"], c["steps"])


def test_c_abi_matches_the_reference_kernels(pb):
    """The drop-in float C ABI (SimulateODE with the case's UFunc through
    RegisterInput) against the reference's own OpenCL kernels run on a B200
    (tests/golden/ref_kernel_outputs.json: the reference tests' fixtures, the
    n=8 benchmark system and its ABM twin, systems with no C and D).  The
    library computes in FP64, the kernels in FP32: the agreement is the
    reference's FP32 accuracy."""
    import base64

    pb.set_option(pb.OPT_PATH, 0)
    path = os.path.join(os.path.dirname(GOLDEN), "ref_kernel_outputs.json")
    with open(path) as fh:
        cases = json.load(fh)["cases"]
    checked = 0
    for c in cases:
        if c["max_batch"]:
            continue  # the cap on the reference's time batches has no counterpart here
        # the OpenCL extension pragma is not C++; the function body is
        src = "\n".join(ln for ln in c["ufunc"].splitlines() if not ln.startswith("#pragma OPENCL"))
        u = pb.register_input(src)
        arr = lambda k: None if c[k] is None else np.array(c[k], dtype=np.float64)
        t, y, err = pb.simulate_f32(arr("A"), arr("B"), arr("C"), arr("D"), arr("x0"), u, c["t0"], c["t_end"], c["h"],
                                    solver=c["solver"])
        assert err == 0, c["name"]
        yk = np.frombuffer(base64.b64decode(c["y_f32"]), dtype=np.float32).reshape(c["T"], c["q"])
        tk = np.frombuffer(base64.b64decode(c["time_f32"]), dtype=np.float32)
        assert y.shape == yk.shape, c["name"]
        assert np.array_equal(t, tk), c["name"]
        e = oracle.rel_err(y.astype(np.float64), yk.astype(np.float64))
        assert e <= 5e-5, (c["name"], e)
        checked += 1
    assert checked >= 15


def test_python_module_reference_script(pb):
    """PythonInterface/TestPythonODESolvers.py of the reference, in Python 3."""
    import ParODE

    gpus, err = ParODE.GetAvailableGPUs()
    assert err == 0 and len(gpus) >= 1
    name, err = ParODE.GetDeviceName(gpus[0])
    assert err == 0 and "B200" in name
    assert ParODE.InitializeSelectedGPUs(gpus) == 0
    A = [[-2.0, 1.0], [0.5, -3.0]]
    I = [[1.0, 0.0], [0.0, 1.0]]
    src = ("fType UFunc(fType t, int nInputIndex){\nfType fVal = nInputIndex == 0 ? t :\nnInputIndex == 1 ? t :\n"
           "0.0;\nreturn fVal;\n}\n")
    uIndex, err = ParODE.RegisterInput(src)
    assert err == 0 and uIndex >= 0
    assert ParODE.StartTimer() == 0
    tv, xv, err = ParODE.SimulateODE(A, I, I, I, uIndex, 0.0, 0.1, 50, [-1.0, 1.0], 1)
    ms, err2 = ParODE.StopTimer()
    assert err == 0 and err2 == 0 and ms >= 0.0
    assert len(tv) == 50 and len(xv) == 50 and len(xv[0]) == 2
    sysd = oracle.System(np.array(A), np.eye(2), np.eye(2), np.eye(2), np.array([-1.0, 1.0]))
    inp = oracle.Input.callable(lambda t, i: t, float_time=True)
    y2 = oracle.stepper(sysd, inp, 1, 0.0, 0.1, 50, use_float=True)
    assert oracle.l2_err(np.array(xv), y2, 4, 49) < 0.1
    ParODE.CloseGPU()
    pb.init()


def test_error_codes(pb):
    case = wl.small(3, 0, 4, 2, 2, 20)
    with pytest.raises(pb.ParODEError) as ei:
        pb.simulate(case.A, case.B, case.C, case.D, case.x0, 9999, 0.0, case.t_end, case.h)
    assert ei.value.code == -8
    u = pb.register_sinusoid(case.u.a, case.u.f, case.u.phi)
    with pytest.raises(pb.ParODEError) as ei:
        pb.simulate(case.A, case.B, case.C, case.D, case.x0, u, 0.0, case.t_end, case.h, solver=5)
    assert ei.value.code == -7
    with pytest.raises(pb.ParODEError) as ei:
        pb.simulate(case.A, case.B, case.C, case.D, case.x0, u, 0.0, -1.0, case.h)
    assert ei.value.code == -6
    with pytest.raises(pb.ParODEError) as ei:
        pb.register_input("this is not C++")
    assert ei.value.code == -3
    # no input needed when B and D are absent
    _, y = pb.simulate(case.A, None, case.C, None, case.x0, 9999, 0.0, case.t_end, case.h)
    assert y.shape == (case.T, case.p)
