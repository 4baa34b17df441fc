"""GPU parity of the general affine scan (per-step maps, every pair composed).

ParODE_AffineScanGeneral takes a distinct map per step, x_{k+1} = M_k x_k + v_k
(a time-varying system), and composes the pairs of every up-sweep level,
matrices and vectors, as the reference's MM / MVV scan kernels do
(Kernels/MMKernelScanUpsweep.cl:13-56, Kernels/MVVKernelScanUpsweep.cl:14-50).
Checked against a sequential FP64 recurrence on random time-varying maps, and,
through SimulateODE's general path (PARODE_OPT_PATH 5: a copy of Phi per
step, the reference's pipeline), against the FP64 oracle O1 and the default
power-table path on LTI systems.

Tolerances (per-channel relative error): 1e-12 for the FP64 form, 1e-6 for
the mixed form (3xTF32 compositions on tcgen05 below the top four levels).
"""
import numpy as np
import pytest

from oracle import oracle
from parode_b200 import workloads as wl

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_MIXED = 1e-6


def _ltv(ns, count, seed, h=1e-2):
    rng = np.random.default_rng(seed)
    M = np.empty((count, ns, ns))
    for k in range(count):
        A = -np.eye(ns) + 0.5 * rng.standard_normal((ns, ns)) / np.sqrt(ns)
        M[k] = np.eye(ns) + h * A + 0.5 * (h * A) @ (h * A)
    V = h * rng.standard_normal((count, ns))
    x0 = rng.standard_normal(ns)
    X = np.empty((count, ns))
    x = x0.copy()
    for k in range(count):
        X[k] = x
        x = M[k] @ x + V[k]
    return M, V, x0, X


def _run(pb, torch, M, V, x0, precision):
    dev = torch.device("cuda", 0)
    count, ns = V.shape
    dM = torch.from_numpy(np.ascontiguousarray(M)).to(dev)
    dV = torch.from_numpy(np.ascontiguousarray(V)).to(dev)
    dx0 = torch.from_numpy(np.ascontiguousarray(x0)).to(dev)
    dX = torch.full((count, ns), float("nan"), dtype=torch.float64, device=dev)
    pb.affine_scan_general(dM.data_ptr(), dV.data_ptr(), dx0.data_ptr(), ns, count, dX.data_ptr(), precision,
                           torch.cuda.current_stream(dev).cuda_stream)
    return dX.cpu().numpy()


@pytest.mark.parametrize("ns,count", [(3, 1), (3, 2), (5, 7), (8, 1000), (13, 4097), (20, 2500), (32, 3000),
                                      (64, 1025)])
@pytest.mark.parametrize("precision", [0, 1])
def test_time_varying_maps_match_recurrence(pb, ns, count, precision):
    torch = pytest.importorskip("torch")
    M, V, x0, X = _ltv(ns, count, 1000 + ns + count)
    got = _run(pb, torch, M, V, x0, precision)
    err = oracle.rel_err(got, X)
    assert err <= (TOL_FP64 if precision == 0 else TOL_MIXED), err


def test_general_scan_rejects_bad_arguments(pb):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    M = torch.zeros((4, 65, 65), dtype=torch.float64, device=dev)
    X = torch.zeros((4, 65), dtype=torch.float64, device=dev)
    with pytest.raises(pb.ParODEError) as e:
        pb.affine_scan_general(M.data_ptr(), 0, 0, 65, 4, X.data_ptr())
    assert e.value.code == -9


def _oracle(c):
    return oracle.simulate_affine(oracle.System(c.A, c.B, c.C, c.D, c.x0),
                                  oracle.Input.sinusoid(c.u.a, c.u.f, c.u.phi), c.solver, c.t0, c.t_end, c.h)


CASES = [(0, 8, 2, 2, 4096), (0, 40, 4, 5, 3000), (1, 10, 2, 3, 2500), (1, 16, 2, 2, 2000), (0, 64, 8, 8, 5000)]


@pytest.mark.parametrize("solver,n,m,p,T", CASES)
@pytest.mark.parametrize("precision", [0, 1])
def test_general_path_matches_oracle_and_power_table(pb, solver, n, m, p, T, precision):
    c = wl.small(3300 + n + T, solver, n, m, p, T, h=1e-3)
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    pb.set_option(pb.OPT_PATH, pb.PATH_GENERAL)
    try:
        plan = pb.Plan(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver, precision=precision)
        assert plan.path == pb.PATH_GENERAL
        plan.execute()
        _, y = plan.output()
        plan.close()
    finally:
        pb.set_option(pb.OPT_PATH, 0)
    tol = TOL_FP64 if precision == 0 else TOL_MIXED
    assert oracle.rel_err(y, _oracle(c)) <= tol
    _, y_default = pb.simulate(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver)
    assert oracle.rel_err(y, y_default) <= tol
