"""ParODE_AffineScanDevice: the allocation-free affine scan over device buffers.

Compared with the existing entry point ParODE_SimulateODE_d (no B, C, D: the
outputs are the states, x_k = Phi^k x0) and with a sequential FP64 recurrence
on random forcing, on two calls in a row each.  The file name sorts last so
that the test also runs after every other GPU test in one session.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64 scan vs FP64 references, per-channel relative error


def _entry(pb):
    f = pb.lib.ParODE_AffineScanDevice
    f.restype = None
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p,
                  C.POINTER(C.c_int)]
    return f


def _scan(pb, torch, phi, gamma, x0, count):
    """Runs the entry point on device copies; returns (status, X on the host)."""
    ns = phi.shape[0]
    dev = torch.device("cuda", 0)
    d_phi = torch.from_numpy(np.ascontiguousarray(phi)).to(dev)
    d_gamma = None if gamma is None else torch.from_numpy(np.ascontiguousarray(gamma)).to(dev)
    d_x0 = torch.from_numpy(np.ascontiguousarray(x0)).to(dev)
    d_x = torch.full((count, ns), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    err = C.c_int(1)
    _entry(pb)(d_phi.data_ptr(), None if d_gamma is None else d_gamma.data_ptr(), d_x0.data_ptr(), ns, count,
               d_x.data_ptr(), stream.cuda_stream, C.byref(err))
    torch.cuda.synchronize()
    return err.value, d_x.cpu().numpy()


def _system(n, seed):
    rng = np.random.default_rng(seed)
    A = -2.0 * np.eye(n) + 0.5 * rng.standard_normal((n, n)) / np.sqrt(n)
    x0 = rng.standard_normal(n)
    return A, x0, rng


@pytest.mark.parametrize("n,T", [(8, 4096), (64, 20000)])
def test_homogeneous_matches_simulate(pb, n, T):
    torch = pytest.importorskip("torch")
    A, x0, _ = _system(n, 11 + n)
    h = 1e-3
    _, y = pb.simulate(A, None, None, None, x0, 0, 0.0, (T - 0.5) * h, h, solver=pb.RK4, precision=pb.FP64)
    assert y.shape == (T, n)
    phi, _ = oracle.discretise(oracle.RK4, A, None, h)
    first = None
    for _ in range(2):
        err, X = _scan(pb, torch, phi, None, x0, T)
        assert err == 0
        assert oracle.rel_err(X, y) <= TOL
        if first is None:
            first = X
        else:
            assert np.array_equal(first, X)


@pytest.mark.parametrize("n,T", [(5, 3000), (64, 20000)])
def test_forced_matches_recurrence(pb, n, T):
    torch = pytest.importorskip("torch")
    A, x0, rng = _system(n, 23 + n)
    phi, _ = oracle.discretise(oracle.RK4, A, None, 1e-3)
    gamma = 1e-2 * rng.standard_normal((T, n))
    ref = np.empty((T, n))
    x = x0.copy()
    for k in range(T):
        ref[k] = x
        x = phi @ x + gamma[k]
    for _ in range(2):
        err, X = _scan(pb, torch, phi, gamma, x0, T)
        assert err == 0
        assert oracle.rel_err(X, ref) <= TOL


def test_no_initial_state_starts_from_zero(pb):
    """dX0 = NULL: the recurrence starts from x_0 = 0."""
    torch = pytest.importorskip("torch")
    n, T = 16, 5000
    A, _, rng = _system(n, 41)
    phi, _ = oracle.discretise(oracle.RK4, A, None, 1e-3)
    gamma = rng.standard_normal((T, n))
    ref = np.empty((T, n))
    x = np.zeros(n)
    for k in range(T):
        ref[k] = x
        x = phi @ x + gamma[k]
    dev = torch.device("cuda", 0)
    d_phi = torch.from_numpy(phi).to(dev)
    d_gamma = torch.from_numpy(gamma).to(dev)
    d_x = torch.full((T, n), float("nan"), dtype=torch.float64, device=dev)
    err = C.c_int(1)
    _entry(pb)(d_phi.data_ptr(), d_gamma.data_ptr(), None, n, T, d_x.data_ptr(),
               torch.cuda.current_stream(dev).cuda_stream, C.byref(err))
    torch.cuda.synchronize()
    assert err.value == 0
    assert oracle.rel_err(d_x.cpu().numpy(), ref) <= TOL


def test_calls_map_no_device_memory(pb):
    """After the first call, further calls leave the device's free memory unchanged."""
    torch = pytest.importorskip("torch")
    n, T = 64, 20000
    A, x0, rng = _system(n, 53)
    phi, _ = oracle.discretise(oracle.RK4, A, None, 1e-3)
    gamma = 1e-2 * rng.standard_normal((T, n))
    dev = torch.device("cuda", 0)
    d_phi = torch.from_numpy(phi).to(dev)
    d_gamma = torch.from_numpy(gamma).to(dev)
    d_x0 = torch.from_numpy(x0).to(dev)
    d_x = torch.empty((T, n), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    err = C.c_int(1)
    f = _entry(pb)
    f(d_phi.data_ptr(), d_gamma.data_ptr(), d_x0.data_ptr(), n, T, d_x.data_ptr(), stream, C.byref(err))
    torch.cuda.synchronize()
    assert err.value == 0
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(3):
        f(d_phi.data_ptr(), d_gamma.data_ptr(), d_x0.data_ptr(), n, T, d_x.data_ptr(), stream, C.byref(err))
        assert err.value == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0


def test_rejects_beyond_scratch_and_bad_dimension(pb):
    torch = pytest.importorskip("torch")
    phi = np.eye(64) * 0.5
    err, _ = _scan(pb, torch, phi, None, np.ones(64), 200000)
    assert err == -4  # NotEnoughResources: more than the static scratch
    err, _ = _scan(pb, torch, np.eye(65), None, np.ones(65), 16)
    assert err == -9  # InvalidArgument: ns above 64
