"""parode_b200 -- Python host API over libParODEShared.so (B200 build of ParODE).

The drop-in surface is the C ABI (include/ParODECInterface.h) and the
`ParODE` extension module built next to this file; this package is a thin
ctypes layer for Python callers, tests and benchmarks:

    import parode_b200 as pb
    pb.init()                                  # InitializeAllGPUs
    u = pb.register_sinusoid(a, f, phi)        # or pb.register_input(src)
    t, y = pb.simulate(A, B, C, D, x0, u, t0, t_end, h, solver=pb.RK4)

Every call goes to the CUDA library.  There is no CPU fallback: the first
call that needs libParODEShared.so loads it and fails (ImportError) if it is
missing, and solves report ParODE error codes as exceptions.  Importing the
package alone maps no library, so `parode_b200.workloads` (the seeded
generators) serves processes that never touch the GPU.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libParODEShared.so")

RK4 = 0
ABM = 1
FP64 = 0
MIXED = 1
TF32 = 2   # single-pass TF32 response GEMMs (single solves; a batch or server runs MIXED)

OPT_PRECISION = 1
OPT_PATH = 2
OPT_LOG = 3
OPT_EXECUTIONS = 4
OPT_FAULT_ALLOC = 5      # test hook: the k-th device allocation from now fails (-1: off)
OPT_FAULT_WITHHOLD = 6   # test hook: the mixed response kernel withholds one arrive (bounded waits give up)
OPT_POOL_KEEP = 7        # bytes of freed device memory the stream-ordered pool keeps mapped for later plans
OPT_DISCRETISE = 8       # where batches discretise: DISCRETISE_AUTO (by cost), _HOST or _DEVICE (same bits)
DISCRETISE_AUTO = 0
DISCRETISE_HOST = 1
DISCRETISE_DEVICE = 2

PATH_AUTO = 0
PATH_LEVEL = 1
PATH_BLOCKED = 2
PATH_BLOCKED_RESPONSE = 3
PATH_BLOCKED_SWEEP = 4
PATH_GENERAL = 5

ERRORS = {
    0: "OK", -1: "NoGPU", -2: "NotInitialized", -3: "CouldNotCreateGPUKernels", -4: "NotEnoughResources",
    -5: "InvalidDeviceId", -6: "InvalidSystem", -7: "InvalidSolverType", -8: "InvalidInput",
    -9: "InvalidArgument", -10: "DeviceError",
}


class ParODEError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = int(code)
        super().__init__(f"{where}: ParODE error {code} ({ERRORS.get(int(code), '?')})")


def build() -> None:
    """Compile libParODEShared.so and the ParODE module (nvcc, sm_100a)."""
    subprocess.run(["make", "-s", "-C", _HERE, "-j8"], check=True)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run parode_b200.build() (make -C parode_b200)")
    L = C.CDLL(LIB_PATH)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    L.GetErrorDescription.argtypes = [ip, C.c_char_p]
    L.InitializeAllGPUs.argtypes = [C.c_char_p, C.c_char_p, ip]
    L.GetAvailableGPUs.argtypes = [ip, ip, ip]
    L.GetDeviceName.argtypes = [ip, C.c_char_p, ip]
    L.InitializeSelectedGPUs.argtypes = [ip, ip, C.c_char_p, C.c_char_p, ip]
    fp = C.POINTER(C.c_float)
    L.SimulateODE.argtypes = [fp, fp, fp, fp, ip, ip, ip, ip, ip, ip, ip, dp, dp, dp, fp, ip, fp, fp, ip, ip]
    L.RegisterInput.argtypes = [C.c_char_p, ip, ip]
    L.CloseGPUC.argtypes = []
    L.StartTimer.argtypes = [ip]
    L.StopTimer.argtypes = [fp, ip]
    L.ParODE_SetOption.argtypes = [C.c_int, C.c_longlong, ip]
    L.ParODE_GetOption.argtypes = [C.c_int, ip]
    L.ParODE_GetOption.restype = C.c_longlong
    L.ParODE_NumOutputs.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double]
    L.ParODE_NumOutputs.restype = C.c_longlong
    L.ParODE_RegisterSinusoidInput.argtypes = [C.c_int, C.c_int, dp, dp, dp, ip, ip]
    L.ParODE_SimulateODE_d.argtypes = [dp, dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.c_double, C.c_double, C.c_double, dp, C.c_int, C.c_int, dp, dp,
                                       C.POINTER(C.c_longlong), ip]
    L.ParODE_PlanCreate.argtypes = [dp, dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_double, C.c_double, C.c_double, dp, C.c_int, C.c_int, ip]
    L.ParODE_PlanCreate.restype = C.c_void_p
    L.ParODE_PlanExecute.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, ip]
    L.ParODE_PlanGetOutput.argtypes = [C.c_void_p, dp, dp, ip]
    L.ParODE_PlanNumOutputs.argtypes = [C.c_void_p]
    L.ParODE_PlanNumOutputs.restype = C.c_longlong
    L.ParODE_PlanNumOutputChannels.argtypes = [C.c_void_p]
    L.ParODE_PlanLaunchCount.argtypes = [C.c_void_p]
    L.ParODE_PlanDestroy.argtypes = [C.c_void_p]
    L.ParODE_PlanPrecision.argtypes = [C.c_void_p]
    L.ParODE_PlanPath.argtypes = [C.c_void_p]
    L.ParODE_PlanResponseShape.argtypes = [C.c_void_p, C.POINTER(C.c_longlong)]
    L.ParODE_PlanResponseShape.restype = None
    L.ParODE_PlanSetProfiling.argtypes = [C.c_void_p, C.c_int, ip]
    L.ParODE_PlanStageTimes.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_int, C.c_char_p, C.c_int, ip]
    L.ParODE_PlanStageTimes.restype = C.c_int
    L.ParODE_PlanCreateShard.argtypes = [dp, dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_int, C.c_double, C.c_double, C.c_double, dp, C.c_int, C.c_int,
                                         C.c_int, C.c_int, ip]
    L.ParODE_PlanCreateShard.restype = C.c_void_p
    L.ParODE_PlanShardInfo.argtypes = [C.c_void_p, C.POINTER(C.c_longlong)]
    L.ParODE_PlanShardInfo.restype = None
    L.ParODE_PlanShardUp.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, ip]
    L.ParODE_PlanShardDown.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, ip]
    pp = C.POINTER(C.c_void_p)
    L.ParODE_BatchCreate.argtypes = [C.c_int, pp, pp, pp, pp, ip, ip, ip, ip, ip, ip, ip, dp, dp, dp, pp, ip,
                                     C.c_int, ip]
    L.ParODE_BatchCreate.restype = C.c_void_p
    L.ParODE_BatchExecute.argtypes = [C.c_void_p, C.c_void_p, ip]
    L.ParODE_BatchNumOutputs.argtypes = [C.c_void_p, C.c_int]
    L.ParODE_BatchNumOutputs.restype = C.c_longlong
    L.ParODE_BatchNumOutputChannels.argtypes = [C.c_void_p, C.c_int]
    L.ParODE_BatchDeviceOutput.argtypes = [C.c_void_p, C.c_int]
    L.ParODE_BatchDeviceOutput.restype = C.c_void_p
    L.ParODE_BatchGetOutput.argtypes = [C.c_void_p, C.c_int, dp, dp, ip]
    L.ParODE_BatchLaunchCount.argtypes = [C.c_void_p]
    L.ParODE_BatchPath.argtypes = [C.c_void_p, C.c_int]
    L.ParODE_BatchPrecision.argtypes = [C.c_void_p, C.c_int]
    L.ParODE_BatchStateSteps.argtypes = [C.c_void_p]
    L.ParODE_BatchStateSteps.restype = C.c_double
    L.ParODE_BatchDestroy.argtypes = [C.c_void_p]
    L.ParODE_ServerCreate.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, ip]
    L.ParODE_ServerCreate.restype = C.c_void_p
    L.ParODE_ServerSubmit.argtypes = [C.c_void_p, dp, dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, dp, C.c_int, ip]
    L.ParODE_ServerSubmit.restype = C.c_longlong
    L.ParODE_ServerPoll.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(C.c_longlong), ip, ip]
    L.ParODE_ServerPoll.restype = C.c_int
    L.ParODE_ServerResult.argtypes = [C.c_void_p, C.c_longlong, dp, dp, dp, ip]
    L.ParODE_ServerStats.argtypes = [C.c_void_p, dp, ip]
    L.ParODE_ServerDestroy.argtypes = [C.c_void_p]
    L.ParODE_AffineScanDevice.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_void_p,
                                          C.c_void_p, ip]
    L.ParODE_AffineScanDevice.restype = None
    L.ParODE_AffineScanGeneral.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_int,
                                           C.c_void_p, C.c_void_p, ip]
    L.ParODE_AffineScanGeneral.restype = None
    fp = C.POINTER(C.c_float)
    L.ParODE_TuneResponseBlock.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_longlong, C.c_int, ip, fp, fp, ip]
    L.ParODE_TuneResponseBlock.restype = None
    L.ParODE_TuneSave.argtypes = [C.c_char_p, C.c_char_p, ip]
    L.ParODE_TuneSave.restype = C.c_int
    L.ParODE_TuneLoad.argtypes = [C.c_char_p, C.c_char_p, ip]
    L.ParODE_TuneLoad.restype = C.c_int
    L.ParODE_TuneClear.argtypes = []
    L.ParODE_TuneClear.restype = None
    return L


class _Library:
    """libParODEShared.so, loaded with its ctypes signatures on first use."""

    _handle = None

    def __getattr__(self, name):
        if _Library._handle is None:
            _Library._handle = _load()
        return getattr(_Library._handle, name)


lib = _Library()


def _dp(a: Optional[np.ndarray]):
    return C.POINTER(C.c_double)() if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _check(err: C.c_int, where: str) -> None:
    if err.value != 0:
        raise ParODEError(err.value, where)


def error_description(code: int) -> str:
    buf = C.create_string_buffer(256)
    c = C.c_int(code)
    lib.GetErrorDescription(C.byref(c), buf)
    return buf.value.decode()


def available_gpus():
    n = C.c_int(0)
    ids = (C.c_int * 64)()
    e = C.c_int(0)
    lib.GetAvailableGPUs(C.byref(n), ids, C.byref(e))
    _check(e, "GetAvailableGPUs")
    return [ids[i] for i in range(n.value)]


def init(device_ids=None) -> None:
    """InitializeAllGPUs, or GetAvailableGPUs + InitializeSelectedGPUs."""
    e = C.c_int(0)
    if device_ids is None:
        lib.InitializeAllGPUs(b"", b"", C.byref(e))
        _check(e, "InitializeAllGPUs")
        return
    available_gpus()
    ids = (C.c_int * len(device_ids))(*device_ids)
    n = C.c_int(len(device_ids))
    lib.InitializeSelectedGPUs(C.byref(n), ids, b"", b"", C.byref(e))
    _check(e, "InitializeSelectedGPUs")


def close() -> None:
    lib.CloseGPUC()


def set_option(option: int, value: int) -> None:
    e = C.c_int(0)
    lib.ParODE_SetOption(option, value, C.byref(e))
    _check(e, "ParODE_SetOption")


def get_option(option: int) -> int:
    e = C.c_int(0)
    v = lib.ParODE_GetOption(option, C.byref(e))
    _check(e, "ParODE_GetOption")
    return int(v)


def num_outputs(solver: int, t0: float, t_end: float, h: float) -> int:
    return int(lib.ParODE_NumOutputs(solver, t0, t_end, h))


def register_input(source: str) -> int:
    """RegisterInput: `fType UFunc(fType t, int nInputIndex)` in CUDA C++ (NVRTC)."""
    idx = C.c_int(-1)
    e = C.c_int(0)
    lib.RegisterInput(source.encode(), C.byref(idx), C.byref(e))
    _check(e, "RegisterInput")
    return idx.value


def register_sinusoid(a, f, phi) -> int:
    """Built-in input u_i(t) = sum_k a[i,k] sin(2 pi f[i,k] t + phi[i,k])."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    f = np.ascontiguousarray(f, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    m, K = a.shape
    idx = C.c_int(-1)
    e = C.c_int(0)
    lib.ParODE_RegisterSinusoidInput(m, K, _dp(a), _dp(f), _dp(phi), C.byref(idx), C.byref(e))
    _check(e, "ParODE_RegisterSinusoidInput")
    return idx.value


def _f64(a):
    """a as a C-contiguous float64 array (itself when it already is one)."""
    if type(a) is np.ndarray and a.dtype == np.float64 and a.flags.c_contiguous:
        return a
    return np.ascontiguousarray(a, dtype=np.float64)


def _sys_arrays(A, B, Cm, D, x0):
    if (type(A) is np.ndarray and type(x0) is np.ndarray and A.ndim == 2 and A.dtype == np.float64 and
            A.flags.c_contiguous and x0.dtype == np.float64 and x0.flags.c_contiguous):
        # already C-contiguous float64 (a batch of thousands passes here)
        B = None if B is None or np.size(B) == 0 else _f64(B)
        Cm = None if Cm is None or np.size(Cm) == 0 else _f64(Cm)
        D = None if D is None or np.size(D) == 0 else _f64(D)
        n = A.shape[0]
        m = B.shape[1] if B is not None else (D.shape[1] if D is not None else 0)
        p = Cm.shape[0] if Cm is not None else (D.shape[0] if D is not None else 0)
        return A, B, Cm, D, x0, n, m, p
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    B = None if B is None or np.size(B) == 0 else np.ascontiguousarray(B, dtype=np.float64)
    Cm = None if Cm is None or np.size(Cm) == 0 else np.ascontiguousarray(Cm, dtype=np.float64)
    D = None if D is None or np.size(D) == 0 else np.ascontiguousarray(D, dtype=np.float64)
    x0 = np.ascontiguousarray(np.zeros(n) if x0 is None else x0, dtype=np.float64)
    m = B.shape[1] if B is not None else (D.shape[1] if D is not None else 0)
    p = Cm.shape[0] if Cm is not None else (D.shape[0] if D is not None else 0)
    return A, B, Cm, D, x0, n, m, p


def simulate(A, B, Cm, D, x0, u_index: int, t0: float, t_end: float, h: float, solver: int = RK4,
             precision: int = FP64, t_out=None, y_out=None):
    """ParODE_SimulateODE_d: returns (t, y) with y of shape (T, outputs).

    t_out / y_out: optional caller-owned float64 arrays of T and (T, outputs)
    elements (C-contiguous; pinned host memory makes the copy-out fastest),
    filled in place and returned instead of new arrays."""
    A, B, Cm, D, x0, n, m, p = _sys_arrays(A, B, Cm, D, x0)
    T = num_outputs(solver, t0, t_end, h)
    if T <= 0:
        raise ParODEError(-6, "simulate")
    q = n if (Cm is None and D is None) else p
    t = np.zeros(T) if t_out is None else t_out
    y = np.zeros((T, q)) if y_out is None else y_out
    for arr, size in ((t, T), (y, T * q)):
        if arr.dtype != np.float64 or not arr.flags.c_contiguous or arr.size < size:
            raise ValueError("simulate: output arrays must be C-contiguous float64 of the output size")
    ns = C.c_longlong(0)
    e = C.c_int(0)
    lib.ParODE_SimulateODE_d(_dp(A), _dp(B), _dp(Cm), _dp(D), m, n, p, int(B is None), int(Cm is None),
                             int(D is None), u_index, t0, t_end, h, _dp(x0), solver, precision, _dp(t), _dp(y),
                             C.byref(ns), C.byref(e))
    _check(e, "ParODE_SimulateODE_d")
    return t[:ns.value], y[:ns.value]


def affine_scan_general(M_ptr: int, V_ptr: int, x0_ptr: int, ns: int, count: int, X_ptr: int,
                        precision: int = FP64, stream: int = 0) -> None:
    """ParODE_AffineScanGeneral on device pointers (e.g. torch CUDA tensors'
    data_ptr()): X[k] = x_k, x_{k+1} = M[k] x_k + V[k], x_0 = x0 (0 pointers:
    zero), all row-major FP64.  Returns when the scan is done."""
    e = C.c_int(0)
    lib.ParODE_AffineScanGeneral(C.c_void_p(M_ptr or None), C.c_void_p(V_ptr or None), C.c_void_p(x0_ptr or None),
                                 ns, count, precision, C.c_void_p(X_ptr or None), C.c_void_p(stream or None),
                                 C.byref(e))
    _check(e, "ParODE_AffineScanGeneral")


def tune_response_block(solver: int, n: int, m: int, p: int, T: int, precision: int = FP64):
    """ParODE_TuneResponseBlock: times the response leaf's block lengths for
    this class of systems on the current device and records the fastest.
    Returns (log2 of the block length, its median ms, the untuned choice's ms)."""
    r = C.c_int(0)
    best, model = C.c_float(0), C.c_float(0)
    e = C.c_int(0)
    lib.ParODE_TuneResponseBlock(solver, n, m, p, T, precision, C.byref(r), C.byref(best), C.byref(model), C.byref(e))
    _check(e, "ParODE_TuneResponseBlock")
    return r.value, float(best.value), float(model.value)


def tune_save(path: str, gpu: Optional[str] = None) -> int:
    e = C.c_int(0)
    n = lib.ParODE_TuneSave(path.encode(), None if gpu is None else gpu.encode(), C.byref(e))
    _check(e, "ParODE_TuneSave")
    return int(n)


def tune_load(path: str, gpu: Optional[str] = None) -> int:
    e = C.c_int(0)
    n = lib.ParODE_TuneLoad(path.encode(), None if gpu is None else gpu.encode(), C.byref(e))
    _check(e, "ParODE_TuneLoad")
    return int(n)


def tune_clear() -> None:
    lib.ParODE_TuneClear()


def simulate_f32(A, B, Cm, D, x0, u_index: int, t0: float, t_end: float, h: float, solver: int = RK4, t_out=None,
                 y_out=None):
    """The reference C ABI SimulateODE (float arrays; the precision mode is
    PARODE_OPT_PRECISION's).  Returns (t, y, err).  t_out / y_out: optional
    caller-owned float32 arrays of T and (T, outputs) elements (C-contiguous;
    pinned host memory makes the copy-out fastest), filled in place."""
    A32 = np.ascontiguousarray(A, dtype=np.float32)
    n = A32.shape[0]
    zB, zC, zD = int(B is None or np.size(B) == 0), int(Cm is None or np.size(Cm) == 0), int(D is None or np.size(D) == 0)
    B32 = np.ascontiguousarray(B if not zB else np.zeros(1), dtype=np.float32)
    C32 = np.ascontiguousarray(Cm if not zC else np.zeros(1), dtype=np.float32)
    D32 = np.ascontiguousarray(D if not zD else np.zeros(1), dtype=np.float32)
    x32 = np.ascontiguousarray(x0, dtype=np.float32)
    m = B32.shape[1] if not zB else (D32.shape[1] if not zD else 0)
    p = C32.shape[0] if not zC else (D32.shape[0] if not zD else n)
    T = max(num_outputs(solver, t0, t_end, h), 1)
    t = np.zeros(T, dtype=np.float32) if t_out is None else t_out
    y = np.zeros((T, p), dtype=np.float32) if y_out is None else y_out
    for a_, shape in ((t, (T,)), (y, (T, p))):
        if a_.dtype != np.float32 or a_.shape != shape or not a_.flags.c_contiguous:
            raise ValueError("simulate_f32: t_out / y_out must be C-contiguous float32 arrays of the output shape")
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    args_i = [C.c_int(v) for v in (m, n, p, zB, zC, zD, u_index)]
    ts, te, hs = C.c_double(t0), C.c_double(t_end), C.c_double(h)
    sv = C.c_int(solver)
    nsteps = C.c_int(0)
    e = C.c_int(0)
    lib.SimulateODE(fp(A32), fp(B32), fp(C32), fp(D32), *[C.byref(v) for v in args_i], C.byref(ts), C.byref(te),
                    C.byref(hs), fp(x32), C.byref(sv), fp(t), fp(y), C.byref(nsteps), C.byref(e))
    return t[:nsteps.value], y[:nsteps.value], e.value


class Plan:
    """Device-resident solve (ParODE_PlanCreate / Execute / GetOutput).

    With shards > 1 the plan is time shard `shard` of the solve
    (ParODE_PlanCreateShard): it runs through shard_up / shard_down instead of
    execute (parode_b200.multi.solve_time_partitioned drives them)."""

    def __init__(self, A, B, Cm, D, x0, u_index: int, t0: float, t_end: float, h: float, solver: int = RK4,
                 precision: int = FP64, shard: int = 0, shards: int = 1):
        A, B, Cm, D, x0, n, m, p = _sys_arrays(A, B, Cm, D, x0)
        e = C.c_int(0)
        if shards > 1 or shard != 0:
            self._h = lib.ParODE_PlanCreateShard(_dp(A), _dp(B), _dp(Cm), _dp(D), m, n, p, int(B is None),
                                                 int(Cm is None), int(D is None), u_index, t0, t_end, h, _dp(x0),
                                                 solver, precision, shard, shards, C.byref(e))
            _check(e, "ParODE_PlanCreateShard")
        else:
            self._h = lib.ParODE_PlanCreate(_dp(A), _dp(B), _dp(Cm), _dp(D), m, n, p, int(B is None),
                                            int(Cm is None), int(D is None), u_index, t0, t_end, h, _dp(x0), solver,
                                            precision, C.byref(e))
            _check(e, "ParODE_PlanCreate")
        self.num_outputs = int(lib.ParODE_PlanNumOutputs(self._h))
        self.channels = int(lib.ParODE_PlanNumOutputChannels(self._h))

    @property
    def shard_info(self):
        """(first scan step, scan steps, items per shard, doubles per item, shards)
        of a time-shard plan."""
        info = (C.c_longlong * 5)()
        lib.ParODE_PlanShardInfo(self._h, info)
        return tuple(int(v) for v in info)

    def shard_up(self, top_dev_ptr: int, stream: int = 0) -> None:
        e = C.c_int(0)
        lib.ParODE_PlanShardUp(self._h, C.c_void_p(top_dev_ptr), C.c_void_p(stream or None), C.byref(e))
        _check(e, "ParODE_PlanShardUp")

    def shard_down(self, gathered_dev_ptr: int, y_dev_ptr: int = 0, stream: int = 0) -> None:
        e = C.c_int(0)
        lib.ParODE_PlanShardDown(self._h, C.c_void_p(gathered_dev_ptr), C.c_void_p(y_dev_ptr or None),
                                 C.c_void_p(stream or None), C.byref(e))
        _check(e, "ParODE_PlanShardDown")

    def execute(self, y_dev_ptr: int = 0, stream: int = 0) -> None:
        e = C.c_int(0)
        lib.ParODE_PlanExecute(self._h, C.c_void_p(y_dev_ptr or None), C.c_void_p(stream or None), C.byref(e))
        _check(e, "ParODE_PlanExecute")

    def output(self, t_out=None, y_out=None):
        """(t, y) of the last execute; t_out / y_out: optional caller-owned
        float64 arrays (pinned host memory makes the copy one DMA)."""
        t = np.zeros(self.num_outputs) if t_out is None else t_out
        y = np.zeros((self.num_outputs, self.channels)) if y_out is None else y_out
        e = C.c_int(0)
        lib.ParODE_PlanGetOutput(self._h, _dp(t), _dp(y), C.byref(e))
        _check(e, "ParODE_PlanGetOutput")
        return t, y

    def set_profiling(self, on: bool = True) -> None:
        e = C.c_int(0)
        lib.ParODE_PlanSetProfiling(self._h, int(on), C.byref(e))
        _check(e, "ParODE_PlanSetProfiling")

    def stage_times(self):
        """[(stage, ms)] of the last profiled execute (synchronises)."""
        ms = (C.c_float * 64)()
        names = C.create_string_buffer(4096)
        e = C.c_int(0)
        n = lib.ParODE_PlanStageTimes(self._h, ms, 64, names, 4096, C.byref(e))
        _check(e, "ParODE_PlanStageTimes")
        labels = names.value.decode().split("\n")
        return [(labels[i], float(ms[i])) for i in range(min(n, 64))]

    @property
    def precision(self) -> int:
        """Precision form actually used (FP64, MIXED or TF32)."""
        return int(lib.ParODE_PlanPrecision(self._h))

    @property
    def path(self) -> int:
        return int(lib.ParODE_PlanPath(self._h))

    @property
    def response_shape(self):
        """(B, K, NP, blocks) of the block-response leaf, zeros on other paths."""
        info = (C.c_longlong * 4)()
        lib.ParODE_PlanResponseShape(self._h, info)
        return tuple(int(v) for v in info)

    @property
    def launch_count(self) -> int:
        return int(lib.ParODE_PlanLaunchCount(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.ParODE_PlanDestroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent solves set up once and run together (ParODE_Batch*).

    systems: a sequence of dicts with keys A, B, C, D (None = absent), x0,
    u (input index), t0, t_end, h, solver."""

    def __init__(self, systems, precision: int = FP64):
        N = len(systems)
        keep = []
        cols = {k: [] for k in ("A", "B", "C", "D", "x0", "m", "n", "p", "zB", "zC", "zD", "u", "solver", "t0", "t1",
                                "h")}
        for s in systems:
            A, B, Cm, D, x0, n, m, p = _sys_arrays(s["A"], s.get("B"), s.get("C"), s.get("D"), s["x0"])
            for k, v in (("A", A), ("B", B), ("C", Cm), ("D", D), ("x0", x0)):
                if v is not None:
                    keep.append(v)
                    cols[k].append(v.ctypes.data)
                else:
                    cols[k].append(None)
            cols["m"].append(m)
            cols["n"].append(n)
            cols["p"].append(p)
            cols["zB"].append(int(B is None))
            cols["zC"].append(int(Cm is None))
            cols["zD"].append(int(D is None))
            cols["u"].append(int(s.get("u", 0)))
            cols["solver"].append(int(s.get("solver", RK4)))
            cols["t0"].append(s["t0"])
            cols["t1"].append(s["t_end"])
            cols["h"].append(s["h"])
        # the argument arrays built in bulk (one ctypes construction each)
        arrs = {k: (C.c_void_p * N)(*cols[k]) for k in ("A", "B", "C", "D", "x0")}
        ints = {k: (C.c_int * N)(*cols[k]) for k in ("m", "n", "p", "zB", "zC", "zD", "u", "solver")}
        dbl = {k: (C.c_double * N)(*cols[k]) for k in ("t0", "t1", "h")}
        e = C.c_int(0)
        ip = lambda a: C.cast(a, C.POINTER(C.c_int))
        dpp = lambda a: C.cast(a, C.POINTER(C.c_double))
        vp = lambda a: C.cast(a, C.POINTER(C.c_void_p))
        self._h = lib.ParODE_BatchCreate(N, vp(arrs["A"]), vp(arrs["B"]), vp(arrs["C"]), vp(arrs["D"]),
                                         ip(ints["m"]), ip(ints["n"]), ip(ints["p"]), ip(ints["zB"]), ip(ints["zC"]),
                                         ip(ints["zD"]), ip(ints["u"]), dpp(dbl["t0"]), dpp(dbl["t1"]), dpp(dbl["h"]),
                                         vp(arrs["x0"]), ip(ints["solver"]), precision, C.byref(e))
        _check(e, "ParODE_BatchCreate")
        self.size = N
        self._shapes = None  # (outputs, channels) per system, read on first use

    def _shape_lists(self):
        if self._shapes is None:
            self._shapes = ([int(lib.ParODE_BatchNumOutputs(self._h, i)) for i in range(self.size)],
                            [int(lib.ParODE_BatchNumOutputChannels(self._h, i)) for i in range(self.size)])
        return self._shapes

    @property
    def num_outputs(self):
        return self._shape_lists()[0]

    @property
    def channels(self):
        return self._shape_lists()[1]

    def execute(self, stream: int = 0) -> None:
        e = C.c_int(0)
        lib.ParODE_BatchExecute(self._h, C.c_void_p(stream or None), C.byref(e))
        _check(e, "ParODE_BatchExecute")

    def output(self, i: int):
        t = np.zeros(self.num_outputs[i])
        y = np.zeros((self.num_outputs[i], self.channels[i]))
        e = C.c_int(0)
        lib.ParODE_BatchGetOutput(self._h, i, _dp(t), _dp(y), C.byref(e))
        _check(e, "ParODE_BatchGetOutput")
        return t, y

    def device_output(self, i: int) -> int:
        return int(lib.ParODE_BatchDeviceOutput(self._h, i) or 0)

    def path(self, i: int) -> int:
        return int(lib.ParODE_BatchPath(self._h, i))

    def precision(self, i: int) -> int:
        return int(lib.ParODE_BatchPrecision(self._h, i))

    @property
    def launch_count(self) -> int:
        return int(lib.ParODE_BatchLaunchCount(self._h))

    @property
    def state_steps(self) -> float:
        return float(lib.ParODE_BatchStateSteps(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.ParODE_BatchDestroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Asynchronous solves with continuous batching (ParODE_Server*).

    submit() queues a solve and returns its id; poll(id) tells whether it is
    finished; result(id) returns (t, y, latency_ms) and releases it."""

    STAT_KEYS = ("submitted", "completed", "failed", "p50_ms", "p99_ms", "mean_ms", "max_ms", "state_steps",
                 "span_s", "peak_bytes", "batches")

    def __init__(self, precision: int = FP64, hbm_budget_bytes: float = 150e9, max_batch: int = 256,
                 max_inflight: int = 8):
        e = C.c_int(0)
        self._h = lib.ParODE_ServerCreate(precision, float(hbm_budget_bytes), max_batch, max_inflight, C.byref(e))
        _check(e, "ParODE_ServerCreate")
        self._shape = {}

    def submit(self, A, B, Cm, D, x0, u_index: int, t0: float, t_end: float, h: float, solver: int = RK4) -> int:
        A, B, Cm, D, x0, n, m, p = _sys_arrays(A, B, Cm, D, x0)
        e = C.c_int(0)
        rid = lib.ParODE_ServerSubmit(self._h, _dp(A), _dp(B), _dp(Cm), _dp(D), m, n, p, int(B is None),
                                      int(Cm is None), int(D is None), u_index, t0, t_end, h, _dp(x0), solver,
                                      C.byref(e))
        _check(e, "ParODE_ServerSubmit")
        return int(rid)

    def poll(self, rid: int) -> bool:
        n = C.c_longlong(0)
        c = C.c_int(0)
        e = C.c_int(0)
        done = lib.ParODE_ServerPoll(self._h, rid, C.byref(n), C.byref(c), C.byref(e))
        _check(e, "ParODE_ServerPoll")
        if done:
            self._shape[rid] = (int(n.value), int(c.value))
        return bool(done)

    def result(self, rid: int):
        if rid not in self._shape and not self.poll(rid):
            raise ParODEError(-9, "ParODE_ServerResult: request not finished")
        T, p = self._shape.pop(rid)
        t = np.zeros(T)
        y = np.zeros((T, p))
        lat = C.c_double(0)
        e = C.c_int(0)
        lib.ParODE_ServerResult(self._h, rid, _dp(t), _dp(y), C.byref(lat), C.byref(e))
        _check(e, "ParODE_ServerResult")
        return t, y, float(lat.value)

    def wait(self, rid: int, timeout_s: float = 600.0, interval_s: float = 0.0005):
        import time as _time
        t_end = _time.monotonic() + timeout_s
        while not self.poll(rid):
            if _time.monotonic() > t_end:
                raise TimeoutError(f"request {rid} not finished after {timeout_s} s")
            _time.sleep(interval_s)
        return self.result(rid)

    def stats(self) -> dict:
        v = (C.c_double * 12)()
        e = C.c_int(0)
        lib.ParODE_ServerStats(self._h, v, C.byref(e))
        _check(e, "ParODE_ServerStats")
        return {k: float(v[i]) for i, k in enumerate(self.STAT_KEYS)}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.ParODE_ServerDestroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
