"""ctypes front end of the CPU oracle (oracle/libparode_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker.  The product
library never imports this module.

See parode_oracle.h for what each entry point restates from the reference
(apatriciu/ParODE) and where.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from typing import Callable, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libparode_oracle.so")

RK4 = 0
ABM = 1

_UFUNC = C.CFUNCTYPE(C.c_double, C.c_double, C.c_int, C.c_void_p)


class _Sinusoid(C.Structure):
    _fields_ = [("m", C.c_int), ("K", C.c_int), ("a", C.POINTER(C.c_double)),
                ("f", C.POINTER(C.c_double)), ("phi", C.POINTER(C.c_double))]


class _Input(C.Structure):
    _fields_ = [("fn", C.c_void_p), ("ctx", C.c_void_p), ("float_time", C.c_int)]


class _System(C.Structure):
    _fields_ = [("n", C.c_int), ("m", C.c_int), ("p", C.c_int),
                ("zeroB", C.c_int), ("zeroC", C.c_int), ("zeroD", C.c_int),
                ("A", C.POINTER(C.c_double)), ("B", C.POINTER(C.c_double)),
                ("C", C.POINTER(C.c_double)), ("D", C.POINTER(C.c_double)),
                ("x0", C.POINTER(C.c_double))]


def build() -> str:
    """Compile the oracle with its Makefile (gcc only, seconds)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.po_num_outputs.restype = C.c_long
        L.po_num_outputs.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_long)]
        L.po_time_vector.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_float)]
        L.po_rk4_discretise.argtypes = [C.c_int, C.c_int, dp, dp, C.c_double, dp, dp]
        L.po_abm_discretise.argtypes = [C.c_int, C.c_int, dp, dp, C.c_double, dp, dp]
        L.po_abm_startup.argtypes = [C.POINTER(_System), C.POINTER(_Input), C.c_double, C.c_double, dp]
        L.po_simulate_affine.restype = C.c_int
        L.po_simulate_affine.argtypes = [C.POINTER(_System), C.POINTER(_Input), C.c_int, C.c_double,
                                         C.c_double, C.c_double, dp, C.POINTER(C.c_long)]
        for nm in ("po_stepper_rk4", "po_stepper_abm"):
            getattr(L, nm).restype = C.c_int
            getattr(L, nm).argtypes = [C.POINTER(_System), C.POINTER(_Input), C.c_double, C.c_double,
                                       C.c_long, C.c_int, dp]
        L.po_simulate_refscan_f32.restype = C.c_int
        L.po_simulate_refscan_f32.argtypes = [C.POINTER(_System), C.POINTER(_Input), C.c_int, C.c_double,
                                              C.c_double, C.c_double, C.c_long, C.POINTER(C.c_float),
                                              C.POINTER(C.c_long)]
        L.po_rel_err.restype = C.c_double
        L.po_rel_err.argtypes = [dp, dp, C.c_long, C.c_int]
        L.po_simulate_affine_many.restype = C.c_int
        L.po_simulate_affine_many.argtypes = [C.c_int, C.POINTER(_System), C.POINTER(_Input), C.POINTER(C.c_int),
                                              dp, dp, dp, C.POINTER(dp)]
        L.po_threads.restype = C.c_int
        L.po_sinusoid_eval.restype = C.c_double
        L.po_sinusoid_eval.argtypes = [C.c_double, C.c_int, C.c_void_p]
        _lib = L
    return _lib


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return C.POINTER(C.c_double)()
    return a.ctypes.data_as(C.POINTER(C.c_double))


class System:
    """Row-major FP64 copy of (A, B, C, D, x0) with absent-matrix flags."""

    def __init__(self, A, B=None, Cm=None, D=None, x0=None):
        self.A = np.ascontiguousarray(A, dtype=np.float64)
        n = self.A.shape[0]
        self.B = None if B is None or np.size(B) == 0 else np.ascontiguousarray(B, dtype=np.float64)
        self.C = None if Cm is None or np.size(Cm) == 0 else np.ascontiguousarray(Cm, dtype=np.float64)
        self.D = None if D is None or np.size(D) == 0 else np.ascontiguousarray(D, dtype=np.float64)
        self.x0 = np.ascontiguousarray(np.zeros(n) if x0 is None else x0, dtype=np.float64)
        m = self.B.shape[1] if self.B is not None else (self.D.shape[1] if self.D is not None else 0)
        p = self.C.shape[0] if self.C is not None else (self.D.shape[0] if self.D is not None else 0)
        self.n, self.m, self.p = n, m, p
        self._c = _System(n, m, p, int(self.B is None), int(self.C is None), int(self.D is None),
                          _dptr(self.A), _dptr(self.B), _dptr(self.C), _dptr(self.D), _dptr(self.x0))

    @property
    def out_size(self) -> int:
        return self.n if (self.C is None and self.D is None) else self.p


class Input:
    """An input function u_i(t) for the oracle.

    `sinusoid(a, f, phi)` evaluates natively in C; `callable(fn)` wraps a
    Python function fn(t, i) -> float (slow; small cases only).  With
    float_time=True the time is rounded to float before the call and the
    value after it, the semantics of a UFunc compiled with fType = float.
    """

    def __init__(self):
        self._keep = []
        self._c = _Input(None, None, 0)

    @classmethod
    def zero(cls) -> "Input":
        return cls()

    @classmethod
    def sinusoid(cls, a, f, phi) -> "Input":
        self = cls()
        a = np.ascontiguousarray(a, dtype=np.float64)
        f = np.ascontiguousarray(f, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        m, K = a.shape
        s = _Sinusoid(m, K, _dptr(a), _dptr(f), _dptr(phi))
        self._keep += [a, f, phi, s]
        fp = C.cast(lib().po_sinusoid_eval, C.c_void_p)
        self._c = _Input(fp, C.cast(C.pointer(s), C.c_void_p), 0)
        return self

    @classmethod
    def callable(cls, fn: Callable[[float, int], float], float_time: bool = False) -> "Input":
        self = cls()
        cb = _UFUNC(lambda t, i, ctx: float(fn(t, i)))
        self._keep.append(cb)
        self._c = _Input(C.cast(cb, C.c_void_p), None, int(float_time))
        return self


def num_outputs(solver: int, t0: float, t_end: float, h: float):
    ns = C.c_long(0)
    nt = lib().po_num_outputs(solver, t0, t_end, h, C.byref(ns))
    return int(nt), int(ns.value)


def time_vector(solver: int, t0: float, t_end: float, h: float) -> np.ndarray:
    nt, _ = num_outputs(solver, t0, t_end, h)
    tv = np.zeros(max(nt, 1), dtype=np.float32)
    lib().po_time_vector(solver, t0, t_end, h, tv.ctypes.data_as(C.POINTER(C.c_float)))
    return tv[:nt]


def discretise(solver: int, A, B, h: float):
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    B = np.zeros((n, 0)) if B is None else np.ascontiguousarray(B, dtype=np.float64)
    m = B.shape[1]
    if solver == RK4:
        Phi = np.zeros((n, n)); Bbar = np.zeros((n, 3 * m))
        lib().po_rk4_discretise(n, m, _dptr(A), _dptr(B), h, _dptr(Phi), _dptr(Bbar))
    else:
        Phi = np.zeros((4 * n, 4 * n)); Bbar = np.zeros((n, 5 * m))
        lib().po_abm_discretise(n, m, _dptr(A), _dptr(B), h, _dptr(Phi), _dptr(Bbar))
    return Phi, Bbar


def simulate_affine(sys_: System, inp: Input, solver: int, t0: float, t_end: float, h: float):
    """O1: FP64 sequential recurrence.  Returns y as (T, p)."""
    nt, _ = num_outputs(solver, t0, t_end, h)
    if nt <= 0:
        raise ValueError("empty horizon")
    y = np.zeros((nt, sys_.out_size), dtype=np.float64)
    n_out = C.c_long(0)
    rc = lib().po_simulate_affine(C.byref(sys_._c), C.byref(inp._c), solver, t0, t_end, h, _dptr(y),
                                  C.byref(n_out))
    if rc != 0:
        raise RuntimeError(f"oracle error {rc}")
    return y


def simulate_affine_many(jobs):
    """O1 of many independent systems on all host threads.

    jobs: a sequence of (System, Input, solver, t0, t_end, h) whose inputs are
    sinusoids (thread-safe).  Returns the list of y arrays, each (T, p)."""
    count = len(jobs)
    if count == 0:
        return []
    systems = (_System * count)()
    inputs = (_Input * count)()
    solvers = (C.c_int * count)()
    t0s, t1s, hs = (C.c_double * count)(), (C.c_double * count)(), (C.c_double * count)()
    ys = []
    yp = (C.POINTER(C.c_double) * count)()
    for i, (sys_, inp, solver, t0, t_end, h) in enumerate(jobs):
        if inp._c.fn is not None and inp._c.ctx is None:
            raise ValueError("simulate_affine_many: Python callables are not thread-safe inputs")
        nt, _ = num_outputs(solver, t0, t_end, h)
        if nt <= 0:
            raise ValueError("empty horizon")
        y = np.zeros((nt, sys_.out_size), dtype=np.float64)
        ys.append(y)
        systems[i] = sys_._c
        inputs[i] = inp._c
        solvers[i], t0s[i], t1s[i], hs[i] = solver, t0, t_end, h
        yp[i] = _dptr(y)
    rc = lib().po_simulate_affine_many(count, systems, inputs, solvers, t0s, t1s, hs, yp)
    if rc != 0:
        raise RuntimeError(f"oracle error {rc}")
    return ys


def stepper(sys_: System, inp: Input, solver: int, t0: float, h: float, T: int, use_float: bool):
    """O2: the reference tests' sequential loops (RK4 or AB4/AM4 PECE)."""
    y = np.zeros((T, sys_.out_size), dtype=np.float64)
    fn = lib().po_stepper_rk4 if solver == RK4 else lib().po_stepper_abm
    rc = fn(C.byref(sys_._c), C.byref(inp._c), t0, h, T, int(use_float), _dptr(y))
    if rc != 0:
        raise RuntimeError(f"oracle error {rc}")
    return y


def refscan_f32(sys_: System, inp: Input, solver: int, t0: float, t_end: float, h: float, batch: int = 0):
    """O3: FP32 restatement of the reference's scan pipeline."""
    nt, _ = num_outputs(solver, t0, t_end, h)
    y = np.zeros((nt, sys_.out_size), dtype=np.float32)
    n_out = C.c_long(0)
    rc = lib().po_simulate_refscan_f32(C.byref(sys_._c), C.byref(inp._c), solver, t0, t_end, h, batch,
                                       y.ctypes.data_as(C.POINTER(C.c_float)), C.byref(n_out))
    if rc != 0:
        raise RuntimeError(f"oracle error {rc}")
    return y


def rel_err(y, yref) -> float:
    """Per output channel max_k |y - yref| / max_k |yref|, maximum over channels."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    yref = np.ascontiguousarray(yref, dtype=np.float64)
    T, p = yref.shape
    return float(lib().po_rel_err(_dptr(y), _dptr(yref), T, p))


def l2_err(y, yref, start: int = 1, stop: Optional[int] = None) -> float:
    """The reference tests' criterion sqrt(sum (y - yref)^2) over steps [start, stop)."""
    d = np.asarray(y, dtype=np.float64)[start:stop] - np.asarray(yref, dtype=np.float64)[start:stop]
    return math.sqrt(float(np.sum(d * d)))
