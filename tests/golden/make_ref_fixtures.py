"""Regenerates tests/golden/ref_fixtures.json.

The reference (apatriciu/ParODE) ships no golden vectors.  Its test programs
draw their systems from glibc rand() without calling srand(), i.e. from the
default seed 1, and accept a GPU result when sqrt(sum err^2) < 0.1 against a
sequential CPU loop.  This script replays those draws with the C library's own
rand() (each reference test is a separate process, so every fixture starts
from seed 1) and stores the matrices with the reference's float rounding,
together with the expected outputs of the reference tests' CPU loops as
restated by the oracle (O2, float) and the FP64 recurrence (O1).

    python tests/golden/make_ref_fixtures.py

Fixtures (file:line in the reference):
  rk4_unit   TestsSources/TestRungeKutta4thOrder.cpp:54-97,184-190  n=m=p=2, A=-5I+U, x0=10, h=0.1, 50 steps
  abm_unit   TestsSources/TestAdamsMoulton.cpp:58-95                n=m=p=2, A=-5I+2U, x0=10, h=0.1, 50 steps
  cpp_api    TestsSources/TestParODEInterface.cpp:312-361          n=20, m=p=4, A=-10I+0.01U, x0=1, h=0.1, 1000 steps
  c_abi      TestsSources/TestParODEStaticLibCInterface.cpp:527-604  n=128, m=p=4, A=-10I+0.01U, x0=0, h=0.1, 100..2000 steps
  python     PythonInterface/TestPythonODESolvers.py:8-26           A=[[-2,1],[.5,-3]], B=C=D=I, x0=[-1,1], u=t, ABM
  scilab     SciLabInterface/TestRK4.sce:63-74, TestABM.sce          A=-2I, B=C=D=I, x0=[1,-1], u=t, tEnd + 1e-4 h
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle import oracle  # noqa: E402

RAND_MAX_F = np.float32(2147483647)  # (fType)RAND_MAX rounds to 2^31


class GlibcRand:
    def __init__(self):
        self.libc = ctypes.CDLL("libc.so.6")
        self.libc.srand(1)  # glibc's default seed, as a process that never calls srand()

    def u(self) -> np.float32:
        """(fType)((fType)rand() / (fType)RAND_MAX)"""
        return np.float32(np.float32(self.libc.rand()) / RAND_MAX_F)


def f32(x) -> float:
    return float(np.float32(x))


def rk4_unit():
    r = GlibcRand()
    n = m = p = 2
    A = np.full((n, n), 0, dtype=np.float32)
    for i in range(n):
        A[i, i] = np.float32(-5.0)
    for i in range(n):
        for j in range(n):
            A[i, j] = np.float32(A[i, j] + r.u())          # A(row,col) += (fType)(...)
    B = np.array([[r.u() for _ in range(m)] for _ in range(n)], dtype=np.float32)
    C = np.array([[r.u() for _ in range(n)] for _ in range(p)], dtype=np.float32)
    D = np.array([[r.u() for _ in range(m)] for _ in range(p)], dtype=np.float32)
    return dict(name="rk4_unit", solvers=[0], A=A, B=B, C=C, D=D, x0=np.full(n, 10.0, np.float32), h=0.1,
                steps=[50], input="sin_cos", t_end_rule="(n-1)h",
                source="TestsSources/TestRungeKutta4thOrder.cpp:54-97,184-190")


def abm_unit():
    r = GlibcRand()
    n = m = p = 2
    A = np.zeros((n, n), dtype=np.float32)
    for i in range(n):
        A[i, i] = np.float32(-5.0)
    for i in range(n):
        for j in range(n):
            A[i, j] = np.float32(float(A[i, j]) + 2.0 * float(r.u()))  # A += 2.0 * (fType)(...)
    B = np.array([[r.u() for _ in range(m)] for _ in range(n)], dtype=np.float32)
    C = np.array([[r.u() for _ in range(n)] for _ in range(p)], dtype=np.float32)
    D = np.array([[r.u() for _ in range(m)] for _ in range(p)], dtype=np.float32)
    return dict(name="abm_unit", solvers=[1], A=A, B=B, C=C, D=D, x0=np.full(n, 10.0, np.float32), h=0.1,
                steps=[50], input="sin_cos", t_end_rule="(n-1)h",
                source="TestsSources/TestAdamsMoulton.cpp:58-95")


def api_system(n, m, p):
    r = GlibcRand()
    A = np.zeros((n, n), dtype=np.float32)
    for i in range(n):
        A[i, i] = np.float32(-10.0)
    for i in range(n):
        for j in range(n):
            A[i, j] = np.float32(A[i, j] + np.float32(np.float32(0.01) * r.u()))
    B = np.array([[r.u() for _ in range(m)] for _ in range(n)], dtype=np.float32)
    C = np.array([[r.u() for _ in range(n)] for _ in range(p)], dtype=np.float32)
    D = np.array([[r.u() for _ in range(m)] for _ in range(p)], dtype=np.float32)
    return A, B, C, D


def cpp_api():
    A, B, C, D = api_system(20, 4, 4)
    return dict(name="cpp_api", solvers=[0, 1], A=A, B=B, C=C, D=D, x0=np.ones(20, np.float32), h=0.1, steps=[1000],
                input="sin_cos_4", t_end_rule="(n-1)h", source="TestsSources/TestParODEInterface.cpp:312-361")


def c_abi():
    A, B, C, D = api_system(128, 4, 4)
    return dict(name="c_abi", solvers=[0, 1], A=A, B=B, C=C, D=D, x0=np.zeros(128, np.float32), h=0.1,
                steps=[100, 250, 500, 1000, 2000], input="sin_cos_4", t_end_rule="(n-1)h",
                source="TestsSources/TestParODEStaticLibCInterface.cpp:527-604")


def python_case():
    I = np.eye(2, dtype=np.float32)
    return dict(name="python", solvers=[1], A=np.array([[-2.0, 1.0], [0.5, -3.0]], np.float32), B=I, C=I, D=I,
                x0=np.array([-1.0, 1.0], np.float32), h=0.1, steps=[50], input="t_t", t_end_rule="(n-1)h",
                source="PythonInterface/TestPythonODESolvers.py:8-26")


def scilab_case():
    I = np.eye(2, dtype=np.float32)
    return dict(name="scilab", solvers=[0, 1], A=-2.0 * I, B=I, C=I, D=I, x0=np.array([1.0, -1.0], np.float32), h=0.1,
                steps=[50], input="t_t", t_end_rule="(n-1)h+1e-4h",
                source="SciLabInterface/TestRK4.sce:63-74, SciLabInterface/TestABM.sce:63-74")


INPUTS = {
    # UFunc sources registered by the reference tests (fType = float)
    "sin_cos": "fType UFunc(fType t, int nInputIndex){\n fType fVal = nInputIndex == 0 ? sin(t) :\n"
               " nInputIndex == 1 ? cos(t) :\n 0.0;\n return fVal;\n}\n",
    "sin_cos_4": "fType UFunc(fType t, int nInputIndex){\nfType fVal = nInputIndex == 0 ? (fType)(sin(t)) :\n"
                 "nInputIndex == 1 ? (fType)(cos(t)) :\nnInputIndex == 2 ? (fType)(sin(t)) :\n"
                 "nInputIndex == 3 ? (fType)(cos(t)) :\n0.0;\nreturn fVal;\n}\n",
    "t_t": "fType UFunc(fType t, int nInputIndex){\nfType fVal = nInputIndex == 0 ? t :\nnInputIndex == 1 ? t :\n"
           "0.0;\nreturn fVal;\n}\n",
}


def py_input(kind):
    if kind == "sin_cos":
        return lambda t, i: math.sin(t) if i == 0 else (math.cos(t) if i == 1 else 0.0)
    if kind == "sin_cos_4":
        return lambda t, i: math.sin(t) if i in (0, 2) else (math.cos(t) if i in (1, 3) else 0.0)
    if kind == "t_t":
        return lambda t, i: t if i < 2 else 0.0
    raise KeyError(kind)


def t_end(fx, steps):
    t = (steps - 1) * fx["h"]
    if fx["t_end_rule"].endswith("+1e-4h"):
        t += 1e-4 * fx["h"]
    return t


def main():
    fixtures = [rk4_unit(), abm_unit(), cpp_api(), c_abi(), python_case(), scilab_case()]
    out = []
    for fx in fixtures:
        sysd = oracle.System(fx["A"].astype(np.float64), fx["B"].astype(np.float64), fx["C"].astype(np.float64),
                             fx["D"].astype(np.float64), fx["x0"].astype(np.float64))
        fn = py_input(fx["input"])
        inp32 = oracle.Input.callable(fn, float_time=True)
        cases = []
        for solver in fx["solvers"]:
            for steps in fx["steps"]:
                te = t_end(fx, steps)
                nt, _ = oracle.num_outputs(solver, 0.0, te, fx["h"])
                y_o2 = oracle.stepper(sysd, inp32, solver, 0.0, fx["h"], nt, use_float=True)
                y_o1 = oracle.simulate_affine(sysd, inp32, solver, 0.0, te, fx["h"])
                cases.append(dict(solver=solver, steps=steps, t_end=te, n_out=nt,
                                  time=oracle.time_vector(solver, 0.0, te, fx["h"]).astype(float).tolist(),
                                  y_o2_f32=y_o2.tolist(), y_o1=y_o1.tolist(),
                                  l2_o1_vs_o2=oracle.l2_err(y_o1, y_o2, 1 if solver == 0 else 4,
                                                            None if solver == 0 else nt - 1)))
        rec = {k: (v.astype(float).tolist() if isinstance(v, np.ndarray) else v) for k, v in fx.items()}
        rec["ufunc"] = INPUTS[fx["input"]]
        rec["cases"] = cases
        out.append(rec)
    path = os.path.join(HERE, "ref_fixtures.json")
    with open(path, "w") as fh:
        json.dump({"generator": "tests/golden/make_ref_fixtures.py", "criterion": "sqrt(sum err^2) < 0.1",
                   "fixtures": out}, fh)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.1f} MB)")
    for rec in out:
        for c in rec["cases"]:
            print(f"{rec['name']:9s} solver={c['solver']} steps={c['steps']:5d} n_out={c['n_out']:5d} "
                  f"L2(O1,O2)={c['l2_o1_vs_o2']:.3e}")


if __name__ == "__main__":
    main()
