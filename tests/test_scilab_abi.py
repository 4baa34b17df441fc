"""The reference's Scilab call layout against libParODEShared.so.

tests/scilab_abi.c replays what SciLabInterface/ParODEInterfaceStubs.sci:84-135
hands to SimulateODE through Scilab's `call` (transposed column-major
matrices, tEnd with its 1e-4 h margin, flags and sizes from the matrix
shapes, xVect read back as an nOutputs x nSteps column-major matrix).  It is
compiled against include/ and the library here; on a GPU its outputs are
checked against the FP64 oracle for the Scilab tests' system and for a
non-symmetric one (where a transpose missing on either side would show).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "scilab_abi.c")
LIBDIR = os.path.join(ROOT, "parode_b200")

SYSTEMS = {
    0: dict(A=[[-2, 0], [0, -2]], B=np.eye(2), C=np.eye(2), D=np.eye(2), x0=[1, -1]),
    1: dict(A=[[-2, 1], [0.5, -3]], B=[[1, 2], [0, 1]], C=[[1, 0], [0.5, 1]], D=[[0.1, 0], [0, 0.2]], x0=[0.5, 2]),
}


def _build(tmp_path):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    if not os.path.exists(os.path.join(LIBDIR, "libParODEShared.so")):
        pytest.fail("libParODEShared.so is not built (make -C parode_b200)")
    exe = tmp_path / "scilab_abi"
    subprocess.run([gcc, "-O2", "-std=c11", "-DC_INCLUDE", "-I", os.path.join(ROOT, "include"), SRC, "-L", LIBDIR,
                    "-lParODEShared", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    return exe


def test_scilab_layout_program_builds(tmp_path):
    assert _build(tmp_path).exists()


@pytest.mark.gpu
@pytest.mark.parametrize("solver", [0, 1])
@pytest.mark.parametrize("case", [0, 1])
def test_scilab_layout_matches_oracle(tmp_path, solver, case):
    exe = _build(tmp_path)
    out = subprocess.run([str(exe), str(solver), str(case)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.strip().splitlines()
    n_steps, err = (int(v) for v in lines[0].split())
    assert err == 0 and n_steps == 50
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[1:]])
    t, y = rows[:, 0], rows[:, 1:]
    s = SYSTEMS[case]
    f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
    sysd = oracle.System(f32(s["A"]), f32(s["B"]), f32(s["C"]), f32(s["D"]), f32(s["x0"]))
    inp = oracle.Input.callable(lambda tt, i: tt if i < 2 else 0.0, float_time=True)
    t_end = 0.0 + (50 - 1) * 0.1 + 0.0001 * 0.1
    ref = oracle.simulate_affine(sysd, inp, solver, 0.0, t_end, 0.1)
    # tVect is float, printed with 9 significant digits: rounding the parsed
    # value back to float recovers it exactly
    assert np.array_equal(t.astype(np.float32), oracle.time_vector(solver, 0.0, t_end, 0.1))
    assert oracle.rel_err(y, ref) <= 1e-6, oracle.rel_err(y, ref)
