"""Golden outputs of the reference's own OpenCL kernels.

Runs oracle/_ref/ref_kernels (the reference's Kernels/ .cl files, unmodified,
driven as its scan driver drives them; built by `make -C oracle ref`) on an
OpenCL GPU for:
  - the reference tests' fixtures (tests/golden/ref_fixtures.json: the matrices
    its test programs draw with rand(), their UFunc sources, step counts),
  - the n=8 RK4 benchmark system (cfg1) and its ABM twin, with the sum-of-
    sinusoid input written as a UFunc that evaluates in double from the float
    time the reference's u kernel passes,
  - small systems whose steps per batch are capped at 64 (the reference's
    host carry between time batches) and systems without C and D (y = x),
and writes the float outputs (base64 float32) with their inputs into one JSON
file.  Usage (on a machine with an OpenCL GPU):

    make -C oracle ref
    python tests/golden/make_ref_kernel_outputs.py OUT.json

When no /etc/OpenCL/vendors entry exists, the NVIDIA driver's OpenCL library
is named to the Khronos loader with OCL_ICD_FILENAMES.
"""
import base64
import json
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from parode_b200 import workloads as wl  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_kernels")
KERNELS = os.path.join(ROOT, "oracle", "_ref", "kernels")
FIXTURES = os.path.join(ROOT, "tests", "golden", "ref_fixtures.json")
MAGIC = 0x50524B31
# c_abi ABM (scan dimension 512): the reference's matrix sweeps cost N^3 per
# step, so only its shorter horizons are run
C_ABI_ABM_MAX_STEPS = 500


def sinusoid_ufunc(u):
    """OpenCL C UFunc of u_i(t) = sum_k a_ik sin(2 pi f_ik t + phi_ik), in double."""
    lines = ["#pragma OPENCL EXTENSION cl_khr_fp64 : enable",
             "fType UFunc(fType t, int nInputIndex){", " double tt = t;", " double v = 0.0;"]
    for i in range(u.a.shape[0]):
        terms = []
        for k in range(u.a.shape[1]):
            terms.append(f"{float(u.a[i, k])!r} * sin(({float(2.0 * np.pi * u.f[i, k])!r}) * tt + {float(u.phi[i, k])!r})")
        lines.append(f" if (nInputIndex == {i}) {{ v = 0.0;" + "".join(f" v = v + {t};" for t in terms) + " }")
    lines.append(" return (fType)v;")
    lines.append("}")
    return "\n".join(lines) + "\n"


def write_case(path, solver, A, B, C, D, x0, t0, t_end, h, ufunc, max_batch=0):
    A = np.asarray(A, np.float32)
    B = np.asarray(B, np.float32)
    n, m = B.shape
    zC, zD = C is None, D is None
    p = (np.asarray(C).shape[0] if not zC else (np.asarray(D).shape[0] if not zD else 0))
    with open(path, "wb") as fh:
        fh.write(struct.pack("<8i", MAGIC, solver, n, m, p, int(zC), int(zD), max_batch))
        fh.write(struct.pack("<3d", t0, t_end, h))
        fh.write(A.tobytes() + B.tobytes())
        if not zC:
            fh.write(np.asarray(C, np.float32).tobytes())
        if not zD:
            fh.write(np.asarray(D, np.float32).tobytes())
        fh.write(np.asarray(x0, np.float32).tobytes())
        src = ufunc.encode()
        fh.write(struct.pack("<i", len(src)) + src)


def run_case(tmp, name, solver, A, B, C, D, x0, t0, t_end, h, ufunc, max_batch=0):
    cpath = os.path.join(tmp, name + ".case")
    opath = os.path.join(tmp, name + ".out")
    write_case(cpath, solver, A, B, C, D, x0, t0, t_end, h, ufunc, max_batch)
    subprocess.run([HARNESS, KERNELS, cpath, opath], check=True)
    with open(opath, "rb") as fh:
        T, q = struct.unpack("<2i", fh.read(8))
        tv = np.frombuffer(fh.read(4 * T), np.float32)
        y = np.frombuffer(fh.read(4 * T * q), np.float32).reshape(T, q)
    f32 = lambda a: None if a is None else np.asarray(a, np.float32).astype(float).tolist()
    return {"name": name, "solver": solver, "A": f32(A), "B": f32(B), "C": f32(C), "D": f32(D), "x0": f32(x0),
            "t0": t0, "t_end": t_end, "h": h, "ufunc": ufunc, "max_batch": max_batch, "T": T, "q": q,
            "time_f32": base64.b64encode(tv.tobytes()).decode(), "y_f32": base64.b64encode(y.tobytes()).decode()}


def cases():
    with open(FIXTURES) as fh:
        fixtures = json.load(fh)["fixtures"]
    for fx in fixtures:
        for c in fx["cases"]:
            if fx["name"] == "c_abi" and c["solver"] == 1 and c["steps"] > C_ABI_ABM_MAX_STEPS:
                continue
            yield (f"{fx['name']}_{'rk4' if c['solver'] == 0 else 'abm'}_{c['steps']}", c["solver"], fx["A"],
                   fx["B"], fx["C"], fx["D"], fx["x0"], 0.0, c["t_end"], fx["h"], fx["ufunc"], 0)
    c1 = wl.cfg1()
    uf = sinusoid_ufunc(c1.u)
    yield ("cfg1_rk4", 0, c1.A, c1.B, c1.C, c1.D, c1.x0, c1.t0, c1.t_end, c1.h, uf, 0)
    yield ("cfg1_abm", 1, c1.A, c1.B, c1.C, c1.D, c1.x0, c1.t0, c1.t_end, c1.h, uf, 0)
    for solver in (0, 1):
        s = wl.small(31 + solver, solver, 6, 2, 3, 700, h=0.01)
        uf = sinusoid_ufunc(s.u)
        tag = "rk4" if solver == 0 else "abm"
        yield (f"small_{tag}_batch64", solver, s.A, s.B, s.C, s.D, s.x0, s.t0, s.t_end, s.h, uf, 64)
        yield (f"small_{tag}_y_is_x", solver, s.A, s.B, None, None, s.x0, s.t0, s.t_end, s.h, uf, 0)


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "ref_kernel_outputs.json")
    if not os.path.isdir("/etc/OpenCL/vendors") and "OCL_ICD_FILENAMES" not in os.environ:
        for lib in ("/usr/lib/libnvidia-opencl.so.1", "/usr/lib/x86_64-linux-gnu/libnvidia-opencl.so.1"):
            if os.path.exists(lib):
                os.environ["OCL_ICD_FILENAMES"] = lib
                break
    res = []
    with tempfile.TemporaryDirectory() as tmp:
        for args in cases():
            print("case", args[0], flush=True)
            res.append(run_case(tmp, *args))
    doc = {"generator": "tests/golden/make_ref_kernel_outputs.py",
           "harness": "oracle/ref_kernels.c (the reference's Kernels/ .cl files through OpenCL)",
           "cases": res}
    with open(out, "w") as fh:
        json.dump(doc, fh)
    print("wrote", out, len(res), "cases")


if __name__ == "__main__":
    main()
