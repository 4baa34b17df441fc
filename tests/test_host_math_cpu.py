"""Host FP64 set-up (parode_b200/csrc/host_math.cpp) on the CPU.

The discretisation is pure C++: compiled here with g++ beside a small driver,
its maps are checked against numpy restatements of the formulas the reference
uses (RK4 series, Sources/RungeKutta4thOrder.cpp:36-70; the ABM companion map,
Sources/AdamsMoulton.cpp:238-316), and the compact form the batch stages (the
ABM map's last block row alone) against the full map.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "parode_b200", "csrc")

DRIVER = r"""
#include "host_math.h"
#include <cmath>
#include <cstdio>
#include <vector>
using namespace parode;
int main()
{
    const int n = 5, m = 2;
    const double h = 0.01;
    std::vector<double> A(n * n), B(n * m);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) A[i * n + j] = std::sin(7.0 * i + j) - (i == j ? 2.0 : 0.0);
    for (int i = 0; i < n * m; ++i) B[i] = std::cos(3.0 * i);
    std::vector<double> P4(n * n), B4(n * 3 * m), PA(16 * n * n), BA(n * 5 * m), L(n * 4 * n), BL(n * 5 * m);
    discretise_rk4(n, m, A.data(), B.data(), h, P4.data(), B4.data());
    discretise_abm(n, m, A.data(), B.data(), h, PA.data(), BA.data());
    discretise_abm_last(n, m, A.data(), B.data(), h, L.data(), BL.data());
    auto dump = [](const char* name, const std::vector<double>& v) {
        std::printf("%s", name);
        for (double x : v) std::printf(" %.17g", x);
        std::printf("\n");
    };
    dump("P4", P4); dump("B4", B4); dump("PA", PA); dump("BA", BA); dump("L", L); dump("BL", BL);
    return 0;
}
"""


@pytest.fixture(scope="module")
def maps(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("host_math")
    drv = d / "driver.cpp"
    drv.write_text(DRIVER)
    exe = d / "driver"
    subprocess.run([gxx, "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC, str(drv),
                    os.path.join(CSRC, "host_math.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.strip().splitlines():
        name, *vals = line.split()
        res[name] = np.array([float(v) for v in vals])
    n, m, h = 5, 2, 0.01
    A = np.array([[np.sin(7.0 * i + j) - (2.0 if i == j else 0.0) for j in range(n)] for i in range(n)])
    B = np.array([np.cos(3.0 * i) for i in range(n * m)]).reshape(n, m)
    return res, A, B, n, m, h


def test_rk4_map_is_the_fourth_order_series(maps):
    res, A, B, n, m, h = maps
    hA = h * A
    I = np.eye(n)
    phi = I + hA + hA @ hA / 2 + hA @ hA @ hA / 6 + hA @ hA @ hA @ hA / 24
    assert np.allclose(res["P4"].reshape(n, n), phi, rtol=0, atol=1e-15)
    # B1 = h/6 (I + hA + h^2A^2/2 + h^3A^3/4) B, B2 = h/6 (4I + 2hA + h^2A^2/2) B, B3 = h/6 B
    b1 = h / 6 * (I + hA + hA @ hA / 2 + hA @ hA @ hA / 4) @ B
    b2 = h / 6 * (4 * I + 2 * hA + hA @ hA / 2) @ B
    b3 = h / 6 * B
    assert np.allclose(res["B4"].reshape(n, 3 * m), np.hstack([b1, b2, b3]), rtol=0, atol=1e-16)


def test_abm_map_is_the_companion_form(maps):
    res, A, B, n, m, h = maps
    N = 4 * n
    P = res["PA"].reshape(N, N)
    # block rows 0..2 shift exactly: block b reads block b + 1
    shift = np.zeros((3 * n, N))
    for r in range(3 * n):
        shift[r, r + n] = 1.0
    assert np.array_equal(P[: 3 * n], shift)
    hA = h * A
    A2 = hA @ hA
    last = np.hstack([-81 / 576 * A2, hA / 24 + 333 / 576 * A2, -5 * hA / 24 - 531 / 576 * A2,
                      np.eye(n) + 28 * hA / 24 + 495 / 576 * A2])
    assert np.allclose(P[3 * n:], last, rtol=0, atol=1e-15)


def test_abm_compact_rows_equal_the_full_map(maps):
    res, A, B, n, m, h = maps
    N = 4 * n
    assert np.array_equal(res["L"].reshape(n, N), res["PA"].reshape(N, N)[3 * n:])
    assert np.array_equal(res["BL"], res["BA"])
