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


TIME_DRIVER = r"""
#include "host_math.h"
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>
using namespace parode;
// the reference's accumulation, one dependent step at a time
// (Sources/GPUFixedStepIterative.cpp:141-146)
static void plain(int solver, double t0, double tEnd, double h, double* tv)
{
    long ns = 0;
    long nt = num_outputs(solver, t0, tEnd, h, &ns);
    if (nt <= 0) return;
    long pre = nt - ns;
    double ts = solver == 1 ? t0 + 3.0 * h : t0;
    for (long i = 0; i < pre; ++i) tv[i] = (double)(float)(ts - (double)(pre - i) * h);
    float prev = (float)ts;
    tv[pre] = prev;
    for (long i = 1; i < ns; ++i) {
        prev = (float)((double)prev + h);
        tv[pre + i] = prev;
    }
}
int main()
{
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<double> a, b;
    int cases = 0, bad = 0;
    const double hs[] = {1e-4, 1e-3, 0.1, 0.5, 1.0 / 3.0, 5e-4, 1e-5, 0.25, 0.7, 1e-7, 0.0625};
    const double t0s[] = {0.0, 1.0, -1.0, -3.7, 100.0, 1e-3, -0.05, 12345.678, -100.0, 2.5, -0.5};
    auto run = [&](int solver, double t0, double h, long T) {
        const double t1 = t0 + (double)(T - 1) * h;
        long nt = num_outputs(solver, t0, t1, h, nullptr);
        if (nt <= 0) return;
        a.assign(nt, 0.0);
        b.assign(nt, 1.0);
        plain(solver, t0, t1, h, a.data());
        time_vector(solver, t0, t1, h, b.data());
        ++cases;
        if (std::memcmp(a.data(), b.data(), sizeof(double) * nt) != 0) {
            ++bad;
            std::printf("mismatch solver=%d t0=%.17g h=%.17g T=%ld\n", solver, t0, h, T);
        }
    };
    for (double h : hs)
        for (double t0 : t0s)
            for (int solver = 0; solver < 2; ++solver) run(solver, t0, h, 300000);
    for (int r = 0; r < 400; ++r) {
        const double h = std::pow(10.0, -1.0 - 6.0 * std::fabs(U(rng)));
        const double t0 = U(rng) * std::pow(10.0, 3.0 * U(rng));
        run(r & 1, t0, h, 1 + (long)(rng() % 120000));
    }
    for (long T = 1; T < 40; ++T) run(0, 0.3, 0.1, T), run(1, -0.3, 0.1, T);
    std::printf("cases %d bad %d\n", cases, bad);
    return bad != 0;
}
"""


def test_time_vector_is_the_reference_accumulation(tmp_path):
    """The fast time vector equals the reference's float accumulation bit for bit."""
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    drv = tmp_path / "tv.cpp"
    drv.write_text(TIME_DRIVER)
    exe = tmp_path / "tv"
    subprocess.run([gxx, "-O3", "-std=c++17", "-I", CSRC, str(drv), os.path.join(CSRC, "host_math.cpp"), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout[-2000:]
    assert "bad 0" in out.stdout


CHAIN_DRIVER = r"""
#include "host_math.h"
#include <cstdio>
#include <vector>
using namespace parode;
int main()
{
    // (solver, t0, h, steps): one thread and several, ties of the float
    // rounding (h = 1.5 2^-12), a negative start, late starts, a tiny step
    struct C { int solver; double t0, h; long steps; };
    const C cs[] = {{0, 0.0, 1e-4, 1L << 20}, {1, 0.0, 1e-3, 300000}, {0, 0.5, 3e-5, 1500000},
                    {0, 0.0, 1.5 / 4096.0, 400000}, {0, -2.0, 1e-4, 300000}, {0, 1000.0, 1e-3, 300000},
                    {0, 0.0, 1e-7, 300000}, {1, 3.0, 0.1, 70000}, {0, 0.25, 1e-3, 1000}};
    for (const C& c : cs) {
        const double t1 = c.t0 + (double)(c.steps - 1) * c.h;
        long ns = 0;
        const long T = num_outputs(c.solver, c.t0, t1, c.h, &ns);
        std::vector<double> td((size_t)T), ref((size_t)T);
        std::vector<float> tf((size_t)T);
        time_vector(c.solver, c.t0, t1, c.h, td.data());
        time_vector_f(c.solver, c.t0, t1, c.h, tf.data());
        // the plain sequential chain
        const long pre = T - ns;
        const double ts = c.solver == 1 ? c.t0 + 3.0 * c.h : c.t0;
        for (long i = 0; i < pre; ++i) ref[i] = (double)(float)(ts - (double)(pre - i) * c.h);
        ref[pre] = (double)(float)ts;
        for (long i = pre; i + 1 < T; ++i) ref[i + 1] = (double)(float)(ref[i] + c.h);
        long bad = 0;
        for (long i = 0; i < T; ++i) bad += (td[i] != ref[i]) + ((double)tf[i] != ref[i]);
        std::printf("%ld %ld\n", T, bad);
    }
    return 0;
}
"""


def test_time_vector_is_the_sequential_float_chain(tmp_path):
    """time_vector / time_vector_f (speculated, and split over host threads
    from binade-predicted slice starts) equal the plain link-by-link float
    chain element for element."""
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    drv = tmp_path / "tv.cpp"
    drv.write_text(CHAIN_DRIVER)
    exe = tmp_path / "tv"
    subprocess.run([gxx, "-O2", "-std=c++17", "-ffp-contract=off", "-pthread", "-I", CSRC, str(drv),
                    os.path.join(CSRC, "host_math.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    rows = [tuple(int(v) for v in line.split()) for line in out.strip().splitlines()]
    assert len(rows) == 9
    for T, bad in rows:
        assert T > 0 and bad == 0, (T, bad)
