// host_math.cpp -- host FP64 set-up of a solve (see host_math.h).
#include "host_math.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

namespace parode {

namespace {

// Z (r x c) = X (r x k) * Y (k x c), row-major.  The inner loop runs over
// contiguous columns, so it vectorises; each element still accumulates in
// the order q = 0, 1, ..., so every clone gives the same bits (no FMA
// contraction: this file is built with -ffp-contract=off).
#if defined(__GNUC__) && !defined(__clang__) && defined(__x86_64__) && !defined(__CUDACC__)
__attribute__((target_clones("avx2", "default")))
#endif
void gemm(int r, int k, int c, const double* X, const double* Y, double* Z)
{
    for (int i = 0; i < r; ++i) {
        double* z = Z + (long)i * c;
        for (int j = 0; j < c; ++j) z[j] = 0.0;
        for (int q = 0; q < k; ++q) {
            double x = X[(long)i * k + q];
            const double* y = Y + (long)q * c;
            for (int j = 0; j < c; ++j) z[j] += x * y[j];
        }
    }
}

void derivative(const SystemDesc& s, const double* x, const double* u, double* dx)
{
    for (int r = 0; r < s.n; ++r) {
        double v = 0.0;
        for (int c = 0; c < s.n; ++c) v += s.A[(long)r * s.n + c] * x[c];
        if (!s.zeroB)
            for (int c = 0; c < s.m; ++c) v += s.B[(long)r * s.m + c] * u[c];
        dx[r] = v;
    }
}

}  // namespace

long num_outputs(int solver, double t0, double tEnd, double h, long* n_scan)
{
    if (!(h > 0.0)) return -1;
    double ts = (solver == 1) ? t0 + 3.0 * h : t0;
    double q = (tEnd - ts) / h;
    if (!(q > -1.0) || q > 4.0e18) return -1;
    long ns = (long)q + 1;
    if (n_scan) *n_scan = ns;
    return solver == 1 ? ns + 3 : ns;
}

namespace {

// One link of the reference's time accumulation: the float time plus the
// double step, rounded back to float (Sources/GPUFixedStepIterative.cpp:141-146).
inline double time_link(double prev, double h) { return (double)(float)(prev + h); }

}  // namespace

// The chain in either storage type (every element is a float value, so the
// float form stores the same numbers; each link is checked in double on the
// stored values, so the speculation stays exact).
template <class T>
void time_chain_t(T* tv, long count, double h)
{
    // The chain tv[i+1] = time_link(tv[i]) is one dependent float round trip
    // per element (~5 ms for 2^20).  Within a binade of the float values it
    // advances by a constant increment, so it is filled by speculation and
    // checked link by link: from a checked element, the arithmetic progression
    // with the next increment is written for a block, every link of the block
    // is checked independently (no dependency between the checks), and the
    // first failing link, if any, is recomputed and the speculation restarts
    // after it.  Every element is therefore exactly the chain's.  A failure
    // near the start of a block (an increment that alternates, as at exact
    // rounding ties) switches to plain chaining for a stretch.
    constexpr long kBlock = 2048, kEarly = 16, kStretch = 256;
    long s = 0;
    while (s + 1 < count) {
        const double v = tv[s];
        const double d = time_link(v, h) - v;
        const long e = std::min(count - 1, s + kBlock);
        for (long j = s + 1; j <= e; ++j) tv[j] = (T)(v + (double)(j - s) * d);
        int ok = 1;
        for (long j = s; j < e; ++j) ok &= (time_link((double)tv[j], h) == (double)tv[j + 1]) ? 1 : 0;
        if (ok) {
            s = e;
            continue;
        }
        long j = s;
        while (time_link((double)tv[j], h) == (double)tv[j + 1]) ++j;
        tv[j + 1] = (T)time_link((double)tv[j], h);
        long next = j + 1;
        if (j - s < kEarly) {
            const long stop = std::min(count - 1, next + kStretch);
            for (; next < stop; ++next) tv[next + 1] = (T)time_link((double)tv[next], h);
        }
        s = next;
    }
}

// The same chain on several host threads, every element still exactly the
// chain's.  Within a float binade [2^e, 2^(e+1)) the link adds a constant
// (the step rounded to the binade's spacing; an exact tie would alternate),
// so a walk over the binades -- a few dozen links -- predicts the value at any
// index.  Each thread fills its slice from the predicted start by the checked
// speculation above; then the first link into every slice is checked in order
// and a slice whose start was mispredicted is filled again from the true one.
// Negative times (whose spacing shrinks towards zero) run on one thread.
template <class T>
void time_chain_par(T* tv, long count, double h)
{
    const unsigned hw = std::thread::hardware_concurrency();
    const int P = (int)std::min<unsigned>(std::max(1u, hw / 2), 8u);
    if (count < (1L << 16) || P <= 1 || !((double)tv[0] >= 0.0)) return time_chain_t<T>(tv, count, h);
    // binade runs: from index s the values are v + k d while below hi
    struct Run {
        long s;
        double v, d;
    };
    std::vector<Run> runs;
    long s = 0;
    double v = tv[0];
    while (s < count - 1 && runs.size() < 4096) {
        const double d = time_link(v, h) - v;
        runs.push_back({s, v, d});
        if (!(d > 0.0)) break;  // a step below the spacing: the chain stalls
        long k = 1;
        if (v > 0.0) {
            int e = 0;
            std::frexp(v, &e);
            const double hi = std::ldexp(1.0, e);  // v in [hi / 2, hi)
            k = std::max(1L, (long)((hi - v) / d));
            while (k > 1 && v + (double)k * d >= hi) --k;
            while (v + (double)(k + 1) * d < hi) ++k;
        }
        if (s + k >= count - 1) break;
        s += k + 1;
        v = time_link(v + (double)k * d, h);
    }
    auto predict = [&](long i) {
        const Run* r = &runs[0];
        for (const Run& q : runs)
            if (q.s <= i) r = &q;
        return r->v + (double)(i - r->s) * r->d;
    };
    std::vector<long> a(P + 1);
    for (int t = 0; t <= P; ++t) a[t] = count * t / P;
    std::vector<std::thread> th;
    for (int t = 1; t < P; ++t)
        th.emplace_back([&, t] {
            tv[a[t]] = (T)predict(a[t]);
            time_chain_t<T>(tv + a[t], a[t + 1] - a[t], h);
        });
    time_chain_t<T>(tv, a[1], h);
    for (auto& x : th) x.join();
    for (int t = 1; t < P; ++t) {
        const T want = (T)time_link((double)tv[a[t] - 1], h);
        if (tv[a[t]] == want) continue;
        tv[a[t]] = want;
        time_chain_t<T>(tv + a[t], a[t + 1] - a[t], h);
    }
}

void time_chain(double* tv, long count, double h) { time_chain_t<double>(tv, count, h); }

template <class T>
void time_vector_t(int solver, double t0, double tEnd, double h, T* tv)
{
    long ns = 0;
    long nt = num_outputs(solver, t0, tEnd, h, &ns);
    if (nt <= 0) return;
    long pre = nt - ns;
    double ts = (solver == 1) ? t0 + 3.0 * h : t0;
    for (long i = 0; i < pre; ++i) tv[i] = (T)(float)(ts - (double)(pre - i) * h);
    tv[pre] = (T)(float)ts;
    time_chain_par<T>(tv + pre, ns, h);
}

void time_vector(int solver, double t0, double tEnd, double h, double* tv) { time_vector_t<double>(solver, t0, tEnd, h, tv); }
void time_vector_f(int solver, double t0, double tEnd, double h, float* tv) { time_vector_t<float>(solver, t0, tEnd, h, tv); }

void discretise_rk4(int n, int m, const double* A, const double* B, double h, double* Phi, double* Bbar)
{
    // Abar = I + hA + h^2/2 A^2 + h^3/6 A^3 + h^4/24 A^4 and
    // Bbar = [B1 B2 B3] with the coefficients of the reference
    // (Sources/RungeKutta4thOrder.cpp:42-57).
    std::vector<double> A2((size_t)n * n), A3((size_t)n * n), A4((size_t)n * n);
    gemm(n, n, n, A, A, A2.data());
    gemm(n, n, n, A2.data(), A, A3.data());
    gemm(n, n, n, A, A3.data(), A4.data());
    const double h2 = h * h, h3 = h * h * h, h4 = h * h * h * h;
    for (long q = 0; q < (long)n * n; ++q) {
        int i = (int)(q / n), j = (int)(q % n);
        Phi[q] = (i == j ? 1.0 : 0.0) + h * A[q] + 0.5 * h2 * A2[q] + (1.0 / 6.0) * h3 * A3[q] +
                 (1.0 / 24.0) * h4 * A4[q];
    }
    if (m <= 0) return;
    std::vector<double> AB((size_t)n * m), A2B((size_t)n * m), A3B((size_t)n * m);
    gemm(n, n, m, A, B, AB.data());
    gemm(n, n, m, A2.data(), B, A2B.data());
    gemm(n, n, m, A3.data(), B, A3B.data());
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) {
            long q = (long)i * m + j;
            double* row = Bbar + (long)i * 3 * m;
            row[j] = (1.0 / 6.0) * (h * B[q] + h2 * AB[q] + 0.5 * h3 * A2B[q] + 0.25 * h4 * A3B[q]);
            row[m + j] = (1.0 / 6.0) * (4.0 * h * B[q] + 2.0 * h2 * AB[q] + 0.5 * h3 * A2B[q]);
            row[2 * m + j] = (1.0 / 6.0) * h * B[q];
        }
}

void discretise_abm(int n, int m, const double* A, const double* B, double h, double* Phi, double* Bbar)
{
    // Companion map of the linear AB4-predictor / AM4-corrector step
    // (reference Sources/AdamsMoulton.cpp:253-316): the shift rows, then the
    // last block row.
    const int N = 4 * n;
    std::memset(Phi, 0, sizeof(double) * (size_t)N * N);
    for (int r = 0; r < n; ++r) {
        Phi[(long)r * N + n + r] = 1.0;
        Phi[(long)(n + r) * N + 2 * n + r] = 1.0;
        Phi[(long)(2 * n + r) * N + 3 * n + r] = 1.0;
    }
    discretise_abm_last(n, m, A, B, h, Phi + (long)3 * n * N, Bbar);
}

void discretise_abm_last(int n, int m, const double* A, const double* B, double h, double* lastRows, double* Bbar)
{
    // coefficients of the AB4 predictor folded into the AM4 corrector
    // (reference Sources/AdamsMoulton.cpp:253-316)
    const int N = 4 * n;
    std::vector<double> A2((size_t)n * n);
    gemm(n, n, n, A, A, A2.data());
    const double h2 = h * h;
    for (int r = 0; r < n; ++r) {
        double* last = lastRows + (long)r * N;
        for (int c = 0; c < n; ++c) {
            long q = (long)r * n + c;
            last[c] = (-81.0 * h2 / 576.0) * A2[q];
            last[n + c] = (1.0 * h / 24.0) * A[q] + (333.0 * h2 / 576.0) * A2[q];
            last[2 * n + c] = (-5.0 * h / 24.0) * A[q] + (-531.0 * h2 / 576.0) * A2[q];
            last[3 * n + c] = (r == c ? 1.0 : 0.0) + (28.0 * h / 24.0) * A[q] + (495.0 * h2 / 576.0) * A2[q];
        }
    }
    if (m <= 0) return;
    std::vector<double> AB((size_t)n * m);
    gemm(n, n, m, A, B, AB.data());
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < m; ++c) {
            long q = (long)r * m + c;
            double* row = Bbar + (long)r * 5 * m;
            row[c] = (-81.0 * h2 / 576.0) * AB[q];
            row[m + c] = (h / 24.0) * B[q] + (333.0 * h2 / 576.0) * AB[q];
            row[2 * m + c] = (-5.0 * h / 24.0) * B[q] + (-531.0 * h2 / 576.0) * AB[q];
            row[3 * m + c] = (19.0 * h / 24.0) * B[q] + (495.0 * h2 / 576.0) * AB[q];
            row[4 * m + c] = (9.0 * h / 24.0) * B[q];
        }
}

void abm_startup(const SystemDesc& s, const double* U9, double h, double* X0)
{
    const int n = s.n, m = s.m;
    std::vector<double> x(s.x0), k1(n), k2(n), k3(n), k4(n), xt(n);
    for (int r = 0; r < n; ++r) X0[r] = x[r];
    for (int st = 1; st < 4; ++st) {
        const double* u0 = U9 + (long)(2 * st - 2) * m;
        const double* uh = U9 + (long)(2 * st - 1) * m;
        const double* u1 = U9 + (long)(2 * st) * m;
        derivative(s, x.data(), u0, k1.data());
        for (int i = 0; i < n; ++i) xt[i] = x[i] + 0.5 * h * k1[i];
        derivative(s, xt.data(), uh, k2.data());
        for (int i = 0; i < n; ++i) xt[i] = x[i] + 0.5 * h * k2[i];
        derivative(s, xt.data(), uh, k3.data());
        for (int i = 0; i < n; ++i) xt[i] = x[i] + h * k3[i];
        derivative(s, xt.data(), u1, k4.data());
        for (int i = 0; i < n; ++i)
            x[i] = x[i] + (h / 6.0) * k1[i] + (h / 3.0) * k2[i] + (h / 3.0) * k3[i] + (h / 6.0) * k4[i];
        for (int r = 0; r < n; ++r) X0[(long)st * n + r] = x[r];
    }
}

}  // namespace parode
