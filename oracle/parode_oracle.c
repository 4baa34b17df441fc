/*
 * parode_oracle.c -- CPU oracle for the ParODE LTI path (test infrastructure;
 * see parode_oracle.h for what each function restates and where).
 */
#include "parode_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* small dense helpers (row-major)                                      */
/* ------------------------------------------------------------------ */

static void mm_d(int r, int k, int c, const double* X, const double* Y, double* Z)
{
    for (int i = 0; i < r; ++i)
        for (int j = 0; j < c; ++j) {
            double s = 0.0;
            for (int q = 0; q < k; ++q) s += X[(long)i * k + q] * Y[(long)q * c + j];
            Z[(long)i * c + j] = s;
        }
}

/* uBLAS prod() on matrix<float>: sequential-k float accumulation. */
static void mm_f(int r, int k, int c, const float* X, const float* Y, float* Z)
{
    for (int i = 0; i < r; ++i)
        for (int j = 0; j < c; ++j) {
            float s = 0.0f;
            for (int q = 0; q < k; ++q) s += X[(long)i * k + q] * Y[(long)q * c + j];
            Z[(long)i * c + j] = s;
        }
}

static double* dalloc(long n) { return (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }
static float* falloc(long n) { return (float*)calloc((size_t)(n > 0 ? n : 1), sizeof(float)); }

double po_sinusoid_eval(double t, int i, void* ctx)
{
    const po_sinusoid* s = (const po_sinusoid*)ctx;
    double v = 0.0;
    const double two_pi = 6.283185307179586476925286766559;
    for (int k = 0; k < s->K; ++k) {
        long q = (long)i * s->K + k;
        v += s->a[q] * sin(two_pi * s->f[q] * t + s->phi[q]);
    }
    return v;
}

static double eval_u(const po_input* in, double t, int i)
{
    if (in == NULL || in->fn == NULL) return 0.0;
    if (in->float_time) return (double)(float)in->fn((double)(float)t, i, in->ctx);
    return in->fn(t, i, in->ctx);
}

/* ------------------------------------------------------------------ */
/* step counts, output size, time vector                                */
/* ------------------------------------------------------------------ */

long po_num_outputs(int solver, double t0, double tEnd, double h, long* n_scan)
{
    /* RK4: _nSteps = (unsigned long)((tEnd - tStart)/tStep) + 1
     *      (Sources/RungeKutta4thOrder.cpp:20).
     * ABM: tStart += 3*tStep; _nSteps as above; total = _nSteps + 3
     *      (Sources/AdamsMoulton.cpp:356-358).
     * A quotient at or below -1 would wrap the unsigned cast in the
     * reference; it is reported as an empty horizon here. */
    if (!(h > 0.0)) return -1;
    double ts = (solver == PO_ABM) ? t0 + 3.0 * h : t0;
    double q = (tEnd - ts) / h;
    if (!(q > -1.0) || q > 4.0e18) return -1;
    long ns = (long)q + 1;
    if (n_scan) *n_scan = ns;
    return (solver == PO_ABM) ? ns + 3 : ns;
}

int po_output_size(const po_system* s)
{
    /* _nOutputSize = max(C.size1(), D.size1()), or the state size when both
     * are absent (Sources/GPUFixedStepIterative.cpp:62-74,122-123). */
    if (s->zeroC && s->zeroD) return s->n;
    return s->p;
}

void po_time_vector(int solver, double t0, double tEnd, double h, float* tv)
{
    long ns = 0;
    long nt = po_num_outputs(solver, t0, tEnd, h, &ns);
    if (nt <= 0) return;
    long pre = nt - ns;
    double ts = (solver == PO_ABM) ? t0 + 3.0 * h : t0;
    /* Sources/GPUFixedStepIterative.cpp:141-146 (tVect is a float vector). */
    for (long i = 0; i < pre; ++i) tv[i] = (float)(ts - (double)(pre - i) * h);
    tv[pre] = (float)ts;
    for (long i = 1; i < ns; ++i) tv[pre + i] = (float)((double)tv[pre + i - 1] + h);
}

/* ------------------------------------------------------------------ */
/* FP64 discretisations                                                 */
/* ------------------------------------------------------------------ */

void po_rk4_discretise(int n, int m, const double* A, const double* B, double h,
                       double* Phi, double* Bbar)
{
    /* Sources/RungeKutta4thOrder.cpp:36-70:
     *   Abar = I + hA + h^2/2 A^2 + h^3/6 A^3 + h^4/24 A(A^3)
     *   B1 = 1/6 (hB + h^2 AB + 0.5 h^3 A^2B + 0.25 h^4 A^3B)
     *   B2 = 1/6 (4hB + 2h^2 AB + 0.5 h^3 A^2B)
     *   B3 = 1/6 hB,  Bbar = [B1 B2 B3] (n x 3m) */
    long nn = (long)n * n, nm = (long)n * m;
    double *A2 = dalloc(nn), *A3 = dalloc(nn), *A4 = dalloc(nn);
    double *AB = dalloc(nm), *A2B = dalloc(nm), *A3B = dalloc(nm);
    mm_d(n, n, n, A, A, A2);
    mm_d(n, n, n, A2, A, A3);
    mm_d(n, n, n, A, A3, A4);
    if (m > 0) {
        mm_d(n, n, m, A, B, AB);
        mm_d(n, n, m, A2, B, A2B);
        mm_d(n, n, m, A3, B, A3B);
    }
    double h2 = h * h, h3 = h * h * h, h4 = h * h * h * h;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            long q = (long)i * n + j;
            Phi[q] = (i == j ? 1.0 : 0.0) + h * A[q] + 0.5 * h2 * A2[q] + (1.0 / 6.0) * h3 * A3[q] +
                     (1.0 / 24.0) * h4 * A4[q];
        }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) {
            long q = (long)i * m + j;
            double b1 = (1.0 / 6.0) * (h * B[q] + h2 * AB[q] + 0.5 * h3 * A2B[q] + 0.25 * h4 * A3B[q]);
            double b2 = (1.0 / 6.0) * (4.0 * h * B[q] + 2.0 * h2 * AB[q] + 0.5 * h3 * A2B[q]);
            double b3 = (1.0 / 6.0) * h * B[q];
            Bbar[(long)i * 3 * m + j] = b1;
            Bbar[(long)i * 3 * m + m + j] = b2;
            Bbar[(long)i * 3 * m + 2 * m + j] = b3;
        }
    free(A2); free(A3); free(A4); free(AB); free(A2B); free(A3B);
}

void po_abm_discretise(int n, int m, const double* A, const double* B, double h,
                       double* Phi, double* Bbar)
{
    /* Sources/AdamsMoulton.cpp:238-316: AB4 predictor substituted into the AM4
     * corrector gives x_{k+4} = A3 x_k + A2 x_{k+1} + A1 x_{k+2} + A0 x_{k+3}
     *   + B3 u_k + B2 u_{k+1} + B1 u_{k+2} + B0 u_{k+3} + B-1 u_{k+4};
     * companion Abar = [0 I 0 0; 0 0 I 0; 0 0 0 I; A3 A2 A1 A0] (4n x 4n),
     * Bbar = [B3 B2 B1 B0 B-1] (n x 5m). */
    long nn = (long)n * n, nm = (long)n * m;
    int N = 4 * n;
    double *A2 = dalloc(nn), *AB = dalloc(nm);
    mm_d(n, n, n, A, A, A2);
    if (m > 0) mm_d(n, n, m, A, B, AB);
    double h2 = h * h;
    memset(Phi, 0, sizeof(double) * (size_t)N * N);
    for (int r = 0; r < n; ++r) {
        for (int c = 0; c < n; ++c) {
            long q = (long)r * n + c;
            double a0 = (r == c ? 1.0 : 0.0) + (28.0 * h / 24.0) * A[q] + (495.0 * h2 / 576.0) * A2[q];
            double a1 = (-5.0 * h / 24.0) * A[q] + (-531.0 * h2 / 576.0) * A2[q];
            double a2 = (1.0 * h / 24.0) * A[q] + (333.0 * h2 / 576.0) * A2[q];
            double a3 = (-81.0 * h2 / 576.0) * A2[q];
            long row = (long)(3 * n + r) * N;
            Phi[row + c] = a3;
            Phi[row + n + c] = a2;
            Phi[row + 2 * n + c] = a1;
            Phi[row + 3 * n + c] = a0;
        }
        Phi[(long)r * N + n + r] = 1.0;
        Phi[(long)(n + r) * N + 2 * n + r] = 1.0;
        Phi[(long)(2 * n + r) * N + 3 * n + r] = 1.0;
    }
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < m; ++c) {
            long q = (long)r * m + c;
            double bm1 = (9.0 * h / 24.0) * B[q];
            double b0 = (19.0 * h / 24.0) * B[q] + (495.0 * h2 / 576.0) * AB[q];
            double b1 = (-5.0 * h / 24.0) * B[q] + (-531.0 * h2 / 576.0) * AB[q];
            double b2 = (h / 24.0) * B[q] + (333.0 * h2 / 576.0) * AB[q];
            double b3 = (-81.0 * h2 / 576.0) * AB[q];
            long row = (long)r * 5 * m;
            Bbar[row + c] = b3;
            Bbar[row + m + c] = b2;
            Bbar[row + 2 * m + c] = b1;
            Bbar[row + 3 * m + c] = b0;
            Bbar[row + 4 * m + c] = bm1;
        }
    free(A2); free(AB);
}

/* ------------------------------------------------------------------ */
/* classical RK4 step on x' = A x + B u (FP64)                           */
/* ------------------------------------------------------------------ */

static void deriv_d(int n, int m, const double* A, const double* B, int zeroB, const double* x,
                    const double* u, double* dx)
{
    for (int r = 0; r < n; ++r) {
        double s = 0.0;
        for (int c = 0; c < n; ++c) s += A[(long)r * n + c] * x[c];
        if (!zeroB)
            for (int c = 0; c < m; ++c) s += B[(long)r * m + c] * u[c];
        dx[r] = s;
    }
}

/* One classical RK4 step with inputs u0 (t), uh (t+h/2), u1 (t+h). */
static void rk4_step_d(int n, int m, const double* A, const double* B, int zeroB, double* x,
                       const double* u0, const double* uh, const double* u1, double h, double* work)
{
    double *k1 = work, *k2 = work + n, *k3 = work + 2 * n, *k4 = work + 3 * n, *xt = work + 4 * n;
    deriv_d(n, m, A, B, zeroB, x, u0, k1);
    for (int i = 0; i < n; ++i) xt[i] = x[i] + 0.5 * h * k1[i];
    deriv_d(n, m, A, B, zeroB, xt, uh, k2);
    for (int i = 0; i < n; ++i) xt[i] = x[i] + 0.5 * h * k2[i];
    deriv_d(n, m, A, B, zeroB, xt, uh, k3);
    for (int i = 0; i < n; ++i) xt[i] = x[i] + h * k3[i];
    deriv_d(n, m, A, B, zeroB, xt, u1, k4);
    for (int i = 0; i < n; ++i)
        x[i] = x[i] + (h / 6.0) * k1[i] + (h / 3.0) * k2[i] + (h / 3.0) * k3[i] + (h / 6.0) * k4[i];
}

void po_abm_startup(const po_system* s, const po_input* in, double t0, double h, double* X0)
{
    /* Sources/AdamsMoulton.cpp:39-103: nine inputs at half steps
     * t0 + j h/2 (j = 0..8), three RK4 steps of size h whose stage inputs
     * are picked by index round(t/(h/2)). */
    int n = s->n, m = s->m;
    double* U = dalloc(9L * (m > 0 ? m : 1));
    for (int j = 0; j < 9; ++j)
        for (int i = 0; i < m; ++i) U[(long)j * m + i] = eval_u(in, t0 + (0.5 * h) * (double)j, i);
    double* x = dalloc(n);
    double* work = dalloc(5L * n);
    for (int r = 0; r < n; ++r) X0[r] = x[r] = s->x0[r];
    for (int st = 1; st < 4; ++st) {
        int j = 2 * (st - 1);
        rk4_step_d(n, m, s->A, s->B, s->zeroB, x, U + (long)j * m, U + (long)(j + 1) * m,
                   U + (long)(j + 2) * m, h, work);
        for (int r = 0; r < n; ++r) X0[(long)st * n + r] = x[r];
    }
    free(U); free(x); free(work);
}

/* y = C x + D u (or x when C and D are both absent). */
static void output_d(const po_system* s, const double* x, const double* u, double* y)
{
    int p = po_output_size(s);
    if (s->zeroC && s->zeroD) {
        for (int r = 0; r < p; ++r) y[r] = x[r];
        return;
    }
    for (int r = 0; r < p; ++r) {
        double v = 0.0;
        if (!s->zeroC)
            for (int c = 0; c < s->n; ++c) v += s->C[(long)r * s->n + c] * x[c];
        if (!s->zeroD)
            for (int c = 0; c < s->m; ++c) v += s->D[(long)r * s->m + c] * u[c];
        y[r] = v;
    }
}

/* ------------------------------------------------------------------ */
/* O1: FP64 sequential affine recurrence                                */
/* ------------------------------------------------------------------ */

int po_simulate_affine(const po_system* s, const po_input* in, int solver,
                       double t0, double tEnd, double h, double* y, long* n_out)
{
    if (s->n <= 0) return -6;
    if (solver != PO_RK4 && solver != PO_ABM) return -7;
    long ns = 0;
    long nt = po_num_outputs(solver, t0, tEnd, h, &ns);
    if (nt <= 0) return -6;
    if (n_out) *n_out = nt;
    int n = s->n, m = s->zeroB ? 0 : s->m, mu = s->m;
    int p = po_output_size(s);
    int N = (solver == PO_ABM) ? 4 * n : n;
    int W = (solver == PO_ABM) ? 5 : 3;
    double* Phi = dalloc((long)N * N);
    double* Bbar = dalloc((long)n * W * (m > 0 ? m : 1));
    if (solver == PO_RK4)
        po_rk4_discretise(n, m, s->A, s->B, h, Phi, Bbar);
    else
        po_abm_discretise(n, m, s->A, s->B, h, Phi, Bbar);
    double* X = dalloc(N);
    double* Xn = dalloc(N);
    double* win = dalloc((long)W * (mu > 0 ? mu : 1));
    double* uo = dalloc(mu > 0 ? mu : 1);
    if (solver == PO_RK4) {
        /* Gamma_k = Bbar [u(t_k); u(t_k + h/2); u(t_k + h)]; u sampled on the
         * half-step grid t0 + j (h/2) (Sources/RungeKutta4thOrder.cpp:255-285,
         * Kernels/BTimesURK4thOrder.cl:15-37); y_k = C x_k + D u_{2k}
         * (input stride 2, Sources/RungeKutta4thOrder.cpp:209). */
        const double dt = 0.5 * h;
        for (int r = 0; r < n; ++r) X[r] = s->x0[r];
        for (long k = 0; k < ns; ++k) {
            for (int q = 0; q < 3; ++q)
                for (int i = 0; i < mu; ++i) win[(long)q * mu + i] = eval_u(in, t0 + dt * (double)(2 * k + q), i);
            output_d(s, X, win, y + k * p);
            for (int r = 0; r < n; ++r) {
                double v = 0.0;
                for (int c = 0; c < n; ++c) v += Phi[(long)r * n + c] * X[c];
                double g = 0.0;
                for (int q = 0; q < 3 * m; ++q) g += Bbar[(long)r * 3 * m + q] * win[q];
                Xn[r] = v + g;
            }
            memcpy(X, Xn, sizeof(double) * n);
        }
    } else {
        /* X_0 = [x0; x1; x2; x3] from the RK4 start-up; outputs 0..2 from it
         * with u on the half-step grid (Sources/AdamsMoulton.cpp:106-116,
         * Sources/GPUFixedStepIterative.cpp:150-172).  The scan inputs sit on
         * the grid (t0 + 3h) - 3h + j h (Sources/AdamsMoulton.cpp:426-432);
         * output k+3 = C x_{k+3} + D u_{k+3} (strides 4/1, offsets 3/3,
         * Sources/AdamsMoulton.cpp:398). */
        po_abm_startup(s, in, t0, h, X);
        for (int i = 0; i < 3; ++i) {
            for (int c = 0; c < mu; ++c) uo[c] = eval_u(in, t0 + (0.5 * h) * (double)(2 * i), c);
            output_d(s, X + (long)i * n, uo, y + (long)i * p);
        }
        const double base = (t0 + 3.0 * h) - 3.0 * h;
        for (long k = 0; k < ns; ++k) {
            for (int q = 0; q < 5; ++q)
                for (int i = 0; i < mu; ++i) win[(long)q * mu + i] = eval_u(in, base + h * (double)(k + q), i);
            output_d(s, X + 3L * n, win + 3L * mu, y + (k + 3) * p);
            for (int r = 0; r < N; ++r) {
                double v = 0.0;
                /* rows 0..3n-1 of the companion matrix hold one 1.0 and zeros:
                 * the sum is exactly the shifted component, so the zero terms
                 * are skipped (bit-identical to the dense product) */
                if (r < 3 * n) {
                    Xn[r] = X[r + n];
                    continue;
                }
                for (int c = 0; c < N; ++c) v += Phi[(long)r * N + c] * X[c];
                if (r >= 3 * n) {
                    double g = 0.0;
                    for (int q = 0; q < 5 * m; ++q) {
                        int blk = q / (m > 0 ? m : 1), col = q % (m > 0 ? m : 1);
                        g += Bbar[(long)(r - 3 * n) * 5 * m + q] * win[(long)blk * mu + col];
                    }
                    v += g;
                }
                Xn[r] = v;
            }
            memcpy(X, Xn, sizeof(double) * N);
        }
    }
    free(Phi); free(Bbar); free(X); free(Xn); free(win); free(uo);
    return 0;
}

/* ------------------------------------------------------------------ */
/* O2: the reference tests' sequential loops                            */
/* ------------------------------------------------------------------ */

/* Derivative in float with float accumulation, as the tests' sys(). */
static void deriv_f(int n, int m, const float* A, const float* B, int zeroB, const float* x,
                    const float* u, float* dx)
{
    for (int r = 0; r < n; ++r) {
        float s = 0.0f;
        for (int c = 0; c < n; ++c) s += A[(long)r * n + c] * x[c];
        if (!zeroB)
            for (int c = 0; c < m; ++c) s += B[(long)r * m + c] * u[c];
        dx[r] = s;
    }
}

/* Generic-RK combination as odeint's scale_sum: double coefficients,
 * float storage. */
static void rk4_step_f(int n, int m, const float* A, const float* B, int zeroB, float* x,
                       const float* u0, const float* uh, const float* u1, double h, float* work)
{
    float *k1 = work, *k2 = work + n, *k3 = work + 2 * n, *k4 = work + 3 * n, *xt = work + 4 * n;
    deriv_f(n, m, A, B, zeroB, x, u0, k1);
    for (int i = 0; i < n; ++i) xt[i] = (float)((double)x[i] + 0.5 * h * (double)k1[i]);
    deriv_f(n, m, A, B, zeroB, xt, uh, k2);
    for (int i = 0; i < n; ++i) xt[i] = (float)((double)x[i] + 0.5 * h * (double)k2[i]);
    deriv_f(n, m, A, B, zeroB, xt, uh, k3);
    for (int i = 0; i < n; ++i) xt[i] = (float)((double)x[i] + h * (double)k3[i]);
    deriv_f(n, m, A, B, zeroB, xt, u1, k4);
    for (int i = 0; i < n; ++i)
        x[i] = (float)((double)x[i] + (h / 6.0) * k1[i] + (h / 3.0) * k2[i] + (h / 3.0) * k3[i] +
                       (h / 6.0) * k4[i]);
}

static void output_f(const po_system* s, const float* Cf, const float* Df, const float* x, const float* u,
                     double* y)
{
    int p = po_output_size(s);
    if (s->zeroC && s->zeroD) {
        for (int r = 0; r < p; ++r) y[r] = x[r];
        return;
    }
    for (int r = 0; r < p; ++r) {
        float v = 0.0f, w = 0.0f;
        if (!s->zeroC)
            for (int c = 0; c < s->n; ++c) v += Cf[(long)r * s->n + c] * x[c];
        if (!s->zeroD)
            for (int c = 0; c < s->m; ++c) w += Df[(long)r * s->m + c] * u[c];
        y[r] = (double)(v + w);
    }
}

typedef struct {
    int use_float;
    float *Af, *Bf, *Cf, *Df;
} fcopy;

static void make_fcopy(const po_system* s, fcopy* f)
{
    int n = s->n, m = s->m, p = s->p;
    f->Af = falloc((long)n * n);
    f->Bf = falloc((long)n * (m > 0 ? m : 1));
    f->Cf = falloc((long)(p > 0 ? p : 1) * n);
    f->Df = falloc((long)(p > 0 ? p : 1) * (m > 0 ? m : 1));
    for (long i = 0; i < (long)n * n; ++i) f->Af[i] = (float)s->A[i];
    if (!s->zeroB)
        for (long i = 0; i < (long)n * m; ++i) f->Bf[i] = (float)s->B[i];
    if (!s->zeroC)
        for (long i = 0; i < (long)p * n; ++i) f->Cf[i] = (float)s->C[i];
    if (!s->zeroD)
        for (long i = 0; i < (long)p * m; ++i) f->Df[i] = (float)s->D[i];
}

static void free_fcopy(fcopy* f) { free(f->Af); free(f->Bf); free(f->Cf); free(f->Df); }

int po_stepper_rk4(const po_system* s, const po_input* in, double t0, double h, long T, int use_float,
                   double* y)
{
    /* TestsSources/TestParODEStaticLibCInterface.cpp:158-204: x advanced by
     * odeint runge_kutta4 with u evaluated at the stage times, tDisc
     * accumulated in double, y_k = C x_k + D u(tDisc). */
    int n = s->n, m = s->m, p = po_output_size(s);
    if (n <= 0 || T <= 0) return -6;
    double tD = t0;
    if (!use_float) {
        double *x = dalloc(n), *work = dalloc(5L * n);
        double *u0 = dalloc(m + 1), *uh = dalloc(m + 1), *u1 = dalloc(m + 1);
        for (int r = 0; r < n; ++r) x[r] = s->x0[r];
        for (int i = 0; i < m; ++i) u0[i] = eval_u(in, tD, i);
        output_d(s, x, u0, y);
        for (long k = 1; k < T; ++k) {
            for (int i = 0; i < m; ++i) {
                u0[i] = eval_u(in, tD, i);
                uh[i] = eval_u(in, tD + 0.5 * h, i);
                u1[i] = eval_u(in, tD + h, i);
            }
            rk4_step_d(n, m, s->A, s->B, s->zeroB, x, u0, uh, u1, h, work);
            tD += h;
            for (int i = 0; i < m; ++i) u0[i] = eval_u(in, tD, i);
            output_d(s, x, u0, y + k * p);
        }
        free(x); free(work); free(u0); free(uh); free(u1);
    } else {
        fcopy f;
        make_fcopy(s, &f);
        float *x = falloc(n), *work = falloc(5L * n);
        float *u0 = falloc(m + 1), *uh = falloc(m + 1), *u1 = falloc(m + 1);
        for (int r = 0; r < n; ++r) x[r] = (float)s->x0[r];
        for (int i = 0; i < m; ++i) u0[i] = (float)eval_u(in, tD, i);
        output_f(s, f.Cf, f.Df, x, u0, y);
        for (long k = 1; k < T; ++k) {
            for (int i = 0; i < m; ++i) {
                u0[i] = (float)eval_u(in, tD, i);
                uh[i] = (float)eval_u(in, tD + 0.5 * h, i);
                u1[i] = (float)eval_u(in, tD + h, i);
            }
            rk4_step_f(n, m, f.Af, f.Bf, s->zeroB, x, u0, uh, u1, h, work);
            tD += h;
            for (int i = 0; i < m; ++i) u0[i] = (float)eval_u(in, tD, i);
            output_f(s, f.Cf, f.Df, x, u0, y + k * p);
        }
        free(x); free(work); free(u0); free(uh); free(u1);
        free_fcopy(&f);
    }
    return 0;
}

int po_stepper_abm(const po_system* s, const po_input* in, double t0, double h, long T, int use_float,
                   double* y)
{
    /* TestsSources/TestParODEStaticLibCInterface.cpp:336-466: three odeint
     * RK4 steps, then AB4 predictor (55,-59,37,-9)/24 and AM4 corrector
     * (9,19,-5,1)/24 with derivatives f(x_k, t_k). */
    int n = s->n, m = s->m, p = po_output_size(s);
    if (n <= 0 || T <= 0) return -6;
    const double ab[4] = {55.0 / 24.0, -59.0 / 24.0, 37.0 / 24.0, -9.0 / 24.0};
    const double am[4] = {9.0 / 24.0, 19.0 / 24.0, -5.0 / 24.0, 1.0 / 24.0};
    double tD = t0;
    if (!use_float) {
        double *x = dalloc(n), *work = dalloc(5L * n), *pr = dalloc(n), *fp = dalloc(n);
        double* f[4];
        for (int q = 0; q < 4; ++q) f[q] = dalloc(n); /* f[0] newest */
        double *u0 = dalloc(m + 1), *uh = dalloc(m + 1), *u1 = dalloc(m + 1);
        for (int r = 0; r < n; ++r) x[r] = s->x0[r];
        for (long k = 0; k < 4 && k < T; ++k) {
            for (int i = 0; i < m; ++i) u0[i] = eval_u(in, tD, i);
            output_d(s, x, u0, y + k * p);
            if (k < 3) {
                deriv_d(n, m, s->A, s->B, s->zeroB, x, u0, f[2 - k]);
                for (int i = 0; i < m; ++i) {
                    uh[i] = eval_u(in, tD + 0.5 * h, i);
                    u1[i] = eval_u(in, tD + h, i);
                }
                rk4_step_d(n, m, s->A, s->B, s->zeroB, x, u0, uh, u1, h, work);
                tD += h;
            }
        }
        /* f[2] = f(x0), f[1] = f(x1), f[0] = f(x2); x = x3 at tD = t3. */
        for (long k = 4; k < T; ++k) {
            double* old = f[3];
            f[3] = f[2]; f[2] = f[1]; f[1] = f[0]; f[0] = old;
            for (int i = 0; i < m; ++i) u0[i] = eval_u(in, tD, i);
            deriv_d(n, m, s->A, s->B, s->zeroB, x, u0, f[0]);
            for (int r = 0; r < n; ++r)
                pr[r] = x[r] + h * (ab[0] * f[0][r] + ab[1] * f[1][r] + ab[2] * f[2][r] + ab[3] * f[3][r]);
            tD += h;
            for (int i = 0; i < m; ++i) u0[i] = eval_u(in, tD, i);
            deriv_d(n, m, s->A, s->B, s->zeroB, pr, u0, fp);
            for (int r = 0; r < n; ++r)
                x[r] = x[r] + h * (am[0] * fp[r] + am[1] * f[0][r] + am[2] * f[1][r] + am[3] * f[2][r]);
            output_d(s, x, u0, y + k * p);
        }
        free(x); free(work); free(pr); free(fp);
        for (int q = 0; q < 4; ++q) free(f[q]);
        free(u0); free(uh); free(u1);
    } else {
        fcopy fc;
        make_fcopy(s, &fc);
        float *x = falloc(n), *work = falloc(5L * n), *pr = falloc(n), *fp = falloc(n);
        float* f[4];
        for (int q = 0; q < 4; ++q) f[q] = falloc(n);
        float *u0 = falloc(m + 1), *uh = falloc(m + 1), *u1 = falloc(m + 1);
        for (int r = 0; r < n; ++r) x[r] = (float)s->x0[r];
        for (long k = 0; k < 4 && k < T; ++k) {
            for (int i = 0; i < m; ++i) u0[i] = (float)eval_u(in, tD, i);
            output_f(s, fc.Cf, fc.Df, x, u0, y + k * p);
            if (k < 3) {
                deriv_f(n, m, fc.Af, fc.Bf, s->zeroB, x, u0, f[2 - k]);
                for (int i = 0; i < m; ++i) {
                    uh[i] = (float)eval_u(in, tD + 0.5 * h, i);
                    u1[i] = (float)eval_u(in, tD + h, i);
                }
                rk4_step_f(n, m, fc.Af, fc.Bf, s->zeroB, x, u0, uh, u1, h, work);
                tD += h;
            }
        }
        for (long k = 4; k < T; ++k) {
            float* old = f[3];
            f[3] = f[2]; f[2] = f[1]; f[1] = f[0]; f[0] = old;
            for (int i = 0; i < m; ++i) u0[i] = (float)eval_u(in, tD, i);
            deriv_f(n, m, fc.Af, fc.Bf, s->zeroB, x, u0, f[0]);
            for (int r = 0; r < n; ++r)
                pr[r] = (float)((double)x[r] +
                                h * (ab[0] * f[0][r] + ab[1] * f[1][r] + ab[2] * f[2][r] + ab[3] * f[3][r]));
            tD += h;
            for (int i = 0; i < m; ++i) u0[i] = (float)eval_u(in, tD, i);
            deriv_f(n, m, fc.Af, fc.Bf, s->zeroB, pr, u0, fp);
            for (int r = 0; r < n; ++r)
                x[r] = (float)((double)x[r] +
                               h * (am[0] * fp[r] + am[1] * f[0][r] + am[2] * f[1][r] + am[3] * f[2][r]));
            output_f(s, fc.Cf, fc.Df, x, u0, y + k * p);
        }
        free(x); free(work); free(pr); free(fp);
        for (int q = 0; q < 4; ++q) free(f[q]);
        free(u0); free(uh); free(u1);
        free_fcopy(&fc);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* O3: FP32 restatement of the reference scan pipeline                  */
/* ------------------------------------------------------------------ */

static long next_pow2(long v)
{
    long p = 1;
    while (p < v) p <<= 1;
    return p;
}

/* Work-group reduction of Kernels/MVVKernelScanUpsweep.cl:29-47: each lane
 * accumulates a strided column subset in float, then a halving tree. */
static float wg_dot(const float* row, const float* v, int len, int lanes, float* part)
{
    for (int l = 0; l < lanes; ++l) {
        float acc = 0.0f;
        for (int cs = 0; cs < len; cs += lanes)
            if (cs + l < len) acc += row[cs + l] * v[cs + l];
        part[l] = acc;
    }
    for (int st = lanes >> 1; st > 0; st >>= 1)
        for (int l = 0; l < st; ++l) part[l] += part[l + st];
    return part[0];
}

void po_ref_discretise_f32(const po_system* s, int solver, double h, float* Phi, float* Bb)
{
    /* float discretisation: uBLAS prod() in float, linear combinations
     * evaluated in double (double scalars) and stored to float
     * (Sources/RungeKutta4thOrder.cpp:36-70, Sources/AdamsMoulton.cpp:238-316). */
    int n = s->n, m = s->zeroB ? 0 : s->m;
    int N = (solver == PO_ABM) ? 4 * n : n;
    fcopy fc;
    make_fcopy(s, &fc);
    {
        long nn = (long)n * n, nm = (long)n * (m > 0 ? m : 1);
        float *A2 = falloc(nn), *A3 = falloc(nn), *A4 = falloc(nn);
        float *AB = falloc(nm), *A2B = falloc(nm), *A3B = falloc(nm);
        mm_f(n, n, n, fc.Af, fc.Af, A2);
        if (m > 0) mm_f(n, n, m, fc.Af, fc.Bf, AB);
        double h2 = h * h, h3 = h * h * h, h4 = h * h * h * h;
        if (solver == PO_RK4) {
            mm_f(n, n, n, A2, fc.Af, A3);
            mm_f(n, n, n, fc.Af, A3, A4);
            if (m > 0) { mm_f(n, n, m, A2, fc.Bf, A2B); mm_f(n, n, m, A3, fc.Bf, A3B); }
            for (long q = 0; q < nn; ++q) {
                int i = (int)(q / n), j = (int)(q % n);
                Phi[q] = (float)((i == j ? 1.0 : 0.0) + h * fc.Af[q] + 0.5 * h2 * A2[q] +
                                 (1.0 / 6.0) * h3 * A3[q] + (1.0 / 24.0) * h4 * A4[q]);
            }
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < m; ++j) {
                    long q = (long)i * m + j;
                    Bb[(long)i * 3 * m + j] = (float)((1.0 / 6.0) * (h * fc.Bf[q] + h2 * AB[q] +
                                                                     0.5 * h3 * A2B[q] + 0.25 * h4 * A3B[q]));
                    Bb[(long)i * 3 * m + m + j] =
                        (float)((1.0 / 6.0) * (4.0 * h * fc.Bf[q] + 2.0 * h2 * AB[q] + 0.5 * h3 * A2B[q]));
                    Bb[(long)i * 3 * m + 2 * m + j] = (float)((1.0 / 6.0) * h * fc.Bf[q]);
                }
        } else {
            memset(Phi, 0, sizeof(float) * (size_t)N * N);
            for (int r = 0; r < n; ++r) {
                for (int c = 0; c < n; ++c) {
                    long q = (long)r * n + c;
                    long row = (long)(3 * n + r) * N;
                    Phi[row + 3 * n + c] = (float)((r == c ? 1.0 : 0.0) + (28.0 * h / 24.0) * fc.Af[q] +
                                                   (495.0 * h2 / 576.0) * A2[q]);
                    Phi[row + 2 * n + c] = (float)((-5.0 * h / 24.0) * fc.Af[q] + (-531.0 * h2 / 576.0) * A2[q]);
                    Phi[row + n + c] = (float)((1.0 * h / 24.0) * fc.Af[q] + (333.0 * h2 / 576.0) * A2[q]);
                    Phi[row + c] = (float)((-81.0 * h2 / 576.0) * A2[q]);
                }
                Phi[(long)r * N + n + r] = 1.0f;
                Phi[(long)(n + r) * N + 2 * n + r] = 1.0f;
                Phi[(long)(2 * n + r) * N + 3 * n + r] = 1.0f;
            }
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < m; ++c) {
                    long q = (long)r * m + c, row = (long)r * 5 * m;
                    Bb[row + c] = (float)((-81.0 * h2 / 576.0) * AB[q]);
                    Bb[row + m + c] = (float)((h / 24.0) * fc.Bf[q] + (333.0 * h2 / 576.0) * AB[q]);
                    Bb[row + 2 * m + c] = (float)((-5.0 * h / 24.0) * fc.Bf[q] + (-531.0 * h2 / 576.0) * AB[q]);
                    Bb[row + 3 * m + c] = (float)((19.0 * h / 24.0) * fc.Bf[q] + (495.0 * h2 / 576.0) * AB[q]);
                    Bb[row + 4 * m + c] = (float)((9.0 * h / 24.0) * fc.Bf[q]);
                }
        }
        free(A2); free(A3); free(A4); free(AB); free(A2B); free(A3B);
    }
    free_fcopy(&fc);
}

void po_ref_abm_startup_f32(const po_system* s, double h, const float* U9, float* X0, float* ypre)
{
    /* x1..x3 by three float RK4 steps with the inputs U9 = u(t0 + j h/2),
     * j = 0..8 (Sources/AdamsMoulton.cpp:29-104); X0 = [x0; x1; x2; x3];
     * outputs 0..2 with float accumulation (Sources/GPUFixedStepIterative.cpp:155-171). */
    int n = s->n, m = s->zeroB ? 0 : s->m, mu = s->m, p = po_output_size(s);
    fcopy fc;
    make_fcopy(s, &fc);
    float *x = falloc(n), *work = falloc(5L * n);
    for (int r = 0; r < n; ++r) X0[r] = x[r] = (float)s->x0[r];
    for (int st = 1; st < 4; ++st) {
        int j = 2 * (st - 1);
        rk4_step_f(n, m, fc.Af, fc.Bf, s->zeroB, x, U9 + (long)j * mu, U9 + (long)(j + 1) * mu,
                   U9 + (long)(j + 2) * mu, h, work);
        for (int r = 0; r < n; ++r) X0[(long)st * n + r] = x[r];
    }
    for (int i = 0; i < 3; ++i) {
        if (s->zeroC && s->zeroD) {
            for (int r = 0; r < p; ++r) ypre[(long)i * p + r] = X0[(long)i * n + r];
        } else {
            for (int r = 0; r < p; ++r) {
                float v = 0.0f;
                if (!s->zeroC)
                    for (int c = 0; c < n; ++c) v += fc.Cf[(long)r * n + c] * X0[(long)i * n + c];
                if (!s->zeroD)
                    for (int c = 0; c < mu; ++c) v += fc.Df[(long)r * mu + c] * U9[(long)(2 * i) * mu + c];
                ypre[(long)i * p + r] = v;
            }
        }
    }
    free(x); free(work);
    free_fcopy(&fc);
}

int po_simulate_refscan_f32(const po_system* s, const po_input* in, int solver,
                            double t0, double tEnd, double h, long batch, float* y, long* n_out)
{
    if (s->n <= 0) return -6;
    if (solver != PO_RK4 && solver != PO_ABM) return -7;
    long ns = 0;
    long nt = po_num_outputs(solver, t0, tEnd, h, &ns);
    if (nt <= 0) return -6;
    if (n_out) *n_out = nt;
    int n = s->n, m = s->zeroB ? 0 : s->m, mu = s->m, p = po_output_size(s);
    int N = (solver == PO_ABM) ? 4 * n : n;
    int W = (solver == PO_ABM) ? 5 : 3;
    fcopy fc;
    make_fcopy(s, &fc);

    float* Phi = falloc((long)N * N);
    float* Bb = falloc((long)n * W * (m > 0 ? m : 1));
    po_ref_discretise_f32(s, solver, h, Phi, Bb);

    /* Work-group column widths: next power of two >= 3 m for RK4
     * (Sources/RungeKutta4thOrder.cpp:85), >= 4n for ABM
     * (Sources/AdamsMoulton.cpp:147). */
    int lanes = 1;
    if (solver == PO_RK4) { while (lanes < 3 * m) lanes <<= 1; }
    else { while (lanes < N) lanes <<= 1; }
    float* part = falloc(lanes);

    /* Initial scan vector and host-side outputs. */
    float* X0 = falloc(N);
    long pre = 0;
    if (solver == PO_RK4) {
        for (int r = 0; r < n; ++r) X0[r] = (float)s->x0[r];
    } else {
        /* float RK4 start-up at float sample times (Sources/AdamsMoulton.cpp:53-103) */
        float tsf = (float)t0, dtf = (float)(h / 2.0);
        float* U9 = falloc(9L * (mu + 1));
        for (int j = 0; j < 9; ++j)
            for (int i = 0; i < mu; ++i) U9[(long)j * mu + i] = (float)eval_u(in, (double)(tsf + dtf * (float)j), i);
        po_ref_abm_startup_f32(s, h, U9, X0, y);
        pre = 3;
        free(U9);
    }

    long NSB = batch > 0 ? batch : next_pow2(ns);
    double ts = (solver == PO_ABM) ? t0 + 3.0 * h : t0;
    /* accumulators (Sources/GPUFixedStepIterative.cpp:191-198) */
    float* accM = falloc((long)N * N);
    float* accV = falloc(N);
    for (int i = 0; i < N; ++i) { accV[i] = X0[i]; accM[(long)i * N + i] = 1.0f; }
    long nlev_max = 1;
    while ((1L << nlev_max) < NSB) ++nlev_max;
    /* power table in float: M at up-sweep level l of every node is Abar^(2^l)
     * computed as M[k] M[k-d] with sequential-k float sums
     * (Kernels/MMKernelScanUpsweep.cl:37-49); all nodes of a level are equal. */
    float** Pw = (float**)calloc((size_t)(nlev_max + 2), sizeof(float*));
    Pw[0] = falloc((long)N * N);
    memcpy(Pw[0], Phi, sizeof(float) * (size_t)N * N);
    for (long l = 1; l <= nlev_max; ++l) {
        Pw[l] = falloc((long)N * N);
        mm_f(N, N, N, Pw[l - 1], Pw[l - 1], Pw[l]);
    }
    float* V = falloc(NSB * N);
    float* tmp = falloc(N);
    float* tM = falloc((long)N * N);
    float* uw = falloc((long)(2 * NSB + 5) * (mu + 1));
    long gidx = pre;
    long done = 0;
    for (long nB = 0; done < ns; ++nB) {
        long left = ns - done;
        long steps = NSB;
        if (left <= NSB) steps = next_pow2(left);
        double tsb = ts + (double)(nB * NSB) * h;
        /* inputs in float time (Kernels/u.cl:7-10) */
        long nsmp;
        float tf, df;
        if (solver == PO_RK4) { tf = (float)tsb; df = (float)(h / 2.0); nsmp = 2 * steps + 1; }
        else { tf = (float)(tsb - 3.0 * h); df = (float)h; nsmp = steps + 4; }
        for (long j = 0; j < nsmp; ++j)
            for (int i = 0; i < mu; ++i) uw[j * mu + i] = (float)eval_u(in, (double)(tf + df * (float)j), i);
        /* forcing (Kernels/BTimesURK4thOrder.cl, Kernels/BTimesUAdamsMoulton.cl) */
        memset(V, 0, sizeof(float) * (size_t)steps * N);
        for (long k = 0; k < steps; ++k) {
            if (m == 0) continue;
            if (solver == PO_RK4) {
                for (int r = 0; r < n; ++r)
                    V[k * N + r] = wg_dot(Bb + (long)r * 3 * m, uw + 2 * k * mu, 3 * m, lanes, part);
            } else {
                for (int r = 0; r < n; ++r)
                    V[k * N + 3 * n + r] = wg_dot(Bb + (long)r * 5 * m, uw + k * mu, 5 * m, lanes, part);
            }
        }
        /* up-sweep (Kernels/MVVKernelScanUpsweep.cl:25-48) */
        int lev = 0;
        for (long d = 1; d < steps; d <<= 1, ++lev) {
            for (long k = 2 * d - 1; k < steps; k += 2 * d) {
                for (int r = 0; r < N; ++r)
                    tmp[r] = wg_dot(Pw[lev] + (long)r * N, V + (k - d) * N, N, lanes, part) + V[k * N + r];
                memcpy(V + k * N, tmp, sizeof(float) * N);
            }
        }
        /* host carry (Sources/GPUFixedStepIterative.cpp:300-333) */
        {
            float* rootM = Pw[lev];
            float* rootV = V + (steps - 1) * N;
            memcpy(tM, accM, sizeof(float) * (size_t)N * N);
            memcpy(tmp, accV, sizeof(float) * N);
            for (int r = 0; r < N; ++r)
                for (int c = 0; c < N; ++c) {
                    float acc = 0.0f;
                    for (int q = 0; q < N; ++q) acc += rootM[(long)r * N + q] * tM[(long)q * N + c];
                    accM[(long)r * N + c] = acc;
                }
            for (int r = 0; r < N; ++r) {
                float acc = 0.0f;
                for (int q = 0; q < N; ++q) acc += rootM[(long)r * N + q] * tmp[q];
                accV[r] = acc + rootV[r];
            }
            memcpy(rootV, tmp, sizeof(float) * N);
        }
        /* down-sweep (Kernels/MVVKernelScanDownsweep.cl:25-48,
         * Kernels/RootCopyKernelScanDownsweep.cl:11-19) */
        for (long d = steps / 2; d > 0; d >>= 1) {
            --lev;
            for (long k = 2 * d - 1; k < steps; k += 2 * d) {
                for (int r = 0; r < N; ++r)
                    tmp[r] = wg_dot(Pw[lev] + (long)r * N, V + k * N, N, lanes, part) + V[(k - d) * N + r];
                memcpy(V + (k - d) * N, V + k * N, sizeof(float) * N);
                memcpy(V + k * N, tmp, sizeof(float) * N);
            }
        }
        /* output (Kernels/SystemOutput.cl:28-59) with strides (1,0)/(2,0) for
         * RK4 and (4,3)/(1,3) for ABM */
        for (long k = 0; k < steps; ++k) {
            if (gidx + k >= nt) break;
            float* xs = V + k * N + (solver == PO_ABM ? 3L * n : 0);
            float* us = uw + (solver == PO_ABM ? (k + 3) * mu : 2 * k * mu);
            float* yo = y + (gidx + k) * p;
            if (s->zeroC && s->zeroD) {
                for (int r = 0; r < p; ++r) yo[r] = xs[r];
                continue;
            }
            for (int r = 0; r < p; ++r) {
                for (int l = 0; l < lanes; ++l) {
                    float acc = 0.0f;
                    if (!s->zeroC)
                        for (int cs = 0; cs < n; cs += lanes)
                            if (cs + l < n) acc += fc.Cf[(long)r * n + cs + l] * xs[cs + l];
                    if (!s->zeroD)
                        for (int cs = 0; cs < mu; cs += lanes)
                            if (cs + l < mu) acc += fc.Df[(long)r * mu + cs + l] * us[cs + l];
                    part[l] = acc;
                }
                for (int st = lanes >> 1; st > 0; st >>= 1)
                    for (int l = 0; l < st; ++l) part[l] += part[l + st];
                yo[r] = part[0];
            }
        }
        gidx += steps;
        done += (left <= NSB) ? left : NSB;
    }
    for (long l = 0; l <= nlev_max; ++l) free(Pw[l]);
    free(Pw); free(V); free(tmp); free(tM); free(uw); free(accM); free(accV); free(X0);
    free(part); free(Phi); free(Bb);
    free_fcopy(&fc);
    return 0;
}

/* ------------------------------------------------------------------ */

double po_rel_err(const double* y, const double* yref, long T, int p)
{
    double worst = 0.0;
    for (int j = 0; j < p; ++j) {
        double num = 0.0, den = 0.0;
        for (long k = 0; k < T; ++k) {
            double e = fabs(y[k * p + j] - yref[k * p + j]);
            double a = fabs(yref[k * p + j]);
            if (e > num || e != e) num = e;
            if (a > den) den = a;
        }
        double r = den > 0.0 ? num / den : num;
        if (r > worst || r != r) worst = r;
    }
    return worst;
}

int po_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int po_simulate_affine_many(int count, const po_system* s, const po_input* in, const int* solver,
                            const double* t0, const double* tEnd, const double* h, double* const* y)
{
    /* O1 of each system on its own (the systems are independent); the
     * largest systems first so that the threads finish together. */
    int worst = 0;
    long* order = (long*)malloc(sizeof(long) * (size_t)(count > 0 ? count : 1));
    double* cost = (double*)malloc(sizeof(double) * (size_t)(count > 0 ? count : 1));
    for (int i = 0; i < count; ++i) {
        long ns = 0;
        po_num_outputs(solver[i], t0[i], tEnd[i], h[i], &ns);
        double N = solver[i] == PO_ABM ? 4.0 * s[i].n : (double)s[i].n;
        cost[i] = (double)ns * N * (double)s[i].n;
        order[i] = i;
    }
    for (int i = 1; i < count; ++i) {
        long v = order[i];
        int j = i - 1;
        while (j >= 0 && cost[order[j]] < cost[v]) {
            order[j + 1] = order[j];
            --j;
        }
        order[j + 1] = v;
    }
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) reduction(min : worst)
#endif
    for (int q = 0; q < count; ++q) {
        long i = order[q];
        long n_out = 0;
        int rc = po_simulate_affine(&s[i], &in[i], solver[i], t0[i], tEnd[i], h[i], y[i], &n_out);
        if (rc < worst) worst = rc;
    }
    free(order);
    free(cost);
    return worst;
}
