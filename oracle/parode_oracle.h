/*
 * parode_oracle.h -- CPU oracle for the ParODE parallel-in-time LTI path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: it is linked or
 * called only by tests/, by __graft_entry__.smoke() and by the cpu_baseline
 * leg of bench.py.  The product (libParODEShared.so) never calls it and has
 * no CPU fallback.
 *
 * It restates, on the CPU and in plain C, what apatriciu/ParODE computes for
 * SimulateODE (file:line citations are relative to the reference project):
 *
 *   O1  po_simulate_affine   FP64 sequential recurrence x_{k+1} = Phi x_k + Gamma_k,
 *                            y_k = C x_k + D u_k, with Phi / Bbar formed exactly as
 *                            Sources/RungeKutta4thOrder.cpp:36-70 and
 *                            Sources/AdamsMoulton.cpp:238-316, the ABM start-up of
 *                            Sources/AdamsMoulton.cpp:29-104, the output gather of
 *                            Sources/GPUFixedStepIterative.cpp:141-172,401-446 and
 *                            the input sample grid of Kernels/u.cl:6-11.
 *   O2  po_stepper_rk4 / po_stepper_abm
 *                            the reference tests' own CPU loops: classical RK4
 *                            (TestsSources/TestParODEStaticLibCInterface.cpp:158-204)
 *                            and the AB4/AM4 PECE loop (same file :336-466), in
 *                            float (as the reference) or double.
 *   O3  po_simulate_refscan_f32
 *                            the reference's own pipeline in FP32: uBLAS-style
 *                            float discretisation, ping-pong Blelloch up/down
 *                            sweep on (M, v) pairs with the matrix sweep kept
 *                            (Kernels/MMKernelScanUpsweep.cl:24-53,
 *                            Kernels/MVVKernelScanUpsweep.cl:25-48,
 *                            Kernels/MVVKernelScanDownsweep.cl:25-48,
 *                            Kernels/RootCopyKernelScanDownsweep.cl:11-19) and the
 *                            FP32 host carry between power-of-two time batches
 *                            (Sources/GPUFixedStepIterative.cpp:180-337).
 *
 * Parity pin: the reference ships no golden vectors.  Its tests pin results by
 * sqrt(sum err^2) < 0.1 against O2 on fixtures drawn from glibc rand() with the
 * default seed; tests/golden holds those fixtures and the check is repeated
 * against O1 and O3 in tests/test_oracle.py.
 */
#ifndef PARODE_ORACLE_H
#define PARODE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Solver ids, Include/ParODEEnums.h:11-14. */
enum { PO_RK4 = 0, PO_ABM = 1 };

/* Input function: returns u_i(t).  `ctx` is passed through unchanged. */
typedef double (*po_ufunc)(double t, int i, void* ctx);

/* Built-in sum-of-sinusoids input: u_i(t) = sum_k a[i*K+k] sin(2 pi f[i*K+k] t + phi[i*K+k]). */
typedef struct {
    int m;              /* number of inputs */
    int K;              /* terms per input  */
    const double* a;
    const double* f;
    const double* phi;
} po_sinusoid;

double po_sinusoid_eval(double t, int i, void* sinusoid_ctx);

/* Optional float semantics for the time argument of a user input function:
 * the reference evaluates UFunc(fType t, ...) with fType = float
 * (Kernels/u.cl:6-10).  When `float_time` is non-zero the oracle rounds t
 * to float before the call and the result to float after it. */
typedef struct {
    po_ufunc fn;
    void* ctx;
    int float_time;
} po_input;

/* A linear time-invariant system in row-major FP64.  A is n x n, B n x m,
 * C p x n, D p x m, x0 n.  zeroB/zeroC/zeroD mark absent matrices, as the
 * ZeroB/ZeroC/ZeroD flags of Include/ParODECInterface.h:61-79. */
typedef struct {
    int n, m, p;
    int zeroB, zeroC, zeroD;
    const double* A;
    const double* B;
    const double* C;
    const double* D;
    const double* x0;
} po_system;

/* Number of output samples of a solve, and the number of scan steps.
 * RK4: T = floor((tEnd - t0)/h) + 1      (Sources/RungeKutta4thOrder.cpp:20)
 * ABM: T' = floor((tEnd - (t0+3h))/h) + 1, total T'+3 (Sources/AdamsMoulton.cpp:356-358)
 * Returns the total number of outputs or -1 when the horizon is empty. */
long po_num_outputs(int solver, double t0, double tEnd, double h, long* n_scan);

/* Output count p (Sources/GPUFixedStepIterative.cpp:62-74,122-123). */
int po_output_size(const po_system* s);

/* Time vector in the reference's float semantics
 * (Sources/GPUFixedStepIterative.cpp:141-146). */
void po_time_vector(int solver, double t0, double tEnd, double h, float* tvect);

/* FP64 discretisations.  Phi is Ns x Ns (Ns = n for RK4, 4n for ABM),
 * Bbar is n x 3m (RK4) or n x 5m (ABM). */
void po_rk4_discretise(int n, int m, const double* A, const double* B, double h,
                       double* Phi, double* Bbar);
void po_abm_discretise(int n, int m, const double* A, const double* B, double h,
                       double* Phi, double* Bbar);

/* ABM start-up: three classical RK4 steps with inputs at half steps,
 * X0 = [x0; x1; x2; x3] (Sources/AdamsMoulton.cpp:29-104). */
void po_abm_startup(const po_system* s, const po_input* in, double t0, double h, double* X0);

/* O1: y is T x p (time-major, as xVect of Sources/GPUODESolver.cpp:36-42).
 * Returns 0 or a negative error (-6 invalid system, -7 invalid solver). */
int po_simulate_affine(const po_system* s, const po_input* in, int solver,
                       double t0, double tEnd, double h, double* y, long* n_out);

/* O2: the reference tests' sequential loops.  use_float selects FP32
 * arithmetic for the state and matrices (the tests' fType).  y has the same
 * layout as O1; for ABM entries 0..3 are filled from the start-up as the
 * GPU path reports them. */
int po_stepper_rk4(const po_system* s, const po_input* in, double t0, double h,
                   long T, int use_float, double* y);
int po_stepper_abm(const po_system* s, const po_input* in, double t0, double h,
                   long T, int use_float, double* y);

/* O3: FP32 restatement of the reference pipeline.  batch is the number of
 * scan steps per device batch (a power of two; 0 = one batch holding all). */
int po_simulate_refscan_f32(const po_system* s, const po_input* in, int solver,
                            double t0, double tEnd, double h, long batch,
                            float* y, long* n_out);

/* Relative error used by every parity check: per output channel j,
 * max_k |y - yref| / max_k |yref|; returns the maximum over channels. */
double po_rel_err(const double* y, const double* yref, long T, int p);

/* The float host-side set-up of the reference's solvers, shared by O3 and
 * the harness that runs the reference's own OpenCL kernels (ref_kernels.c):
 * Phi (N x N) and Bbar (n x W m) as uBLAS forms them in float
 * (Sources/RungeKutta4thOrder.cpp:36-70, Sources/AdamsMoulton.cpp:238-316),
 * and the ABM start-up from the nine input samples U9 = u(t0 + j h/2),
 * j = 0..8 (Sources/AdamsMoulton.cpp:29-116): X0 = [x0; x1; x2; x3] and the
 * outputs 0..2 (Sources/GPUFixedStepIterative.cpp:155-171). */
void po_ref_discretise_f32(const po_system* s, int solver, double h, float* Phi, float* Bbar);
void po_ref_abm_startup_f32(const po_system* s, double h, const float* U9, float* X0, float* ypre);

/* Thread-parallel O1 over independent systems (OpenMP when compiled with it). */
int po_threads(void);

/* O1 (po_simulate_affine) of `count` independent systems, spread over the
 * OpenMP threads; y[i] receives system i's outputs.  Input functions must be
 * callable from several threads at once (the built-in sinusoid is).  Returns
 * 0, or the most negative error code of any system. */
int po_simulate_affine_many(int count, const po_system* s, const po_input* in, const int* solver,
                            const double* t0, const double* tEnd, const double* h, double* const* y);

#ifdef __cplusplus
}
#endif

#endif
