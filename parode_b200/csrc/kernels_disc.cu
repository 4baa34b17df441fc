// kernels_disc.cu -- the batch's discretisation on the device: per system the
// RK4 Phi / Bbar (reference Sources/RungeKutta4thOrder.cpp:36-70) or the ABM
// companion map's last block row and Bbar (Sources/AdamsMoulton.cpp:238-316),
// and ||Phi - R||_inf over the stored rows (R the exact 0/1 part: I for RK4,
// the companion shift for ABM).
//
// One CTA per system.  Every product and sum is taken in the order of the
// host restatement (host_math.cpp: discretise_rk4, discretise_abm_last; its
// GEMM accumulates each element over the inner index in order, built without
// FMA contraction): explicit __dmul_rn / __dadd_rn keep the device from
// contracting, so the device gives the host's bits and the batch's layout
// (which the distance to R sizes) is the same either way.
#include "common.h"
#include "kernels.h"

#include <algorithm>

namespace parode {

namespace {

constexpr int kThreads = 256;

// Z (r x c) = X (r x k) Y (k x c), row-major, every element summed over the
// inner index in order; the CTA's threads split the elements.
__device__ void gemm_cta(int r, int k, int c, const double* __restrict__ X, const double* __restrict__ Y,
                         double* __restrict__ Z)
{
    for (int e = threadIdx.x; e < r * c; e += kThreads) {
        const int i = e / c, j = e - i * c;
        double s = 0.0;
        for (int q = 0; q < k; ++q) s = __dadd_rn(s, __dmul_rn(X[(long)i * k + q], Y[(long)q * c + j]));
        Z[e] = s;
    }
    __syncthreads();
}

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }

__global__ void __launch_bounds__(kThreads) k_discretise_batch(const DiscJob* __restrict__ jobs)
{
    const DiscJob jb = jobs[blockIdx.x];
    const int n = jb.n, m = jb.m, N = jb.solver == 0 ? n : 4 * n;
    const double h = jb.h, h2 = mul(h, h);
    const double* A = jb.A;
    const double* B = jb.B;
    double* A2 = jb.work;                  // n x n
    double* A3 = A2 + (long)n * n;         // n x n (RK4)
    double* A4 = A3 + (long)n * n;         // n x n (RK4)
    double* AB = A4 + (long)n * n;         // n x m
    double* A2B = AB + (long)n * std::max(m, 1);
    double* A3B = A2B + (long)n * std::max(m, 1);
    const int W = jb.solver == 0 ? 3 : 5;
    // Bbar starts at zero (the slots a system without B never fills)
    for (int e = threadIdx.x; e < n * W * std::max(m, 1); e += kThreads) jb.bbar[e] = 0.0;
    gemm_cta(n, n, n, A, A, A2);
    if (jb.solver == 0) {
        gemm_cta(n, n, n, A2, A, A3);
        gemm_cta(n, n, n, A, A3, A4);
        const double h3 = mul(mul(h, h), h), h4 = mul(mul(mul(h, h), h), h);
        const double c2 = mul(0.5, h2), c3 = mul(1.0 / 6.0, h3), c4 = mul(1.0 / 24.0, h4);
        for (int q = threadIdx.x; q < n * n; q += kThreads) {
            const int i = q / n, j = q - i * n;
            double v = add(i == j ? 1.0 : 0.0, mul(h, A[q]));
            v = add(v, mul(c2, A2[q]));
            v = add(v, mul(c3, A3[q]));
            jb.phi[q] = add(v, mul(c4, A4[q]));
        }
        if (m > 0) {
            gemm_cta(n, n, m, A, B, AB);
            gemm_cta(n, n, m, A2, B, A2B);
            gemm_cta(n, n, m, A3, B, A3B);
            const double b1 = mul(0.5, h3), b2 = mul(0.25, h4), b3 = mul(4.0, h), b4 = mul(2.0, h2);
            const double sixth = 1.0 / 6.0, b5 = mul(sixth, h);
            for (int q = threadIdx.x; q < n * m; q += kThreads) {
                const int i = q / m, j = q - i * m;
                double* row = jb.bbar + (long)i * 3 * m;
                const double u = add(add(add(mul(h, B[q]), mul(h2, AB[q])), mul(b1, A2B[q])), mul(b2, A3B[q]));
                row[j] = mul(sixth, u);
                row[m + j] = mul(sixth, add(add(mul(b3, B[q]), mul(b4, AB[q])), mul(b1, A2B[q])));
                row[2 * m + j] = mul(b5, B[q]);
            }
        }
    } else {
        // the companion map's last block row [A3 A2 A1 A0]
        const double k81 = -81.0 * h2 / 576.0, k333 = 333.0 * h2 / 576.0, k531 = -531.0 * h2 / 576.0,
                     k495 = 495.0 * h2 / 576.0;
        const double k1 = 1.0 * h / 24.0, k5 = -5.0 * h / 24.0, k28 = 28.0 * h / 24.0;
        for (int q = threadIdx.x; q < n * n; q += kThreads) {
            const int r = q / n, c = q - r * n;
            double* last = jb.phi + (long)r * N;
            last[c] = mul(k81, A2[q]);
            last[n + c] = add(mul(k1, A[q]), mul(k333, A2[q]));
            last[2 * n + c] = add(mul(k5, A[q]), mul(k531, A2[q]));
            last[3 * n + c] = add(add(r == c ? 1.0 : 0.0, mul(k28, A[q])), mul(k495, A2[q]));
        }
        if (m > 0) {
            gemm_cta(n, n, m, A, B, AB);
            const double kb1 = h / 24.0, kb19 = 19.0 * h / 24.0, kb9 = 9.0 * h / 24.0;
            for (int q = threadIdx.x; q < n * m; q += kThreads) {
                const int r = q / m, c = q - r * m;
                double* row = jb.bbar + (long)r * 5 * m;
                row[c] = mul(k81, AB[q]);
                row[m + c] = add(mul(kb1, B[q]), mul(k333, AB[q]));
                row[2 * m + c] = add(mul(k5, B[q]), mul(k531, AB[q]));
                row[3 * m + c] = add(mul(kb19, B[q]), mul(k495, AB[q]));
                row[4 * m + c] = mul(kb9, B[q]);
            }
        }
    }
    __syncthreads();
    // Bbar transposed (level-synchronous systems' coalesced forcing kernel)
    if (jb.bbarT) {
        const int Wm = W * m;
        for (int e = threadIdx.x; e < std::max(Wm, 1) * n; e += kThreads) jb.bbarT[e] = 0.0;
        __syncthreads();
        for (int e = threadIdx.x; e < n * Wm; e += kThreads) {
            const int r = e / Wm, c = e - r * Wm;
            jb.bbarT[(long)c * n + r] = jb.bbar[e];
        }
    }
    // ||Phi - R||_inf over the stored rows (each row summed in order)
    __shared__ double rowmax[kThreads];
    const int d0 = jb.solver == 0 ? 0 : 3 * n;
    double dmax = 0.0;
    for (int r = threadIdx.x; r < n; r += kThreads) {
        double sum = 0.0;
        for (int c = 0; c < N; ++c) sum = add(sum, fabs(add(jb.phi[(long)r * N + c], -(c == d0 + r ? 1.0 : 0.0))));
        dmax = std::max(dmax, sum);
    }
    rowmax[threadIdx.x] = dmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int t = 0; t < kThreads; ++t) v = std::max(v, rowmax[t]);
        *jb.delta = v;
    }
}

}  // namespace

long discretise_work_doubles(int n, int m) { return 3L * n * n + 3L * n * std::max(m, 1); }

void launch_discretise_batch(const DiscJob* jobs, int njobs, cudaStream_t s)
{
    for (int k = 0; k < njobs; k += 65535) {
        const int cnt = std::min(65535, njobs - k);
        k_discretise_batch<<<(unsigned)cnt, kThreads, 0, s>>>(jobs + k);
        PARODE_CUDA(cudaGetLastError());
    }
}

}  // namespace parode
