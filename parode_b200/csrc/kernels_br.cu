// kernels_br.cu -- block response matrices of the blocked scan.
//
// Inside a block of B steps the leaf computes, from a zero state, the local
// states z_j (z_0 = 0, z_{j+1} = Phi z_j + Gamma_j), the local outputs
// y_j = Cext z_j + D u_j and the block aggregate z_B.  All of them are
// linear in the block's input samples (the reference's forcing
// Kernels/BTimesURK4thOrder.cl:15-37, BTimesUAdamsMoulton.cl:17-38 and output
// Kernels/SystemOutput.cl:28-59 composed with the zero-seeded in-block scan),
// so they are one matrix W per system,
//   rows [0, B p)        -> y_j[o] (row j p + o),
//   rows [B p, B p + NP) -> z_B,
//   columns [0, Kpad)    -> the block's sample window, sample s input i at s m + i
//                           (RK4: samples 2bB .. 2bB + 2B, ABM: bB .. bB + B + 3),
//   columns [Kpad, Kpad + NPstate) -> the block's initial state (its carry X_b),
// and the leaf becomes W times the windows of all blocks: one GEMM.  The
// aggregates (state-free part of rows [B p, B p + NP)) go to the carry
// hierarchy first; the outputs are then W's output rows times [window; X_b],
// which folds the fix-up C Phi^j X_b into the same GEMM.  The composition
// across blocks is unchanged, so the result is the blocked Blelloch scan's.
// W is built once per plan in FP64 by running the block recurrence on the
// basis of the window and state columns.
#include "common.h"
#include "kernels.h"

#include <algorithm>

namespace parode {

namespace {

constexpr int kCols = 32;       // window columns per CTA
constexpr int kThreads = 256;

// z (NP x kCols, row-major in shared memory): z <- Phi z + S_j, and the
// output rows of step j, for the CTA's columns [c0, c0 + kCols).
__global__ void __launch_bounds__(kThreads) k_block_response(const ResponseArgs* __restrict__ args)
{
    extern __shared__ double sm[];
    const ResponseArgs a = args[blockIdx.y];
    const int NP = a.NP, B = a.B, p = a.p, m = a.m, n = a.n;
    const int c0 = blockIdx.x * kCols;
    const int ld = a.Kpad + a.NPstate;  // window columns, then the block's initial-state columns
    if (c0 >= ld) return;
    const bool rk4 = a.solver == 0;
    const int W = rk4 ? 3 : 5;
    const int coff = rk4 ? 0 : 3 * n;  // forcing rows / output state block
    double* sPhi = sm;                            // NP x NP
    double* z = sPhi + (long)NP * NP;             // NP x kCols
    double* zn = z + (long)NP * kCols;
    double* sC = zn + (long)NP * kCols;           // p x NP
    for (int e = threadIdx.x; e < NP * NP; e += kThreads) sPhi[e] = a.Phi[e];
    for (int e = threadIdx.x; e < p * NP; e += kThreads) sC[e] = a.Cext[e];
    // z_0: zero on the window columns, the identity on the state columns
    for (int e = threadIdx.x; e < NP * kCols; e += kThreads) {
        const int r = e / kCols, col = c0 + (e - r * kCols);
        z[e] = (col >= a.Kpad && col - a.Kpad == r) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int j = 0; j < B; ++j) {
        // outputs of step j: Cext z_j + D u_j (u_j: sample 2j for RK4, j + 3 for ABM)
        const int su = rk4 ? 2 * j : j + 3;
        for (int e = threadIdx.x; e < p * kCols; e += kThreads) {
            const int o = e / kCols, c = e - o * kCols, col = c0 + c;
            if (col >= ld) continue;
            double v = 0.0;
            if (col < a.K || col >= a.Kpad) {
                for (int r = 0; r < NP; ++r) v = fma(sC[o * NP + r], z[r * kCols + c], v);
                if (col < a.K && !a.zeroD && m > 0 && col / m == su) v += a.D[(long)o * m + col % m];
            }
            a.Wm[(long)(j * p + o) * ld + col] = v;
        }
        // z_{j+1} = Phi z_j + S_j, S_j = the forcing of step j on the window
        for (int e = threadIdx.x; e < NP * kCols; e += kThreads) {
            const int r = e / kCols, c = e - r * kCols, col = c0 + c;
            double v = 0.0;
            for (int k = 0; k < NP; ++k) v = fma(sPhi[r * NP + k], z[k * kCols + c], v);
            if (!a.zeroB && m > 0 && col < a.K && r >= coff && r < coff + n) {
                const int s = col / m, i = col - s * m;
                const int w = rk4 ? s - 2 * j : s - j;  // window slot of sample s at step j
                if (w >= 0 && w < W) v += a.Bbar[(long)(r - coff) * W * m + w * m + i];
            }
            zn[e] = v;
        }
        __syncthreads();
        double* t = z;
        z = zn;
        zn = t;
        __syncthreads();
    }
    // aggregate rows: z_B
    for (int e = threadIdx.x; e < NP * kCols; e += kThreads) {
        const int r = e / kCols, c = e - r * kCols, col = c0 + c;
        if (col < ld) a.Wm[(long)(B * p + r) * ld + col] = (col < a.K || col >= a.Kpad) ? z[e] : 0.0;
    }
}

}  // namespace

int response_window(int solver, int B, int m)
{
    return (solver == 0 ? 2 * B + 1 : B + 4) * m;
}

void launch_block_response(const ResponseArgs* dArgs, int nsys, int max_np, int max_p, int max_kpad, cudaStream_t s)
{
    if (nsys <= 0 || max_kpad <= 0) return;
    const size_t smem = ((size_t)max_np * max_np + 2 * (size_t)max_np * kCols + (size_t)max_p * max_np) * sizeof(double);
    if (smem > 220 * 1024) throw Error(kInvalidArgument, "block response: shared memory");
    PARODE_CUDA(cudaFuncSetAttribute(k_block_response, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((max_kpad + max_np + kCols - 1) / kCols), (unsigned)nsys);
    k_block_response<<<grid, kThreads, smem, s>>>(dArgs);
    PARODE_CUDA(cudaGetLastError());
}

}  // namespace parode
