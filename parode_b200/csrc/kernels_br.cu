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
#include "device_common.cuh"
#include "kernels.h"

#include <algorithm>

namespace parode {

namespace {

constexpr int kCols = 8;        // window columns per CTA (a cfg2 W: 41 CTAs)
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
                // four independent partial sums (NP is a multiple of 8)
                double v4[4] = {0.0, 0.0, 0.0, 0.0};
                for (int r = 0; r < NP; r += 4)
#pragma unroll
                    for (int q = 0; q < 4; ++q) v4[q] = fma(sC[o * NP + r + q], z[(r + q) * kCols + c], v4[q]);
                v = (v4[0] + v4[1]) + (v4[2] + v4[3]);
                if (col < a.K && !a.zeroD && m > 0 && col / m == su) v += a.D[(long)o * m + col % m];
            }
            a.Wm[(long)(j * p + o) * ld + col] = v;
        }
        // z_{j+1} = Phi z_j + S_j, S_j = the forcing of step j on the window
        for (int e = threadIdx.x; e < NP * kCols; e += kThreads) {
            const int r = e / kCols, c = e - r * kCols, col = c0 + c;
            double v4[4] = {0.0, 0.0, 0.0, 0.0};
            for (int k = 0; k < NP; k += 4)
#pragma unroll
                for (int q = 0; q < 4; ++q) v4[q] = fma(sPhi[r * NP + k + q], z[(k + q) * kCols + c], v4[q]);
            double v = (v4[0] + v4[1]) + (v4[2] + v4[3]);
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

// The same recurrence for one system with NP <= 64 (a multiple of 8), its
// product Phi z on the FP64 tensor cores: warp w (< NP / 8) holds Phi's rows
// 8w .. 8w + 7 as DMMA A fragments in registers and forms those rows of
// z_{j+1} for the CTA's 8 columns (m8n8k4 over K = NP, four partial chains),
// the forcing S_j as the accumulators' start; z sits in shared memory with a
// 12-double row pitch (conflict-free B fragments).  The output rows stay as
// above.
template <int NP>
__global__ void __launch_bounds__(kThreads) k_block_response_mma(const ResponseArgs* __restrict__ args)
{
    extern __shared__ double sm[];
    constexpr int ZP = kCols + 4, MT = NP / 8, KS = NP / 4 < 4 ? NP / 4 : 4;
    const ResponseArgs a = args[blockIdx.y];
    const int B = a.B, p = a.p, m = a.m, n = a.n;
    const int c0 = blockIdx.x * kCols;
    const int ld = a.Kpad + a.NPstate;
    if (c0 >= ld) return;
    const bool rk4 = a.solver == 0;
    const int W = rk4 ? 3 : 5;
    const int coff = rk4 ? 0 : 3 * n;
    double* z = sm;             // NP x ZP
    double* zn = z + NP * ZP;   // NP x ZP
    double* sC = zn + NP * ZP;  // p x NP
    for (int e = threadIdx.x; e < p * NP; e += kThreads) sC[e] = a.Cext[e];
    // z_0: zero on the window columns, the identity on the state columns
    for (int e = threadIdx.x; e < NP * ZP; e += kThreads) {
        const int r = e / ZP, cc = e - r * ZP, col = c0 + cc;
        z[e] = (cc < kCols && col >= a.Kpad && col - a.Kpad == r) ? 1.0 : 0.0;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    double qa[NP / 4];
    if (warp < MT)
#pragma unroll
        for (int kk = 0; kk < NP / 4; ++kk) qa[kk] = a.Phi[(warp * 8 + g) * NP + 4 * kk + t];
    __syncthreads();
    for (int j = 0; j < B; ++j) {
        // outputs of step j: Cext z_j + D u_j (u_j: sample 2j for RK4, j + 3 for ABM)
        const int su = rk4 ? 2 * j : j + 3;
        for (int e = threadIdx.x; e < p * kCols; e += kThreads) {
            const int o = e / kCols, c = e - o * kCols, col = c0 + c;
            if (col >= ld) continue;
            double v = 0.0;
            if (col < a.K || col >= a.Kpad) {
                double v4[4] = {0.0, 0.0, 0.0, 0.0};
                for (int r = 0; r < NP; r += 4)
#pragma unroll
                    for (int q = 0; q < 4; ++q) v4[q] = fma(sC[o * NP + r + q], z[(r + q) * ZP + c], v4[q]);
                v = (v4[0] + v4[1]) + (v4[2] + v4[3]);
                if (col < a.K && !a.zeroD && m > 0 && col / m == su) v += a.D[(long)o * m + col % m];
            }
            a.Wm[(long)(j * p + o) * ld + col] = v;
        }
        // z_{j+1} = Phi z_j + S_j, S_j = the forcing of step j on the window
        if (warp < MT) {
            const int r = warp * 8 + g;
            double acc[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int col = c0 + 2 * t + e;
                double sv = 0.0;
                if (!a.zeroB && m > 0 && col < a.K && r >= coff && r < coff + n) {
                    const int sidx = col / m, i = col - sidx * m;
                    const int w = rk4 ? sidx - 2 * j : sidx - j;  // window slot of sample sidx at step j
                    if (w >= 0 && w < W) sv = a.Bbar[(long)(r - coff) * W * m + w * m + i];
                }
                acc[e] = sv;
            }
            double part[KS][2];
#pragma unroll
            for (int q = 0; q < KS; ++q) part[q][0] = part[q][1] = 0.0;
#pragma unroll
            for (int kk = 0; kk < NP / 4; ++kk)
                dmma_m8n8k4(part[kk % KS][0], part[kk % KS][1], qa[kk], z[(4 * kk + t) * ZP + g]);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                double v = acc[e];
#pragma unroll
                for (int q = 0; q < KS; ++q) v += part[q][e];
                zn[r * ZP + 2 * t + e] = v;
            }
        }
        __syncthreads();
        double* tz = z;
        z = zn;
        zn = tz;
    }
    // aggregate rows: z_B
    for (int e = threadIdx.x; e < NP * kCols; e += kThreads) {
        const int r = e / kCols, c = e - r * kCols, col = c0 + c;
        if (col < ld) a.Wm[(long)(B * p + r) * ld + col] = (col < a.K || col >= a.Kpad) ? z[r * ZP + c] : 0.0;
    }
}

template <int NP>
void block_response_mma_t(const ResponseArgs* dArgs, int max_p, int max_kpad, cudaStream_t s)
{
    const size_t smem = (2 * (size_t)NP * (kCols + 4) + (size_t)max_p * NP) * sizeof(double);
    if (smem > 220 * 1024) throw Error(kInvalidArgument, "block response: shared memory");
    PARODE_CUDA(cudaFuncSetAttribute(k_block_response_mma<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((max_kpad + NP + kCols - 1) / kCols), 1);
    k_block_response_mma<NP><<<grid, kThreads, smem, s>>>(dArgs);
    PARODE_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// W for any NP, many systems per launch.  By linearity
//   y_j   = sum_{i<j} Cext Phi^(j-1-i) S_i (+ D u_j),   z_B = sum_{i<B} Phi^(B-1-i) S_i,
// where S_i (the forcing of step i) is non-zero only on the n forcing rows
// coff .. coff + n and reads samples i..i+4 (ABM) or 2i..2i+2 (RK4) through
// the slots of Bbar.  So W needs only CP_k = Cext Phi^k (p x NP) and
// Q_k = Phi^k restricted to the forcing columns (NP x n), k < B, instead of
// B full NP x NP products.  Both tables double with the power table
// P_l = Phi^(2^l): CP_{k + 2^l} = CP_k P_l and Q_{k + 2^l} = P_l Q_k, one
// GEMM launch per l for all k < 2^l (response_doubling_args).  Then two
// GEMMs fold in the slots of Bbar (response_product_args):
//   MT[(L, o)][(w, c)] = (CP_L Bbar_w)[o][c],   NT[(r, L)][(w, c)] = (Q_L Bbar_w)[r][c],
// so every element of W is a sum of at most 5 table entries.
// ---------------------------------------------------------------------------

__host__ __device__ inline int resp_n2(const ResponseArgs& a) { return (a.n + 1) & ~1; }
__host__ __device__ inline int resp_wm2(const ResponseArgs& a) { return ((a.solver == 0 ? 3 : 5) * a.m + 1) & ~1; }

constexpr int kPerThread = 4;
constexpr int kPerCta = kThreads * kPerThread;

__device__ __forceinline__ int find_entry(const long* __restrict__ start, int nent, long t)
{
    int lo = 0, hi = nent - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// CP_0 = Cext, Q_0 = the identity's forcing columns (n2 = n rounded up to
// even columns, the last one zero when n is odd), and BbarE = Bbar in the
// forcing rows of an NP x WM2 zero matrix (WM2 = W m rounded up to even).
__global__ void __launch_bounds__(kThreads) k_response_init(const ResponseArgs* __restrict__ args,
                                                             const long* __restrict__ start, int nent)
{
    const int e = find_entry(start, nent, blockIdx.x);
    const ResponseArgs& a = args[e];
    const int NP = a.NP, p = a.p, n = a.n, n2 = resp_n2(a), wm2 = resp_wm2(a);
    const int Wm = (a.solver == 0 ? 3 : 5) * a.m;
    const int coff = a.solver == 0 ? 0 : 3 * n;
    const long ncp = (long)p * NP, nq = (long)NP * n2, ldq = (long)a.B * n2;
    const long total = ncp + nq + (long)NP * wm2;
    const long base = (blockIdx.x - start[e]) * (long)kPerCta + threadIdx.x;
    for (int t = 0; t < kPerThread; ++t) {
        const long idx = base + (long)t * kThreads;
        if (idx >= total) break;
        if (idx < ncp) {
            a.CPt[idx] = a.Cext[idx];
        } else if (idx < ncp + nq) {
            const long u = idx - ncp;
            const int r = (int)(u / n2), c = (int)(u - (long)r * n2);
            a.Qt[r * ldq + c] = (c < n && r == coff + c) ? 1.0 : 0.0;
        } else {
            const long u = idx - ncp - nq;
            const int r = (int)(u / wm2), c = (int)(u - (long)r * wm2);
            a.BbarE[u] = (!a.zeroB && r >= coff && r < coff + n && c < Wm) ? a.Bbar[(long)(r - coff) * Wm + c] : 0.0;
        }
    }
}

// Every element of W from the tables: sums over the steps i whose forcing
// reads the element's sample (slot w = s - 2i for RK4, s - i for ABM).
__global__ void __launch_bounds__(kThreads) k_response_fill(const ResponseArgs* __restrict__ args,
                                                             const long* __restrict__ start, int nent)
{
    const int e = find_entry(start, nent, blockIdx.x);
    const ResponseArgs& a = args[e];
    const int NP = a.NP, p = a.p, m = a.m, B = a.B, wm2 = resp_wm2(a);
    const bool rk4 = a.solver == 0;
    const long ld = a.Kpad + a.NPstate;
    const long total = ((long)B * p + NP) * ld;
    const long ncp = (long)p * NP;
    const long base = (blockIdx.x - start[e]) * (long)kPerCta + threadIdx.x;
    for (int t = 0; t < kPerThread; ++t) {
        const long idx = base + (long)t * kThreads;
        if (idx >= total) break;
        const long row = idx / ld;
        const int col = (int)(idx - row * ld);
        double v = 0.0;
        if (col < a.K) {
            const int s = col / m, c = col - s * m;
            const int ilo = rk4 ? (s - 1) / 2 : s - 4;  // (s - 2 + 1) / 2 rounds up for s >= 1
            const int ihi = rk4 ? s / 2 : s;
            if (row < (long)B * p) {
                const int j = (int)(row / p), o = (int)(row - (long)j * p);
                for (int i = max(ilo, 0); i <= min(ihi, j - 1); ++i) {
                    const int w = rk4 ? s - 2 * i : s - i;
                    v += a.MT[((long)(j - 1 - i) * p + o) * wm2 + w * m + c];
                }
                if (!a.zeroD && s == (rk4 ? 2 * j : j + 3)) v += a.D[(long)o * m + c];
            } else {
                const long r = row - (long)B * p;
                for (int i = max(ilo, 0); i <= min(ihi, B - 1); ++i) {
                    const int w = rk4 ? s - 2 * i : s - i;
                    v += a.NT[(r * B + (B - 1 - i)) * wm2 + w * m + c];
                }
            }
        } else if (col >= a.Kpad && row < (long)B * p) {
            // initial-state columns of the output rows: Cext Phi^j
            const int j = (int)(row / p), o = (int)(row - (long)j * p);
            v = a.CPt[(long)j * ncp + (long)o * NP + (col - a.Kpad)];
        }
        a.Wm[idx] = v;
    }
}

}  // namespace

int response_window(int solver, int B, int m)
{
    return (solver == 0 ? 2 * B + 1 : B + 4) * m;
}

long response_init_ctas(const ResponseArgs& a)
{
    const long total = (long)a.p * a.NP + (long)a.NP * resp_n2(a) + (long)a.NP * resp_wm2(a);
    return (total + kPerCta - 1) / kPerCta;
}

size_t response_workspace_doubles(const ResponseArgs& a)
{
    const size_t B = a.B, NP = a.NP, n2 = resp_n2(a), wm2 = resp_wm2(a);
    // CPt, Qt, BbarE, MT, NT
    return B * a.p * NP + NP * B * n2 + NP * wm2 + B * a.p * wm2 + NP * B * wm2;
}

void response_workspace_carve(ResponseArgs& a, double* ws)
{
    const size_t B = a.B, NP = a.NP, n2 = resp_n2(a), wm2 = resp_wm2(a);
    a.CPt = ws;
    a.Qt = a.CPt + B * a.p * NP;
    a.BbarE = a.Qt + NP * B * n2;
    a.MT = a.BbarE + NP * wm2;
    a.NT = a.MT + B * a.p * wm2;
}

void response_product_args(const ResponseArgs& a, LevelArgs out[2])
{
    const int wm2 = resp_wm2(a), n2 = resp_n2(a), coff = a.solver == 0 ? 0 : 3 * a.n;
    // MT = CPt (B p x NP) x BbarE (NP x WM2), the source N-contiguous
    LevelArgs mt;
    mt.P = a.CPt;
    mt.ldp = a.NP;
    mt.Np = a.NP;
    mt.M = a.B * a.p;
    mt.K = a.NP;
    mt.ncols = wm2;
    mt.src = a.BbarE;
    mt.src_gs = 1;
    mt.src_ks = wm2;
    mt.dst = a.MT;
    mt.dst_gs = 1;
    mt.dst_is = wm2;
    // NT = Qt as NP B rows (r, L) of n2 (row pitch n2) x the forcing rows of BbarE
    LevelArgs nt;
    nt.P = a.Qt;
    nt.ldp = n2;
    nt.Np = a.NP;
    nt.M = a.NP * a.B;
    nt.K = n2;
    nt.ncols = wm2;
    nt.src = a.BbarE + (long)coff * wm2;
    nt.src_gs = 1;
    nt.src_ks = wm2;
    nt.dst = a.NT;
    nt.dst_gs = 1;
    nt.dst_is = wm2;
    out[0] = mt;
    out[1] = nt;
}

long response_fill_ctas(const ResponseArgs& a)
{
    const long total = ((long)a.B * a.p + a.NP) * (a.Kpad + a.NPstate);
    return (total + kPerCta - 1) / kPerCta;
}

void launch_response_init(const ResponseArgs* dArgs, const long* dStart, int nent, long ctas, cudaStream_t s)
{
    if (nent <= 0 || ctas <= 0) return;
    if (ctas > 0x7fffffffL) throw Error(kInvalidArgument, "response tables: grid too large");
    k_response_init<<<(unsigned)ctas, kThreads, 0, s>>>(dArgs, dStart, nent);
    PARODE_CUDA(cudaGetLastError());
}

int response_doubling_args(const ResponseArgs& a, const double* P, int l, LevelArgs out[2])
{
    const int half = 1 << l;
    if (half >= a.B) return 0;
    const long NP = a.NP, n2 = resp_n2(a), ldq = (long)a.B * n2;
    const double* Pl = P + (long)l * NP * NP;
    // Q_{k + 2^l} = P_l Q_k, k < 2^l: the first 2^l n2 columns of Qt (row pitch
    // B n2) into the next 2^l n2; the source is N-contiguous
    LevelArgs q;
    q.P = Pl;
    q.ldp = NP;
    q.Np = a.NP;
    q.M = a.NP;
    q.K = a.NP;
    q.ncols = (long)half * n2;
    q.src = a.Qt;
    q.src_gs = 1;
    q.src_ks = ldq;
    q.dst = a.Qt + (long)half * n2;
    q.dst_gs = 1;
    q.dst_is = ldq;
    // CP_{k + 2^l} = CP_k P_l, k < 2^l: rows (k, o) of CPt are the MMA's rows,
    // P_l's columns its columns (result(c, (k, o)) = sum_r CP_k[o][r] P_l[r][c])
    LevelArgs c;
    c.P = a.CPt;
    c.ldp = NP;
    c.Np = a.NP;
    c.M = half * a.p;
    c.K = a.NP;
    c.ncols = NP;
    c.src = Pl;
    c.src_gs = 1;
    c.src_ks = NP;
    c.dst = a.CPt + (long)half * a.p * NP;
    c.dst_gs = 1;
    c.dst_is = NP;
    out[0] = q;
    out[1] = c;
    return 2;
}

void launch_response_fill(const ResponseArgs* dArgs, const long* dStart, int nent, long ctas, cudaStream_t s)
{
    if (nent <= 0 || ctas <= 0) return;
    if (ctas > 0x7fffffffL) throw Error(kInvalidArgument, "response fill: grid too large");
    k_response_fill<<<(unsigned)ctas, kThreads, 0, s>>>(dArgs, dStart, nent);
    PARODE_CUDA(cudaGetLastError());
}

int response_log2_block(int solver, int NP, int n, int m, int p, long nScan, double window_weight, double executions,
                        double* flops_per_step)
{
    // per block: aggregates 2 NP Kpad and the outputs' window part 2 B p Kpad
    // (scaled by window_weight: below 1 when they run on the tensor cores),
    // the outputs' state part 2 B p NP, and about 6 NP^2 for the
    // level-synchronous carry (up- and down-sweep, 4 NP^2, at a lower
    // efficiency than the GEMMs).  Per step on top: the FP64 build of W's
    // tables (C P^k and P^k restricted to the input columns for k < B, by
    // doubling, then their products with Bbar), spread over the steps of
    // `executions` solves (0: not counted)
    const double n2 = (double)(n + (n & 1));
    const int wm = (solver == 0 ? 3 : 5) * m;
    const double wm2 = (double)(wm + (wm & 1));
    const double per_build = executions > 0 ? 1.0 / ((double)nScan * executions) : 0.0;
    int best = 2;
    double best_cost = -1.0;
    for (int R = 2; R <= 7; ++R) {
        const long B = 1L << R;
        if (R > 2 && B / 2 >= nScan) break;
        const long K = response_window(solver, (int)B, m), Kp = (K + 1) & ~1L;
        const double wbytes = 8.0 * ((double)B * p + NP) * ((double)Kp + NP);
        if (R > 2 && wbytes > 256e6) break;
        const double build = 2.0 * B * ((double)NP * NP + wm2 * NP) * (p + n2);
        const double cost =
            (window_weight * (2.0 * NP * Kp + 2.0 * B * p * (double)Kp) + 2.0 * B * p * (double)NP + 6.0 * NP * NP) / B +
            build * per_build;
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = R;
        }
    }
    if (flops_per_step) *flops_per_step = best_cost;
    return best;
}

void launch_block_response(const ResponseArgs* dArgs, int nsys, int max_np, int max_p, int max_kpad, cudaStream_t s)
{
    if (nsys <= 0 || max_kpad <= 0) return;
    if (nsys == 1) {  // one system: its NP is max_np
        switch (max_np) {
        case 8: return block_response_mma_t<8>(dArgs, max_p, max_kpad, s);
        case 16: return block_response_mma_t<16>(dArgs, max_p, max_kpad, s);
        case 24: return block_response_mma_t<24>(dArgs, max_p, max_kpad, s);
        case 32: return block_response_mma_t<32>(dArgs, max_p, max_kpad, s);
        case 40: return block_response_mma_t<40>(dArgs, max_p, max_kpad, s);
        case 48: return block_response_mma_t<48>(dArgs, max_p, max_kpad, s);
        case 56: return block_response_mma_t<56>(dArgs, max_p, max_kpad, s);
        case 64: return block_response_mma_t<64>(dArgs, max_p, max_kpad, s);
        default: break;
        }
    }
    const size_t smem = ((size_t)max_np * max_np + 2 * (size_t)max_np * kCols + (size_t)max_p * max_np) * sizeof(double);
    if (smem > 220 * 1024) throw Error(kInvalidArgument, "block response: shared memory");
    PARODE_CUDA(cudaFuncSetAttribute(k_block_response, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((max_kpad + max_np + kCols - 1) / kCols), (unsigned)nsys);
    k_block_response<<<grid, kThreads, smem, s>>>(dArgs);
    PARODE_CUDA(cudaGetLastError());
}

}  // namespace parode
