// kernels_blocked.cu -- FP64 kernels of the blocked Blelloch scan (see blocked.h).
//
// Reference correspondence (apatriciu/ParODE): the leaf kernel fuses the
// u-kernel (Kernels/u.cl), the forcing (Kernels/BTimesURK4thOrder.cl,
// BTimesUAdamsMoulton.cl), the lowest R levels of the vector up/down sweep
// (Kernels/MVVKernelScanUpsweep.cl, MVVKernelScanDownsweep.cl,
// RootCopyKernelScanDownsweep.cl, LeftLeafCopyKernelScanUpsweep.cl) and the
// output (Kernels/SystemOutput.cl).  The matrix sweep is the power table
// (every up-sweep matrix at level l is Phi^(2^l) for an LTI system) and the
// per-batch host carry (Sources/GPUFixedStepIterative.cpp:296-337) becomes
// the device-side scan over block aggregates.
//
// Shared-memory layout: every vector / matrix row holds NP doubles whose
// 32-byte chunks are XOR-swizzled by a fold of the row index, so the eight
// rows an m8n8k4 fragment touches (consecutive rows, or rows 2^l apart) fall
// into distinct bank groups.
#include "blocked.h"
#include "common.h"
#include "device_common.cuh"

#include <algorithm>
#include <vector>

namespace parode {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int fold(int r) { return r ^ (r >> 2) ^ (r >> 4) ^ (r >> 6) ^ (r >> 8) ^ (r >> 10) ^ (r >> 12); }

template <int NP>
__device__ __forceinline__ int sidx(int r, int k)
{
    constexpr int NCH = NP / 4;
    constexpr int MASK = NCH >= 4 ? 3 : NCH - 1;
    return r * NP + ((((k >> 2) ^ (fold(r) & MASK))) << 2) + (k & 3);
}

// Row-major global NP x NP matrix -> swizzled shared copy.
template <int NP>
__device__ void load_matrix(double* dst, const double* __restrict__ src)
{
    for (int e = threadIdx.x; e < NP * NP; e += kThreads) {
        int r = e / NP, k = e - r * NP;
        dst[sidx<NP>(r, k)] = src[e];
    }
}

// Warp-level FP64 MMA with NJ x KS independent accumulator chains: for
// j < NJ fragment columns, acc[j] = sum over `ksteps` k-steps of
// A(step) * B(j, step); k-steps are dealt round-robin to KS partial sums that
// are added at the end.  B200's DMMA pipe needs about eight chains per warp
// in flight to stay busy, so callers pick NJ * KS = 8 whenever they can.
template <int NJ, int KS, class LA, class LB>
__device__ __forceinline__ void warp_mma(double (&acc)[NJ][2], const int ksteps, LA la, LB lb)
{
    double c[KS][NJ][2];
#pragma unroll
    for (int q = 0; q < KS; ++q)
#pragma unroll
        for (int j = 0; j < NJ; ++j) c[q][j][0] = c[q][j][1] = 0.0;
#pragma unroll
    for (int s = 0; s < ksteps; s += KS) {
#pragma unroll
        for (int q = 0; q < KS; ++q) {
            if (s + q < ksteps) {
                const double a = la(s + q);
#pragma unroll
                for (int j = 0; j < NJ; ++j) dmma_m8n8k4(c[q][j][0], c[q][j][1], a, lb(j, s + q));
            }
        }
    }
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
        acc[j][0] = c[0][j][0];
        acc[j][1] = c[0][j][1];
#pragma unroll
        for (int q = 1; q < KS; ++q) {
            acc[j][0] += c[q][j][0];
            acc[j][1] += c[q][j][1];
        }
    }
}

// One Blelloch level on the vectors of a tile: for g < c,
//   V[right(g)] += P V[left(g)],  right(g) = (g+1) 2d - 1,  left(g) = right(g) - d.
// Warps split the NP/8 fragment rows; each warp walks its fragment columns
// NJ at a time.
template <int NP, int NJ, int KS>
__device__ void level_gemm_t(const double* __restrict__ sP, double* sV, int c, int d)
{
    constexpr int RF = NP / 8;
    constexpr int NWC = 8 / RF;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wr = warp % RF, wc = warp / RF;
    const int gq = lane >> 2, tq = lane & 3;
    const int cf = (c + 7) >> 3;
    const int row = wr * 8 + gq;
    const int two_d = 2 * d;
    for (int cb0 = wc; cb0 < cf; cb0 += NWC * NJ) {
        int lB[NJ];
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
            const int gb = (cb0 + j * NWC) * 8 + gq;
            lB[j] = (cb0 + j * NWC < cf && gb < c) ? (gb + 1) * two_d - 1 - d : -1;
        }
        // per-row swizzled bases: element k of row r sits at
        // r*NP + (((k>>2) ^ f(r)) << 2) + (k&3); with k = 4s + tq and s a
        // compile-time constant the XOR only touches the low bits of s
        constexpr int MASK = (NP / 4) >= 4 ? 3 : (NP / 4) - 1;
        const int fa = fold(row) & MASK;
        int fb[NJ];
#pragma unroll
        for (int j = 0; j < NJ; ++j) fb[j] = lB[j] >= 0 ? (fold(lB[j]) & MASK) : 0;
        double acc[NJ][2];
        warp_mma<NJ, KS>(
            acc, NP / 4, [&](int s) { return sP[row * NP + ((s ^ fa) << 2) + tq]; },
            [&](int j, int s) { return lB[j] >= 0 ? sV[lB[j] * NP + ((s ^ fb[j]) << 2) + tq] : 0.0; });
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
            const int cb = cb0 + j * NWC;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int g = cb * 8 + 2 * tq + e;
                if (cb < cf && g < c) {
                    const int idx = sidx<NP>((g + 1) * two_d - 1, row);
                    sV[idx] = acc[j][e] + sV[idx];
                }
            }
        }
    }
}

template <int NP>
__device__ void level_gemm(const double* __restrict__ sP, double* sV, int c, int d)
{
    constexpr int NWC = 8 / (NP / 8);
    constexpr int KSM = NP / 4 < 8 ? NP / 4 : 8;
    const int njw = (((c + 7) >> 3) + NWC - 1) / NWC;  // fragment columns per warp
    if (njw >= 8) level_gemm_t<NP, 8, 1>(sP, sV, c, d);
    else if (njw >= 4) level_gemm_t<NP, 4, (KSM < 2 ? KSM : 2)>(sP, sV, c, d);
    else if (njw >= 2) level_gemm_t<NP, 2, (KSM < 4 ? KSM : 4)>(sP, sV, c, d);
    else level_gemm_t<NP, 1, KSM>(sP, sV, c, d);
}

// Down-sweep bookkeeping of a level: V[left(g)] <-> V[right(g)].  After it,
// level_gemm completes v[right] = P v[parent] + v[left aggregate].
template <int NP>
__device__ void level_swap(double* sV, int c, int d)
{
    for (int e = threadIdx.x; e < c * NP; e += kThreads) {
        int g = e / NP, i = e - g * NP;
        int r = (g + 1) * 2 * d - 1, l = r - d;
        int ir = sidx<NP>(r, i), il = sidx<NP>(l, i);
        double t = sV[ir];
        sV[ir] = sV[il];
        sV[il] = t;
    }
}

// ---------------------------------------------------------------------------
// leaf kernel
// ---------------------------------------------------------------------------

// Shared-memory regions of the leaf: R power-table levels, the tile's vectors,
// its input samples (su_doubles) and, when a.stage is set, Bbar | C | D.
template <int NP>
struct LeafSmem {
    double* sP;
    double* sV;
    double* sU;
    const double* pB;
    const double* pC;
    const double* pD;
};

// Per-system set-up of the leaf: power-table levels (and Bbar / C / D when
// staged) into shared memory.  Ends with the staged data visible to the CTA
// only after the caller's next __syncthreads (every tile starts with one).
template <int NP>
__device__ LeafSmem<NP> leaf_setup(const LeafArgs& a, double* sm, int R, int S, long su_doubles)
{
    LeafSmem<NP> L;
    L.sP = sm;
    L.sV = L.sP + (long)R * NP * NP;
    L.sU = L.sV + (long)S * NP;
    const int m = a.m, n = a.n, p = a.p;
    const int Wm = (a.solver == 0 ? 3 : 5) * m;
    for (int l = 0; l < R; ++l) load_matrix<NP>(L.sP + (long)l * NP * NP, a.P + (long)l * NP * NP);
    L.pB = a.Bbar;
    L.pC = a.C;
    L.pD = a.D;
    if (a.stage) {
        double* sM = L.sU + su_doubles;
        // Bbar is n x W m only when B is present (it is never read otherwise)
        const long nb = a.zeroB ? 0 : (long)n * Wm, nc = (long)p * n, nd = (long)p * m;
        for (long e = threadIdx.x; e < nb; e += kThreads) sM[e] = a.Bbar[e];
        for (long e = threadIdx.x; e < nc; e += kThreads) sM[nb + e] = a.zeroC ? 0.0 : a.C[e];
        for (long e = threadIdx.x; e < nd; e += kThreads) sM[nb + nc + e] = a.zeroD ? 0.0 : a.D[e];
        L.pB = sM;
        L.pC = sM + nb;
        L.pD = sM + nb + nc;
    }
    return L;
}

template <int NP>
__device__ void leaf_tile(const LeafArgs& a, const LeafSmem<NP>& L, long tile, int R, int S);

template <int NP>
__global__ void __launch_bounds__(kThreads, 1) k_leaf(LeafArgs a, int R, int S)
{
    extern __shared__ double sm[];
    const long su = (long)(a.solver == 0 ? 2 * S + 1 : S + 4) * (a.m > 0 ? a.m : 1);
    const LeafSmem<NP> L = leaf_setup<NP>(a, sm, R, S, su);
    for (long tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) leaf_tile<NP>(a, L, tile, R, S);
}

// Batched leaf: work items (system, tile range), dealt round-robin to the
// CTAs in the order given (largest first).
template <int NP>
__global__ void __launch_bounds__(kThreads, 1) k_leaf_batch(const LeafArgs* __restrict__ sys,
                                                            const BatchItem* __restrict__ items, int nitems, int R,
                                                            int S, int ms)
{
    extern __shared__ double sm[];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const BatchItem w = items[it];
        const LeafArgs a = sys[w.sys];
        __syncthreads();  // the previous item's tiles are done with shared memory
        const LeafSmem<NP> L = leaf_setup<NP>(a, sm, R, S, (long)(2 * S + 1) * (ms > 0 ? ms : 1));
        for (long tile = w.t0; tile < w.t1; ++tile) leaf_tile<NP>(a, L, tile, R, S);
    }
}

template <int NP>
__device__ void leaf_tile(const LeafArgs& a, const LeafSmem<NP>& L, long tile, int R, int S)
{
    double* sV = L.sV;
    double* sU = L.sU;
    const double* sP = L.sP;
    const double* pB = L.pB;
    const double* pC = L.pC;
    const double* pD = L.pD;
    const int B = 1 << R;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gq = lane >> 2, tq = lane & 3;
    const int m = a.m, n = a.n, p = a.p;
    const bool rk4 = a.solver == 0;
    const int W = rk4 ? 3 : 5;
    const int Wm = W * m;
    const int mB = a.zeroB ? 0 : m;
    const int nsamp = rk4 ? 2 * S + 1 : S + 4;
    const int coff = rk4 ? 0 : 3 * n;  // forcing rows / output state block
    const long nU = rk4 ? 2 * a.nScan + 1 : a.nScan + 4;
    {
        const long j0 = tile * S;
        const long js0 = rk4 ? 2 * j0 : j0;
        // 1. input samples of the tile (u-kernel of the reference)
        if (m > 0) {
            for (int e = tid; e < nsamp * m; e += kThreads) {
                int jl = e / m, i = e - jl * m;
                long js = js0 + jl;
                double v = 0.0;
                if (a.gen)
                    v = sinusoid_value(a.sa, a.sf, a.sphi, a.K, i, sample_time(a.u_base, a.u_dt, js));
                else if (js < nU)
                    v = a.U[js * m + i];
                sU[e] = v;
            }
        }
        for (int e = tid; e < S * NP; e += kThreads) sV[e] = 0.0;
        __syncthreads();

        // 2. forcing Gamma = Bbar [u windows] (DMMA, K = W m)
        if (mB > 0) {
            constexpr int NJ = 8;
            const int nrf = (n + 7) >> 3;
            const int nch = (S >> 3) / NJ;  // column chunks of NJ fragments
            const int ksteps = (Wm + 3) >> 2;
            for (int f = warp; f < nrf * nch; f += 8) {
                const int rb = f % nrf, ch = f / nrf;
                const int i = rb * 8 + gq;
                const double* brow = pB + (long)i * Wm;
                double acc[NJ][2];
                warp_mma<NJ, 1>(
                    acc, ksteps,
                    [&](int s) {
                        const int q = 4 * s + tq;
                        return (i < n && q < Wm) ? brow[q] : 0.0;
                    },
                    [&](int j, int s) {
                        const int q = 4 * s + tq;
                        const int jb = (ch * NJ + j) * 8 + gq;
                        return q < Wm ? sU[(rk4 ? 2 * jb : jb) * m + q] : 0.0;
                    });
                if (i < n) {
#pragma unroll
                    for (int j = 0; j < NJ; ++j) {
                        const int jc = (ch * NJ + j) * 8 + 2 * tq;
                        if (j0 + jc < a.nScan) sV[sidx<NP>(jc, coff + i)] = acc[j][0];
                        if (j0 + jc + 1 < a.nScan) sV[sidx<NP>(jc + 1, coff + i)] = acc[j][1];
                    }
                }
            }
        }
        __syncthreads();

        // 3. up-sweep of every block of the tile
        for (int l = 0; l < R; ++l) {
            level_gemm<NP>(sP + (long)l * NP * NP, sV, S >> (l + 1), 1 << l);
            __syncthreads();
        }
        // 4. block aggregates out, zero roots
        for (int e = tid; e < (S / B) * NP; e += kThreads) {
            int b = e / NP, i = e - b * NP;
            int r = sidx<NP>(b * B + B - 1, i);
            a.G[(tile * (S / B) + b) * NP + i] = sV[r];
            sV[r] = 0.0;
        }
        __syncthreads();
        // 5. down-sweep from the zero root
        for (int l = R - 1; l >= 0; --l) {
            level_swap<NP>(sV, S >> (l + 1), 1 << l);
            __syncthreads();
            if (l < R - 1) {
                level_gemm<NP>(sP + (long)l * NP * NP, sV, S >> (l + 1), 1 << l);
                __syncthreads();
            }
        }
        // 6. y_local = C z + D u (DMMA); y = x when C and D are absent
        {
            if (a.zeroC && a.zeroD) {
                for (int e = tid; e < S * p; e += kThreads) {
                    int jl = e / p, o = e - jl * p;
                    if (j0 + jl < a.nScan) a.Y[(a.ybase + j0 + jl) * p + o] = sV[sidx<NP>(jl, coff + o)];
                }
            } else {
                constexpr int NJ = 2, KS = 4;
                const int prf = (p + 7) >> 3;
                const int nch = (S >> 3) / NJ;
                const int mD = a.zeroD ? 0 : m;
                const int nC = a.zeroC ? 0 : n;
                const int ksC = (nC + 3) >> 2, ksD = (mD + 3) >> 2;
                for (int f = warp; f < prf * nch; f += 8) {
                    const int rb = f % prf, ch = f / prf;
                    const int o = rb * 8 + gq;
                    double acc[NJ][2];
                    warp_mma<NJ, KS>(
                        acc, ksC + ksD,
                        [&](int s) {
                            if (s < ksC) {
                                const int q = 4 * s + tq;
                                return (o < p && q < nC) ? pC[(long)o * n + q] : 0.0;
                            }
                            const int q = 4 * (s - ksC) + tq;
                            return (o < p && q < mD) ? pD[(long)o * m + q] : 0.0;
                        },
                        [&](int j, int s) {
                            const int jb = (ch * NJ + j) * 8 + gq;
                            if (s < ksC) {
                                const int q = 4 * s + tq;
                                return q < nC ? sV[sidx<NP>(jb, coff + q)] : 0.0;
                            }
                            const int q = 4 * (s - ksC) + tq;
                            return q < mD ? sU[(rk4 ? 2 * jb : jb + 3) * m + q] : 0.0;
                        });
                    if (o < p) {
#pragma unroll
                        for (int j = 0; j < NJ; ++j) {
                            const long jc = j0 + (ch * NJ + j) * 8 + 2 * tq;
                            if (jc < a.nScan) a.Y[(a.ybase + jc) * p + o] = acc[j][0];
                            if (jc + 1 < a.nScan) a.Y[(a.ybase + jc + 1) * p + o] = acc[j][1];
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// carry kernels over items (block aggregates), FP64
// ---------------------------------------------------------------------------

template <int NP>
__global__ void __launch_bounds__(kThreads, 1) k_items_up(double* items, long count, const double* P, int R, int S,
                                                          double* next)
{
    extern __shared__ double sm[];
    double* sP = sm;
    double* sV = sP + (long)R * NP * NP;
    const int B = 1 << R;
    for (int l = 0; l < R; ++l) load_matrix<NP>(sP + (long)l * NP * NP, P + (long)l * NP * NP);
    const long ntiles = (count + S - 1) / S;
    const long nnext = (count + B - 1) / B;
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long i0 = tile * S;
        for (int e = threadIdx.x; e < S * NP; e += kThreads) {
            int r = e / NP, k = e - r * NP;
            sV[sidx<NP>(r, k)] = (i0 + r < count) ? items[(i0 + r) * NP + k] : 0.0;
        }
        __syncthreads();
        for (int l = 0; l < R; ++l) {
            level_gemm<NP>(sP + (long)l * NP * NP, sV, S >> (l + 1), 1 << l);
            __syncthreads();
        }
        for (int e = threadIdx.x; e < S * NP; e += kThreads) {
            int r = e / NP, k = e - r * NP;
            if (i0 + r < count) items[(i0 + r) * NP + k] = sV[sidx<NP>(r, k)];
        }
        for (int e = threadIdx.x; e < (S / B) * NP; e += kThreads) {
            int b = e / NP, k = e - b * NP;
            long q = tile * (S / B) + b;
            if (q < nnext) next[q * NP + k] = sV[sidx<NP>(b * B + B - 1, k)];
        }
        __syncthreads();
    }
}

template <int NP>
__global__ void __launch_bounds__(kThreads, 1) k_items_down(double* items, long count, const double* P, int R, int S,
                                                            const double* carries)
{
    extern __shared__ double sm[];
    double* sP = sm;
    double* sV = sP + (long)R * NP * NP;
    const int B = 1 << R;
    for (int l = 0; l < R; ++l) load_matrix<NP>(sP + (long)l * NP * NP, P + (long)l * NP * NP);
    const long ntiles = (count + S - 1) / S;
    const long nnext = (count + B - 1) / B;
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long i0 = tile * S;
        for (int e = threadIdx.x; e < S * NP; e += kThreads) {
            int r = e / NP, k = e - r * NP;
            sV[sidx<NP>(r, k)] = (i0 + r < count) ? items[(i0 + r) * NP + k] : 0.0;
        }
        __syncthreads();
        // block roots take the block's exclusive prefix (the carry)
        for (int e = threadIdx.x; e < (S / B) * NP; e += kThreads) {
            int b = e / NP, k = e - b * NP;
            long q = tile * (S / B) + b;
            sV[sidx<NP>(b * B + B - 1, k)] = q < nnext ? carries[q * NP + k] : 0.0;
        }
        __syncthreads();
        for (int l = R - 1; l >= 0; --l) {
            level_swap<NP>(sV, S >> (l + 1), 1 << l);
            __syncthreads();
            level_gemm<NP>(sP + (long)l * NP * NP, sV, S >> (l + 1), 1 << l);
            __syncthreads();
        }
        for (int e = threadIdx.x; e < S * NP; e += kThreads) {
            int r = e / NP, k = e - r * NP;
            if (i0 + r < count) items[(i0 + r) * NP + k] = sV[sidx<NP>(r, k)];
        }
        __syncthreads();
    }
}

// Top of the hierarchy: one CTA, all levels of a power-of-two tile of L
// items, root seeded with the initial state.  P levels are staged one at a
// time.
template <int NP>
__global__ void __launch_bounds__(kThreads, 1) k_items_top(double* items, long count, const double* P, int L,
                                                           const double* X0)
{
    extern __shared__ double sm[];
    double* sP = sm;
    double* sV = sP + NP * NP;
    int levels = 0;
    while ((1 << levels) < L) ++levels;
    for (int e = threadIdx.x; e < L * NP; e += kThreads) {
        int r = e / NP, k = e - r * NP;
        sV[sidx<NP>(r, k)] = (r < count) ? items[(long)r * NP + k] : 0.0;
    }
    __syncthreads();
    for (int l = 0; l < levels; ++l) {
        load_matrix<NP>(sP, P + (long)l * NP * NP);
        __syncthreads();
        level_gemm<NP>(sP, sV, L >> (l + 1), 1 << l);
        __syncthreads();
    }
    for (int k = threadIdx.x; k < NP; k += kThreads) sV[sidx<NP>(L - 1, k)] = X0[k];
    __syncthreads();
    for (int l = levels - 1; l >= 0; --l) {
        load_matrix<NP>(sP, P + (long)l * NP * NP);
        level_swap<NP>(sV, L >> (l + 1), 1 << l);
        __syncthreads();
        level_gemm<NP>(sP, sV, L >> (l + 1), 1 << l);
        __syncthreads();
    }
    for (int e = threadIdx.x; e < L * NP; e += kThreads) {
        int r = e / NP, k = e - r * NP;
        if (r < count) items[(long)r * NP + k] = sV[sidx<NP>(r, k)];
    }
}

// y[(ybase + j) p + o] += CP[j mod B][o] . X[j div B] as a DMMA GEMM with
// M = B p (rows (jj, o), contiguous in y per block), K = NP, N = blocks.
template <int NP>
__device__ void fixup_body(double* Y, long ybase, long nScan, int p, const double* CP, const double* X, int B,
                           long cta, long ncta, double* sm);

template <int NP>
__global__ void __launch_bounds__(kThreads) k_fixup(double* Y, long ybase, long nScan, int p, const double* CP,
                                                    const double* X, int B)
{
    extern __shared__ double sm[];
    fixup_body<NP>(Y, ybase, nScan, p, CP, X, B, blockIdx.x, gridDim.x, sm);
}

// Batched fix-up: blockIdx.y selects the system, blockIdx.x strides its blocks.
template <int NP>
__global__ void __launch_bounds__(kThreads) k_fixup_batch(const LeafArgs* __restrict__ sys, const double* const* CPs,
                                                          int B)
{
    extern __shared__ double sm[];
    const LeafArgs& a = sys[blockIdx.y];
    fixup_body<NP>(a.Y, a.ybase, a.nScan, a.p, CPs[blockIdx.y], a.G, B, blockIdx.x, gridDim.x, sm);
}

template <int NP>
__device__ void fixup_body(double* Y, long ybase, long nScan, int p, const double* CP, const double* X, int B,
                           long cta, long ncta, double* sm)
{
    // work items: (8 fragment rows of CP, 8 blocks); one warp per item, so
    // few long blocks (small systems) spread over rows as many short blocks
    // spread over columns.  CP (B p x NP) is small and read through L2.
    (void)sm;
    const int M = B * p;
    const int rfs = (M + 7) >> 3;
    const int rgs = (rfs + 7) >> 3;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gq = lane >> 2, tq = lane & 3;
    const long nblocks = (nScan + B - 1) / B;
    const long cfs = (nblocks + 7) >> 3;
    const long items = (long)rgs * cfs;
    for (long it = cta * (kThreads / 32) + warp; it < items; it += ncta * (kThreads / 32)) {
        const long cb = it % cfs;
        const int rb0 = (int)(it / cfs) * 8;
        const long bb = cb * 8 + gq;
        double bv[NP / 4];
#pragma unroll
        for (int k = 0; k < NP; k += 4) bv[k / 4] = bb < nblocks ? X[bb * NP + k + tq] : 0.0;
        double acc[8][2];
#pragma unroll
        for (int r = 0; r < 8; ++r) acc[r][0] = acc[r][1] = 0.0;
#pragma unroll
        for (int k = 0; k < NP; k += 4)
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int row = (rb0 + r) * 8 + gq;
                const double a = (rb0 + r < rfs && row < M) ? CP[(long)row * NP + k + tq] : 0.0;
                dmma_m8n8k4(acc[r][0], acc[r][1], a, bv[k / 4]);
            }
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int row = (rb0 + r) * 8 + gq;
            if (rb0 + r >= rfs || row >= M) continue;
            const int jj = row / p, o = row - jj * p;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const long b = cb * 8 + 2 * tq + e;
                const long j = b * B + jj;
                if (b < nblocks && j < nScan) Y[(ybase + j) * p + o] += acc[r][e];
            }
        }
    }
}

// Power table continuation and the output table CP (one CTA).
template <int NP>
__device__ void tables_body(double* P, int l0, int l1, double* CP, const double* Cext, int p, int R, double* sm);

template <int NP>
__global__ void __launch_bounds__(kThreads, 1) k_tables(double* P, int l0, int l1, double* CP, const double* Cext,
                                                        int p, int R)
{
    extern __shared__ double sm[];
    tables_body<NP>(P, l0, l1, CP, Cext, p, R, sm);
}

// Batched tables: one CTA per system (P levels 1..l1-1, CP for B = 2^R).
template <int NP>
__global__ void __launch_bounds__(kThreads, 1) k_tables_batch(const LeafArgs* __restrict__ sys, double* const* CPs,
                                                              const double* const* Cexts, int l1, int R)
{
    extern __shared__ double sm[];
    const LeafArgs& a = sys[blockIdx.x];
    tables_body<NP>(const_cast<double*>(a.P), 1, l1, CPs[blockIdx.x], Cexts[blockIdx.x], a.p, R, sm);
}

// Sequential carry over the blocks of one system per CTA (FP64):
//   X_0 = x0, X_{b+1} = P_R X_b + G_b, and G_b <- X_b (the block's carry).
// Row i of the product is owned by thread i (NP <= 64 threads active).
template <int NP>
__global__ void __launch_bounds__(kThreads, 1) k_chain_batch(const LeafArgs* __restrict__ sys,
                                                             const double* const* X0s, int R, int bpt)
{
    __shared__ double sA[NP * (NP + 1)];
    __shared__ double sX[2][NP];
    const LeafArgs& a = sys[blockIdx.x];
    const double* PR = a.P + (long)R * NP * NP;
    for (int e = threadIdx.x; e < NP * NP; e += kThreads) sA[(e / NP) * (NP + 1) + e % NP] = PR[e];
    if (threadIdx.x < NP) sX[0][threadIdx.x] = X0s[blockIdx.x][threadIdx.x];
    __syncthreads();
    const long nb = a.ntiles * bpt;
    const int i = threadIdx.x;
    int cur = 0;
    double g = (i < NP && nb > 0) ? a.G[i] : 0.0;
    for (long b = 0; b < nb; ++b) {
        double gn = (i < NP && b + 1 < nb) ? a.G[(b + 1) * NP + i] : 0.0;  // prefetch the next aggregate
        if (i < NP) {
            const double* row = sA + i * (NP + 1);
            const double* x = sX[cur];
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
            for (int k = 0; k < NP; k += 4) {
                s0 = fma(row[k], x[k], s0);
                s1 = fma(row[k + 1], x[k + 1], s1);
                s2 = fma(row[k + 2], x[k + 2], s2);
                s3 = fma(row[k + 3], x[k + 3], s3);
            }
            a.G[b * NP + i] = x[i];
            sX[cur ^ 1][i] = ((s0 + s1) + (s2 + s3)) + g;
        }
        g = gn;
        cur ^= 1;
        __syncthreads();
    }
}

template <int NP>
__device__ void tables_body(double* P, int l0, int l1, double* CP, const double* Cext, int p, int R, double* sm)
{
    double* sA = sm;             // current P_l (swizzled)
    double* sN = sm + NP * NP;   // next
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gq = lane >> 2, tq = lane & 3;
    constexpr int RF = NP / 8;
    if (l0 < l1) load_matrix<NP>(sA, P + (long)(l0 - 1) * NP * NP);
    __syncthreads();
    for (int l = l0; l < l1; ++l) {
        // sN = sA * sA: warp rb < RF owns fragment row rb and all RF columns
        if (warp < RF) {
            constexpr int KS = (8 / RF) < (NP / 4) ? (8 / RF) : (NP / 4);
            const int rb = warp;
            double acc[RF][2];
            warp_mma<RF, KS>(
                acc, NP / 4, [&](int s) { return sA[sidx<NP>(rb * 8 + gq, 4 * s + tq)]; },
                [&](int j, int s) { return sA[sidx<NP>(4 * s + tq, j * 8 + gq)]; });
#pragma unroll
            for (int cb = 0; cb < RF; ++cb) {
                const int r = rb * 8 + gq, c0 = cb * 8 + 2 * tq;
                sN[sidx<NP>(r, c0)] = acc[cb][0];
                sN[sidx<NP>(r, c0 + 1)] = acc[cb][1];
                P[(long)l * NP * NP + (long)r * NP + c0] = acc[cb][0];
                P[(long)l * NP * NP + (long)r * NP + c0 + 1] = acc[cb][1];
            }
        }
        __syncthreads();
        double* t = sA;
        sA = sN;
        sN = t;
    }
    if (!CP) return;
    // CP[0] = Cext; CP[i + 2^k] = CP[i] P_k (rows (i, o) of a (2^k p) x NP block)
    for (int e = threadIdx.x; e < p * NP; e += kThreads) CP[e] = Cext[e];
    __syncthreads();
    for (int k = 0; k < R; ++k) {
        load_matrix<NP>(sA, P + (long)k * NP * NP);
        __syncthreads();
        const int rows = (1 << k) * p;
        const int rfs = (rows + 7) >> 3;
        for (int f = warp; f < rfs * RF; f += 8) {
            const int rb = f % rfs, cb = f / rfs;
            const int r = rb * 8 + gq;
            double d0 = 0.0, d1 = 0.0;
            for (int q = 0; q < NP; q += 4) {
                const double av = r < rows ? CP[(long)r * NP + q + tq] : 0.0;
                const double bv = sA[sidx<NP>(q + tq, cb * 8 + gq)];
                dmma_m8n8k4(d0, d1, av, bv);
            }
            if (r < rows) {
                const int c0 = cb * 8 + 2 * tq;
                CP[(long)(rows + r) * NP + c0] = d0;
                CP[(long)(rows + r) * NP + c0 + 1] = d1;
            }
        }
        __syncthreads();
    }
}

template <class K>
void set_smem(K kernel, size_t bytes)
{
    PARODE_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

constexpr size_t kSmemCap = 220 * 1024;
constexpr size_t kSmemOptInMax = 232448 - 1024;  // 227 KB per CTA on sm_100, less a little headroom

}  // namespace

bool blocked_shape(int Ns, int m, int solver, BlockedShape* out)
{
    int NP = 8;
    while (NP < Ns) NP <<= 1;
    if (NP > 64) return false;
    BlockedShape sh;
    sh.NP = NP;
    sh.R = NP == 64 ? 4 : NP == 32 ? 6 : NP == 16 ? 8 : 10;
    sh.B = 1 << sh.R;
    const size_t pbytes = (size_t)sh.R * NP * NP * sizeof(double);
    int S = NP == 64 ? 128 : NP == 32 ? 512 : NP == 16 ? 1024 : 2048;
    auto leaf_bytes = [&](int s) {
        long ns = solver == 0 ? 2L * s + 1 : s + 4;
        return pbytes + (size_t)s * NP * sizeof(double) + (size_t)ns * std::max(m, 1) * sizeof(double);
    };
    while (S > sh.B * 8 && leaf_bytes(S) > kSmemCap) S >>= 1;
    if (leaf_bytes(S) > kSmemCap || S < sh.B) return false;
    sh.S = S;
    sh.leaf_smem = leaf_bytes(S);
    int Si = NP == 64 ? 128 : NP == 32 ? 512 : NP == 16 ? 1024 : 2048;
    while (Si > sh.B && pbytes + (size_t)Si * NP * sizeof(double) > kSmemCap) Si >>= 1;
    sh.S_items = Si;
    sh.items_smem = pbytes + (size_t)Si * NP * sizeof(double);
    *out = sh;
    return true;
}

size_t blocked_leaf_stage_bytes(const BlockedShape& sh, int n, int m, int p, int solver)
{
    const int W = solver == 0 ? 3 : 5;
    size_t extra = ((size_t)n * W * m + (size_t)p * n + (size_t)p * m) * sizeof(double);
    size_t total = sh.leaf_smem + extra;
    return total <= kSmemOptInMax ? total : 0;
}

template <int NP>
static void leaf_t(const BlockedShape& sh, const LeafArgs& a, int grid, cudaStream_t s)
{
    size_t smem = a.stage ? blocked_leaf_stage_bytes(sh, a.n, a.m, a.p, a.solver) : sh.leaf_smem;
    if (smem == 0) throw Error(kInvalidArgument, "leaf staging does not fit");
    set_smem(k_leaf<NP>, smem);
    unsigned g = (unsigned)std::max<long>(1, std::min<long>(a.ntiles, grid));
    k_leaf<NP><<<g, kThreads, smem, s>>>(a, sh.R, sh.S);
    PARODE_CUDA(cudaGetLastError());
}

void launch_blocked_leaf(const BlockedShape& sh, const LeafArgs& a, int grid, cudaStream_t s)
{
    switch (sh.NP) {
    case 8: leaf_t<8>(sh, a, grid, s); break;
    case 16: leaf_t<16>(sh, a, grid, s); break;
    case 32: leaf_t<32>(sh, a, grid, s); break;
    case 64: leaf_t<64>(sh, a, grid, s); break;
    default: throw Error(kInvalidArgument, "blocked path: unsupported NP");
    }
}

long blocked_items_scratch(const BlockedShape& sh, long count)
{
    long total = 0;
    long c = count;
    while (c > sh.S_items) {
        c = (c + sh.B - 1) / sh.B;
        total += c;
    }
    return total + 1;
}

template <int NP>
static int carry_t(const BlockedShape& sh, double* items, long count, int base_level, const double* P,
                   const double* X0, double* work, int sms, cudaStream_t s)
{
    const size_t mat = (size_t)NP * NP;
    std::vector<double*> arr{items};
    std::vector<long> cnt{count};
    std::vector<int> lev{base_level};
    int launches = 0;
    set_smem(k_items_up<NP>, sh.items_smem);
    set_smem(k_items_down<NP>, sh.items_smem);
    double* w = work;
    while (cnt.back() > sh.S_items) {
        long c = cnt.back();
        long nn = (c + sh.B - 1) / sh.B;
        unsigned grid = (unsigned)std::min<long>((c + sh.S_items - 1) / sh.S_items, sms);
        k_items_up<NP><<<grid, kThreads, sh.items_smem, s>>>(arr.back(), c, P + lev.back() * mat, sh.R,
                                                              sh.S_items, w);
        PARODE_CUDA(cudaGetLastError());
        ++launches;
        arr.push_back(w);
        cnt.push_back(nn);
        lev.push_back(lev.back() + sh.R);
        w += nn * NP;
    }
    {
        long c = cnt.back();
        int L = 1;
        while (L < c) L <<= 1;
        size_t smem = (mat + (size_t)L * NP) * sizeof(double);
        set_smem(k_items_top<NP>, smem);
        k_items_top<NP><<<1, kThreads, smem, s>>>(arr.back(), c, P + lev.back() * mat, L, X0);
        PARODE_CUDA(cudaGetLastError());
        ++launches;
    }
    for (int h = (int)arr.size() - 2; h >= 0; --h) {
        long c = cnt[h];
        unsigned grid = (unsigned)std::min<long>((c + sh.S_items - 1) / sh.S_items, sms);
        k_items_down<NP><<<grid, kThreads, sh.items_smem, s>>>(arr[h], c, P + lev[h] * mat, sh.R, sh.S_items,
                                                                arr[h + 1]);
        PARODE_CUDA(cudaGetLastError());
        ++launches;
    }
    return launches;
}

int launch_blocked_carry(const BlockedShape& sh, double* items, long count, int base_level, const double* P,
                         const double* X0, double* work, int sms, cudaStream_t s)
{
    switch (sh.NP) {
    case 8: return carry_t<8>(sh, items, count, base_level, P, X0, work, sms, s);
    case 16: return carry_t<16>(sh, items, count, base_level, P, X0, work, sms, s);
    case 32: return carry_t<32>(sh, items, count, base_level, P, X0, work, sms, s);
    case 64: return carry_t<64>(sh, items, count, base_level, P, X0, work, sms, s);
    default: throw Error(kInvalidArgument, "blocked path: unsupported NP");
    }
}

template <int NP>
static void fixup_t(const BlockedShape& sh, double* Y, long ybase, long nScan, int p, const double* CP,
                    const double* X, cudaStream_t s)
{
    const long rgs = ((sh.B * p + 7) / 8 + 7) / 8;
    const long nblocks = (nScan + sh.B - 1) / sh.B;
    const long items = rgs * ((nblocks + 7) / 8);
    const unsigned grid = (unsigned)std::max<long>(1, std::min<long>((items + 7) / 8, 148L * 8));
    k_fixup<NP><<<grid, kThreads, 0, s>>>(Y, ybase, nScan, p, CP, X, sh.B);
    PARODE_CUDA(cudaGetLastError());
}

void launch_blocked_fixup(const BlockedShape& sh, double* Y, long ybase, long nScan, int p, const double* CP,
                          const double* X, cudaStream_t s)
{
    switch (sh.NP) {
    case 8: fixup_t<8>(sh, Y, ybase, nScan, p, CP, X, s); break;
    case 16: fixup_t<16>(sh, Y, ybase, nScan, p, CP, X, s); break;
    case 32: fixup_t<32>(sh, Y, ybase, nScan, p, CP, X, s); break;
    case 64: fixup_t<64>(sh, Y, ybase, nScan, p, CP, X, s); break;
    default: throw Error(kInvalidArgument, "blocked path: unsupported NP");
    }
}

template <int NP>
static void tables_t(const BlockedShape& sh, double* P, int l0, int l1, double* CP, const double* Cext, int p,
                     cudaStream_t s)
{
    size_t smem = 2 * (size_t)NP * NP * sizeof(double);
    set_smem(k_tables<NP>, smem);
    k_tables<NP><<<1, kThreads, smem, s>>>(P, l0, l1, CP, Cext, p, sh.R);
    PARODE_CUDA(cudaGetLastError());
}

template <int NP>
static void preload_carry_t()
{
    cudaFuncAttributes a;
    PARODE_CUDA(cudaFuncGetAttributes(&a, k_items_up<NP>));
    PARODE_CUDA(cudaFuncGetAttributes(&a, k_items_down<NP>));
    PARODE_CUDA(cudaFuncGetAttributes(&a, k_items_top<NP>));
    PARODE_CUDA(cudaFuncGetAttributes(&a, k_tables<NP>));
}

void preload_blocked_carry_kernels()
{
    preload_carry_t<8>();
    preload_carry_t<16>();
    preload_carry_t<32>();
    preload_carry_t<64>();
}

void launch_blocked_tables(const BlockedShape& sh, double* P, int l0, int l1, double* CP, const double* Cext, int p,
                           cudaStream_t s)
{
    switch (sh.NP) {
    case 8: tables_t<8>(sh, P, l0, l1, CP, Cext, p, s); break;
    case 16: tables_t<16>(sh, P, l0, l1, CP, Cext, p, s); break;
    case 32: tables_t<32>(sh, P, l0, l1, CP, Cext, p, s); break;
    case 64: tables_t<64>(sh, P, l0, l1, CP, Cext, p, s); break;
    default: throw Error(kInvalidArgument, "blocked path: unsupported NP");
    }
}

// ---------------------------------------------------------------------------
// batched launchers
// ---------------------------------------------------------------------------

size_t batch_leaf_smem(const BlockedShape& sh, int ms, long stage_doubles)
{
    size_t base = (size_t)sh.R * sh.NP * sh.NP * sizeof(double) + (size_t)sh.S * sh.NP * sizeof(double) +
                  (size_t)(2 * sh.S + 1) * std::max(ms, 1) * sizeof(double);
    return base + (size_t)stage_doubles * sizeof(double);
}

template <int NP>
static void batch_t(int what, const BlockedShape& sh, const BatchLaunch& b, cudaStream_t s)
{
    switch (what) {
    case 0: {
        size_t smem = 2 * (size_t)NP * NP * sizeof(double);
        set_smem(k_tables_batch<NP>, smem);
        k_tables_batch<NP><<<b.nsys, kThreads, smem, s>>>(b.sys, b.CPs, b.Cexts, sh.R + 1, sh.R);
        break;
    }
    case 1: {
        set_smem(k_leaf_batch<NP>, b.leaf_smem);
        k_leaf_batch<NP><<<b.grid, kThreads, b.leaf_smem, s>>>(b.sys, b.items, b.nitems, sh.R, sh.S, b.ms);
        break;
    }
    case 2:
        k_chain_batch<NP><<<b.nsys, kThreads, 0, s>>>(b.sys, b.X0s, sh.R, sh.S / sh.B);
        break;
    case 3: {
        const long rgs = ((sh.B * b.pmax + 7) / 8 + 7) / 8;
        const long items = rgs * ((b.max_blocks + 7) / 8);
        const unsigned gx = (unsigned)std::max<long>(1, std::min<long>((items + 7) / 8, 16));
        dim3 grid(gx, (unsigned)b.nsys);
        k_fixup_batch<NP><<<grid, kThreads, 0, s>>>(b.sys, b.CPs, sh.B);
        break;
    }
    }
    PARODE_CUDA(cudaGetLastError());
}

void launch_batch_stage(int what, const BlockedShape& sh, const BatchLaunch& b, cudaStream_t s)
{
    if (b.nsys <= 0) return;
    switch (sh.NP) {
    case 8: batch_t<8>(what, sh, b, s); break;
    case 16: batch_t<16>(what, sh, b, s); break;
    case 32: batch_t<32>(what, sh, b, s); break;
    case 64: batch_t<64>(what, sh, b, s); break;
    default: throw Error(kInvalidArgument, "batched blocked path: unsupported NP");
    }
}

}  // namespace parode
