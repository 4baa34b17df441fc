// kernels_general.cu -- the general affine scan: a distinct map per step,
// composed pair by pair.
//
// The reference composes a distinct matrix at every tree node: its up-sweep
// computes M[k] <- M[k] M[k-d] and v[k] <- M[k] v[k-d] + v[k] for every pair
// of a level (Kernels/MMKernelScanUpsweep.cl:13-56,
// Kernels/MVVKernelScanUpsweep.cl:14-50), its down-sweep passes prefixes
// down with M[k-d] (Kernels/MVVKernelScanDownsweep.cl:14-50,
// RootCopyKernelScanDownsweep.cl:3-21).  The LTI solves never need the matrix
// products (every node of a level holds the same power of Phi); this path
// takes arbitrary maps x_{k+1} = M_k x_k + v_k, as a time-varying system
// gives them, and is the reference's scan step for step.
//
// Layout, in place: M[Tp][NP][NP] and V[Tp + 1][NP] (slot -1 = x0; NP = the
// scan dimension rounded up to 8, zero padded).  After the up-sweep, slot k of
// a right child holds the composition of its subtree; the down-sweep runs in
// place as the level-synchronous scan's does (the node over [g 2d, g 2d + 2d)
// keeps its prefix in slot g 2d - 1, the left half's total M[g 2d + d - 1]
// carries it to the right half), so x_k ends in slot k - 1.
//
// Two forms of the matrix products: FP64 on the DMMA tensor cores
// (k_compose_f64), and 3xTF32 on tcgen05 with FP32 accumulators in TMEM
// (k_compose_tc, kernels_general_tc.cu).  The vector updates are FP64 in both.
#include "common.h"
#include "device_common.cuh"
#include "general.h"

#include <algorithm>

namespace parode {

namespace {

constexpr int kThreads = 256;

template <int NP>
constexpr int pitch()
{
    return NP + 2;  // doubles: the DMMA fragment reads of B hit distinct banks
}

// One pair per iteration: k = right child, j = k - d (left child).
//   V[k] <- M[k] V[j] + V[k]   (with the old M[k])
//   M[k] <- M[k] M[j]
template <int NP>
__global__ void __launch_bounds__(kThreads) k_compose_f64(double* __restrict__ M, double* __restrict__ V, long d,
                                                           long npairs)
{
    extern __shared__ double sm[];
    double* As = sm;                     // M[k], NP x pitch
    double* Bs = As + NP * pitch<NP>();  // M[j]
    double* vj = Bs + NP * pitch<NP>();  // V[j]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    constexpr int TILES = (NP / 8) * (NP / 8);
    for (long q = blockIdx.x; q < npairs; q += gridDim.x) {
        const long k = q * 2 * d + 2 * d - 1, j = k - d;
        const double* Mk = M + k * (long)NP * NP;
        const double* Mj = M + j * (long)NP * NP;
        for (int e = threadIdx.x; e < NP * NP; e += kThreads) {
            const int r = e / NP, c = e - r * NP;
            As[r * pitch<NP>() + c] = Mk[e];
            Bs[r * pitch<NP>() + c] = Mj[e];
        }
        for (int e = threadIdx.x; e < NP; e += kThreads) vj[e] = V[j * NP + e];
        __syncthreads();
        // vector part, FP64 on the CUDA cores
        for (int r = threadIdx.x; r < NP; r += kThreads) {
            double s = 0.0;
#pragma unroll 8
            for (int c = 0; c < NP; ++c) s = fma(As[r * pitch<NP>() + c], vj[c], s);
            V[k * NP + r] += s;
        }
        // matrix part, FP64 DMMA (m8n8k4), 8 x 8 output tiles dealt to the warps
        double* Mo = M + k * (long)NP * NP;
        for (int tile = warp; tile < TILES; tile += kThreads / 32) {
            const int mt = tile / (NP / 8), nt = tile - mt * (NP / 8);
            double d0 = 0.0, d1 = 0.0;
#pragma unroll 4
            for (int kk = 0; kk < NP / 4; ++kk) {
                const double a = As[(mt * 8 + g) * pitch<NP>() + kk * 4 + t];
                const double b = Bs[(kk * 4 + t) * pitch<NP>() + nt * 8 + g];
                dmma_m8n8k4(d0, d1, a, b);
            }
            Mo[(long)(mt * 8 + g) * NP + nt * 8 + 2 * t] = d0;
            Mo[(long)(mt * 8 + g) * NP + nt * 8 + 2 * t + 1] = d1;
        }
        __syncthreads();
    }
}

// Down-sweep level: for each pair g, L = g 2d + d - 1, p = g 2d - 1:
// V[L] <- M[L] V[p] + V[L].  V points at slot 0 (slot -1 = V - NP).  One
// warp per pair, each lane owning rows lane, lane + 32.
template <int NP>
__global__ void __launch_bounds__(kThreads) k_down_general(const double* __restrict__ M, double* __restrict__ V,
                                                            long d, long npairs)
{
    const int lane = threadIdx.x & 31;
    const long wid = ((long)blockIdx.x * kThreads + threadIdx.x) >> 5;
    const long nw = ((long)gridDim.x * kThreads) >> 5;
    for (long q = wid; q < npairs; q += nw) {
        const long L = q * 2 * d + d - 1, p = q * 2 * d - 1;
        const double* ML = M + L * (long)NP * NP;
        const double* vp = V + p * NP;
        double xp[NP];
#pragma unroll
        for (int c = 0; c < NP; ++c) xp[c] = vp[c];
        for (int r = lane; r < NP; r += 32) {
            double s = 0.0;
#pragma unroll
            for (int c = 0; c < NP; ++c) s = fma(ML[(long)r * NP + c], xp[c], s);
            V[L * NP + r] += s;
        }
    }
}

// Caller arrays (count x ns, row-major) into the padded scan layout; rows
// past count: M = 0, V = 0.
__global__ void k_general_in(double* __restrict__ Mp, double* __restrict__ Vp, const double* __restrict__ M,
                             const double* __restrict__ Vin, const double* __restrict__ x0, int ns, int NP,
                             long count, long Tp)
{
    const long nm = Tp * (long)NP * NP;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < nm; e += (long)gridDim.x * blockDim.x) {
        const long k = e / ((long)NP * NP);
        const int rc = (int)(e - k * (long)NP * NP), r = rc / NP, c = rc - r * NP;
        Mp[e] = (k < count && r < ns && c < ns) ? M[(k * ns + r) * ns + c] : 0.0;
    }
    const long nv = (Tp + 1) * (long)NP;  // slot -1 first
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < nv; e += (long)gridDim.x * blockDim.x) {
        const long s = e / NP - 1;
        const int r = (int)(e - (s + 1) * NP);
        double v = 0.0;
        if (r < ns) {
            if (s < 0) v = x0 ? x0[r] : 0.0;
            else if (s < count && Vin) v = Vin[s * ns + r];
        }
        Vp[e] = v;
    }
}

// Ms[k] = Phi for k < count (the reference's DistributeA, Kernels/DistributeA.cl:6-13).
__global__ void k_distribute(double* __restrict__ Ms, const double* __restrict__ Phi, int NP, long count)
{
    const long per = (long)NP * NP;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < count * per; e += (long)gridDim.x * blockDim.x)
        Ms[e] = Phi[e % per];
}

// x_k (slot k - 1) into the caller's X (count x ns).
__global__ void k_general_out(double* __restrict__ X, const double* __restrict__ Vp, int ns, int NP, long count)
{
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < count * ns; e += (long)gridDim.x * blockDim.x) {
        const long k = e / ns;
        const int r = (int)(e - k * ns);
        X[e] = Vp[k * NP + r];  // Vp = slot -1
    }
}

unsigned grid_for(long work, int per, int cap)
{
    return (unsigned)std::max<long>(1, std::min<long>((work + per - 1) / per, cap));
}

template <int NP>
void compose_f64_t(double* M, double* V1, long d, long npairs, int sms, cudaStream_t s)
{
    const size_t smem = (2 * (size_t)NP * pitch<NP>() + NP) * sizeof(double);
    PARODE_CUDA(cudaFuncSetAttribute(k_compose_f64<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned grid = (unsigned)std::min<long>(npairs, 4L * sms);
    k_compose_f64<NP><<<grid, kThreads, smem, s>>>(M, V1, d, npairs);
    PARODE_CUDA(cudaGetLastError());
}

template <int NP>
void down_t(const double* M, double* V1, long d, long npairs, int sms, cudaStream_t s)
{
    k_down_general<NP><<<grid_for(npairs, kThreads / 32, 8 * sms), kThreads, 0, s>>>(M, V1, d, npairs);
    PARODE_CUDA(cudaGetLastError());
}

}  // namespace

int general_padded_dim(int ns)
{
    int NP = 8;
    while (NP < ns) NP <<= 1;
    return NP;
}

size_t general_scan_bytes(int ns, long count)
{
    const long Tp = next_pow2(std::max<long>(count, 1));
    const long NP = general_padded_dim(ns);
    return sizeof(double) * (size_t)(Tp * NP * NP + (Tp + 1) * NP);
}

void launch_compose(int NP, int precision, double* M, double* V1, long d, long npairs, int sms, int* status,
                    cudaStream_t s)
{
    if (npairs <= 0) return;
    if (precision == kMixed && compose_tc_supported(NP)) {
        launch_compose_tc(NP, M, V1, d, npairs, sms, status, s);
        return;
    }
    switch (NP) {
    case 8: compose_f64_t<8>(M, V1, d, npairs, sms, s); break;
    case 16: compose_f64_t<16>(M, V1, d, npairs, sms, s); break;
    case 32: compose_f64_t<32>(M, V1, d, npairs, sms, s); break;
    case 64: compose_f64_t<64>(M, V1, d, npairs, sms, s); break;
    default: throw Error(kInvalidArgument, "general scan: scan dimension above 64");
    }
}

void launch_down_general(int NP, const double* M, double* V1, long d, long npairs, int sms, cudaStream_t s)
{
    if (npairs <= 0) return;
    switch (NP) {
    case 8: down_t<8>(M, V1, d, npairs, sms, s); break;
    case 16: down_t<16>(M, V1, d, npairs, sms, s); break;
    case 32: down_t<32>(M, V1, d, npairs, sms, s); break;
    case 64: down_t<64>(M, V1, d, npairs, sms, s); break;
    default: throw Error(kInvalidArgument, "general scan: scan dimension above 64");
    }
}

void launch_general_in(double* Mp, double* Vp, const double* M, const double* V, const double* x0, int ns, int NP,
                       long count, long Tp, int sms, cudaStream_t s)
{
    k_general_in<<<grid_for(Tp * (long)NP * NP, 256, 8 * sms), 256, 0, s>>>(Mp, Vp, M, V, x0, ns, NP, count, Tp);
    PARODE_CUDA(cudaGetLastError());
}

void launch_distribute(double* Ms, const double* Phi, int NP, long count, int sms, cudaStream_t s)
{
    k_distribute<<<grid_for(count * (long)NP * NP, 256, 8 * sms), 256, 0, s>>>(Ms, Phi, NP, count);
    PARODE_CUDA(cudaGetLastError());
}

void launch_general_out(double* X, const double* Vp, int ns, int NP, long count, int sms, cudaStream_t s)
{
    k_general_out<<<grid_for(count * ns, 256, 8 * sms), 256, 0, s>>>(X, Vp, ns, NP, count);
    PARODE_CUDA(cudaGetLastError());
}

}  // namespace parode
