// kernels_state.cu -- the initial-state part of the block-response outputs:
//   y[b gs + r] = acc[b gs + r] + sum_k Ws[r][k] X[b][k]
// for the rows r < M of W's state columns (Ws = C Phi^j at the block's steps,
// M = B p rows, K = NP) and the blocks b, where X[b] is the state entering
// block b (the carry's result) and acc the window part of the outputs.  This
// is the reference's SystemOutput C x term (Kernels/SystemOutput.cl:36-42) for
// the steps of a block, with the states those steps reach from X[b].
//
// FP64 on the DMMA tensor cores.  Ws is small (M x NP) and stays in shared
// memory for the CTA's whole run; the CTA walks tiles of 8 blocks: their
// states (8 x NP) into shared memory, each warp the 8-row slices of W it owns
// times the tile (m8n8k4, K = NP), the 8 x M results staged in shared memory
// and then added to acc and stored block by block (M consecutive doubles per
// block).  HBM traffic per block: NP states read, 2 M doubles of y read and
// written.
#include "common.h"
#include "device_common.cuh"
#include "kernels.h"

#include <algorithm>

namespace parode {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

template <int NP>
constexpr int kpitch()
{
    return NP + 4;  // doubles per shared row of W and of the state tile
}

template <int NP>
__global__ void __launch_bounds__(kThreads) k_state_out(const double* __restrict__ W, long ld, int M, int Mp,
                                                        const double* __restrict__ X, const double* __restrict__ acc,
                                                        double* __restrict__ Y, long gs, long nblocks, long limit)
{
    extern __shared__ double sm[];
    double* Ws = sm;                           // Mp x kpitch
    double* Xs = Ws + (long)Mp * kpitch<NP>();  // 8 x kpitch
    double* Ys = Xs + 8 * kpitch<NP>();         // 8 x (Mp + 4)
    const int yp = Mp + 4;
    for (int e = threadIdx.x; e < Mp * NP; e += kThreads) {
        const int r = e / NP, k = e - r * NP;
        Ws[r * kpitch<NP>() + k] = r < M ? W[(long)r * ld + k] : 0.0;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const long tiles = (nblocks + 7) / 8;
    for (long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long b0 = tile * 8;
        for (int e = threadIdx.x; e < 8 * NP; e += kThreads) {
            const int c = e / NP, k = e - c * NP;
            Xs[c * kpitch<NP>() + k] = b0 + c < nblocks ? X[(b0 + c) * NP + k] : 0.0;
        }
        __syncthreads();
        for (int mt = warp; mt < Mp / 8; mt += kWarps) {
            double d0 = 0.0, d1 = 0.0;
#pragma unroll
            for (int kk = 0; kk < NP / 4; ++kk) {
                const double a = Ws[(mt * 8 + g) * kpitch<NP>() + 4 * kk + t];
                const double b = Xs[g * kpitch<NP>() + 4 * kk + t];
                dmma_m8n8k4(d0, d1, a, b);
            }
            Ys[(2 * t) * yp + mt * 8 + g] = d0;
            Ys[(2 * t + 1) * yp + mt * 8 + g] = d1;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < 8 * M; e += kThreads) {
            const int c = e / M, r = e - c * M;
            const long b = b0 + c, off = b * gs + r;
            if (b < nblocks && (limit < 0 || off < limit)) Y[off] = acc[off] + Ys[c * yp + r];
        }
        __syncthreads();
    }
}

template <int NP>
size_t state_smem(int Mp)
{
    return ((size_t)Mp * kpitch<NP>() + 8 * (size_t)kpitch<NP>() + 8 * (size_t)(Mp + 4)) * sizeof(double);
}

template <int NP>
bool state_t(const double* W, long ld, int M, const double* X, const double* acc, double* Y, long gs, long nblocks,
             long limit, int sms, cudaStream_t s)
{
    const int Mp = (M + 7) & ~7;
    const size_t smem = state_smem<NP>(Mp);
    if (smem > 200 * 1024) return false;
    PARODE_CUDA(cudaFuncSetAttribute(k_state_out<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    PARODE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_state_out<NP>, kThreads, smem));
    const long tiles = (nblocks + 7) / 8;
    const unsigned grid = (unsigned)std::max<long>(1, std::min<long>(tiles, (long)sms * std::max(per_sm, 1)));
    k_state_out<NP><<<grid, kThreads, smem, s>>>(W, ld, M, Mp, X, acc, Y, gs, nblocks, limit);
    PARODE_CUDA(cudaGetLastError());
    return true;
}

}  // namespace

bool launch_state_out(int NP, const double* W, long ld, int M, const double* X, const double* acc, double* Y, long gs,
                      long nblocks, long limit, int sms, cudaStream_t s)
{
    if (nblocks <= 0 || M <= 0) return true;
    switch (NP) {
    case 8: return state_t<8>(W, ld, M, X, acc, Y, gs, nblocks, limit, sms, s);
    case 16: return state_t<16>(W, ld, M, X, acc, Y, gs, nblocks, limit, sms, s);
    case 24: return state_t<24>(W, ld, M, X, acc, Y, gs, nblocks, limit, sms, s);
    case 32: return state_t<32>(W, ld, M, X, acc, Y, gs, nblocks, limit, sms, s);
    case 40: return state_t<40>(W, ld, M, X, acc, Y, gs, nblocks, limit, sms, s);
    case 48: return state_t<48>(W, ld, M, X, acc, Y, gs, nblocks, limit, sms, s);
    case 56: return state_t<56>(W, ld, M, X, acc, Y, gs, nblocks, limit, sms, s);
    case 64: return state_t<64>(W, ld, M, X, acc, Y, gs, nblocks, limit, sms, s);
    default: return false;
    }
}

}  // namespace parode
