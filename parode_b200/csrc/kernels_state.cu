// kernels_state.cu -- the initial-state part of the block-response outputs:
//   y[b gs + r] = acc[b gs + r] + sum_k Ws[r][k] X[b][k]
// for the rows r < M of W's state columns (Ws = C Phi^j at the block's steps,
// M = B p rows, K = NP) and the blocks b, where X[b] is the state entering
// block b (the carry's result) and acc the window part of the outputs.  This
// is the reference's SystemOutput C x term (Kernels/SystemOutput.cl:36-42) for
// the steps of a block, with the states those steps reach from X[b].
//
// FP64 on the DMMA tensor cores.  Ws is small (M x NP) and stays in shared
// memory for the CTA's whole run.  Each warp works alone on tiles of 16
// blocks: their states as DMMA B fragments in registers (read once from X),
// then for every 8-row slice of W (m8n8k4, K = NP; each A fragment feeds the
// two 8-block halves) the slice's window part is loaded ahead of the product
// and y written straight to global memory (8 rows of a block are 64
// consecutive bytes).  No block-wide barrier after the staging
// of W, so the warps' loads and products overlap freely.  HBM traffic per
// block: NP states read, M doubles of the window part read, M of y written.
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
                                                        const double* __restrict__ X, const double* acc, double* Y,
                                                        long gs, long nblocks, long limit)
{
    extern __shared__ double sm[];
    double* Ws = sm;  // Mp x kpitch, rows >= M zero
    for (int e = threadIdx.x; e < Mp * NP; e += kThreads) {
        const int r = e / NP, k = e - r * NP;
        Ws[r * kpitch<NP>() + k] = r < M ? W[(long)r * ld + k] : 0.0;
    }
    __syncthreads();
    // launched as a dependent of the carry's last kernel: W (formed with the
    // plan) is staged while it finishes; the states and windows after this
    grid_dep_wait();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    // a warp takes 16 blocks at a time (two 8-block halves): every A fragment
    // read from shared memory feeds two products
    const long tiles = (nblocks + 15) / 16;
    for (long tile = (long)blockIdx.x * kWarps + warp; tile < tiles; tile += (long)gridDim.x * kWarps) {
        const long b0 = tile * 16;
        double bv[2][NP / 4];
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {
            const long bb = b0 + 8 * hf + g;
#pragma unroll
            for (int kk = 0; kk < NP / 4; ++kk) bv[hf][kk] = bb < nblocks ? X[bb * NP + 4 * kk + t] : 0.0;
        }
#pragma unroll 2
        for (int mt = 0; mt < Mp / 8; ++mt) {
            const int r = mt * 8 + g;
            // this lane's four blocks: D fragment columns 2t, 2t + 1 of each half
            long o[4];
            bool v[4];
            double a[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const long c = b0 + 8 * (q >> 1) + 2 * t + (q & 1);
                o[q] = c * gs + r;
                v[q] = r < M && c < nblocks && (limit < 0 || o[q] < limit);
                a[q] = v[q] ? acc[o[q]] : 0.0;
            }
            double d[4] = {0.0, 0.0, 0.0, 0.0};
            const double* wr = Ws + r * kpitch<NP>() + t;
#pragma unroll
            for (int kk = 0; kk < NP / 4; ++kk) {
                const double w = wr[4 * kk];
                dmma_m8n8k4(d[0], d[1], w, bv[0][kk]);
                dmma_m8n8k4(d[2], d[3], w, bv[1][kk]);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (v[q]) Y[o[q]] = a[q] + d[q];
        }
    }
}

template <int NP>
size_t state_smem(int Mp)
{
    return (size_t)Mp * kpitch<NP>() * sizeof(double);
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
    const long tiles = (nblocks + 15) / 16;
    const unsigned grid =
        (unsigned)std::max<long>(1, std::min<long>((tiles + kWarps - 1) / kWarps, (long)sms * std::max(per_sm, 1)));
    launch_dependent(k_state_out<NP>, grid, kThreads, smem, s, W, ld, M, Mp, X, acc, Y, gs, nblocks, limit);
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
