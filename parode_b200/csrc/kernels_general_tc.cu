// kernels_general_tc.cu -- per-pair map composition on tcgen05 (3xTF32), the
// mixed form of the general affine scan (kernels_general.cu).
//
// For each pair of a level (k = right child, j = k - d) one CTA computes
//   V[k] <- M[k] V[j] + V[k]   in FP64 on the CUDA cores (old M[k]),
//   M[k] <- M[k] M[j]          on the tensor cores,
// the reference's MM / MVV up-sweep step (Kernels/MMKernelScanUpsweep.cl:24-53,
// Kernels/MVVKernelScanUpsweep.cl:25-48).  The product is D = A B^T with
// A = M[k] (rows i, K = l: row-major is K-major) and B[c][l] = M[j][l][c]
// (M[j] transposed while it is split).  Only E = M - I goes through the
// tensor cores (M[k] M[j] = M[k] + M[j] - I + E[k] E[j], the first three
// terms in FP64), split into TF32 hi/lo in the MMA's canonical K-major
// layout (8-row x 16-byte core matrices), and
// hi*hi goes to one TMEM accumulator, hi*lo + lo*hi to a second, summed in
// FP64 by the epilogue (the chains are NP/8 and NP/4 MMAs long).  The MMA
// is M = 128: rows NP..127 of A read whatever follows the A tile in shared
// memory, and their results are never stored.  M[k] and M[j] arrive by bulk
// copies (TMA engine); the CTA walks its pairs one at a time, every wait
// bounded (a time-out sets the status word and ends the CTA's loop).
#include "common.h"
#include "general.h"
#include "tc05.cuh"

#include <algorithm>

namespace parode {

namespace {

using namespace tc05;

constexpr int kThreads = 256;
constexpr long long kWaitLimit = 1LL << 31;

template <int NP>
struct Lay {
    static constexpr uint32_t raw = (uint32_t)NP * NP * 8;      // one FP64 matrix
    static constexpr uint32_t half = 128u * NP * 4;            // one TF32 operand of 128 rows x NP K
    static constexpr uint32_t bhalf = (uint32_t)NP * NP * 4;   // B: NP rows x NP K
    static constexpr uint32_t offA = 0;                        // raw M[k], then the output staging
    static constexpr uint32_t offB = raw;                      // raw M[j]
    static constexpr uint32_t offAh = 2 * raw;                 // A hi (the lo block follows at + half)
    static constexpr uint32_t offBh = offAh + 2 * half;        // B hi, B lo at + bhalf
    static constexpr uint32_t offV = offBh + 2 * bhalf;        // V[j] (NP doubles)
    static constexpr uint32_t offBar = offV + NP * 8;          // loaded, mma done
    static constexpr uint32_t offSlot = offBar + 16;
    static constexpr uint32_t bytes = offSlot + 16;
};

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

template <int NP>
__global__ void __launch_bounds__(kThreads, 1) k_compose_tc(double* __restrict__ M, double* __restrict__ V, long d,
                                                             long npairs, int* status)
{
    using L = Lay<NP>;
    extern __shared__ __align__(1024) unsigned char sm[];
    double* Araw = reinterpret_cast<double*>(sm + L::offA);
    double* Braw = reinterpret_cast<double*>(sm + L::offB);
    double* vj = reinterpret_cast<double*>(sm + L::offV);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + L::offBar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + L::offSlot);
    volatile int* failed = reinterpret_cast<volatile int*>(sm + L::offSlot + 8);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        *failed = 0;
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(slot, 128);  // hi*hi: columns 0..NP-1, corrections: 64..64+NP-1
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = *slot;
    uint32_t phase = 0;
    for (long q = blockIdx.x; q < npairs && !*failed; q += gridDim.x, phase ^= 1) {
        const long k = q * 2 * d + 2 * d - 1, j = k - d;
        double* Mk = M + k * (long)NP * NP;
        const double* Mj = M + j * (long)NP * NP;
        if (threadIdx.x == 0) {
            fence_async_smem();  // the staging writes of the last pair precede the copies into it
            mbar_arrive_tx(&bars[0], 2 * L::raw);
            bulk_g2s(Araw, Mk, L::raw, &bars[0]);
            bulk_g2s(Braw, Mj, L::raw, &bars[0]);
        }
        for (int e = threadIdx.x; e < NP; e += kThreads) vj[e] = V[j * NP + e];
        if (!mbar_wait(&bars[0], phase, kWaitLimit)) {
            *failed = 1;
            atomicExch(status, 1);
        }
        __syncthreads();
        if (*failed) break;
        // vector part in FP64 with the old M[k]
        for (int r = threadIdx.x; r < NP; r += kThreads) {
            double s = 0.0;
#pragma unroll 8
            for (int c = 0; c < NP; ++c) s = fma(Araw[r * NP + c], vj[c], s);
            V[k * NP + r] += s;
        }
        // split of E = M - I (the identity part is exact and stays out of the
        // tensor cores: M[k] M[j] = M[k] + M[j] - I + E[k] E[j], so the TF32
        // rounding is relative to E[k] E[j], which is small for maps near the
        // identity): A rows i, K = l from E[k][i][l]; B rows c, K = l from E[j][l][c]
        for (int e = threadIdx.x; e < NP * NP; e += kThreads) {
            const int r = e / NP, c = e - r * NP;
            const double id = r == c ? 1.0 : 0.0;
            float hi, lo;
            split_tf32((float)(Araw[e] - id), hi, lo);
            const uint32_t oa = kmajor_off(r, c, NP);
            *reinterpret_cast<float*>(sm + L::offAh + oa) = hi;
            *reinterpret_cast<float*>(sm + L::offAh + L::half + oa) = lo;
            split_tf32((float)(Braw[e] - id), hi, lo);    // Braw[r][c] = M[j][l = r][c]
            const uint32_t ob = kmajor_off(c, r, NP);     // B row c, K index r
            *reinterpret_cast<float*>(sm + L::offBh + ob) = hi;
            *reinterpret_cast<float*>(sm + L::offBh + L::bhalf + ob) = lo;
        }
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        if (threadIdx.x == 0) {
            constexpr uint32_t SBO = NP * 32;  // 8 rows x NP tf32
            constexpr uint32_t idesc = make_idesc(128, NP);
            const uint32_t a0 = smem_u32(sm + L::offAh), b0 = smem_u32(sm + L::offBh);
            const uint64_t ah = make_desc(a0, 128, SBO), al = make_desc(a0 + L::half, 128, SBO);
            const uint64_t bh = make_desc(b0, 128, SBO), bl = make_desc(b0 + L::bhalf, 128, SBO);
            const uint64_t A[3] = {ah, ah, al};
            const uint64_t B[3] = {bh, bl, bh};
#pragma unroll
            for (int p = 0; p < 3; ++p)
#pragma unroll
                for (int kk = 0; kk < NP / 8; ++kk)
                    mma_tf32(tbase + (p == 0 ? 0u : 64u), A[p] + (uint64_t)(kk * 16), B[p] + (uint64_t)(kk * 16),
                             idesc, (kk == 0 && p < 2) ? 0u : 1u);
            mma_commit(&bars[1]);
        }
        if (!mbar_wait(&bars[1], phase, kWaitLimit)) {
            *failed = 1;
            atomicExch(status, 1);
        }
        __syncthreads();  // every thread sees the same verdict before the warp-wide TMEM loads
        if (*failed) break;
        fence_after_sync();
        // epilogue: rows 0..NP-1 live in TMEM lanes 0..NP-1; warps w % 4 = the
        // lane quarter, w / 4 = which half of the 32-column groups
        if (32 * (warp & 3) < NP) {
            const int row = 32 * (warp & 3) + lane;
            for (int cg = warp >> 2; cg * 32 < NP; cg += 2) {
                uint32_t hh[32], cc[32];
                const uint32_t lanebase = (uint32_t)(32 * (warp & 3)) << 16;
                tmem_ld32(tbase + lanebase + (uint32_t)(cg * 32), hh);
                tmem_ld32(tbase + lanebase + 64u + (uint32_t)(cg * 32), cc);
                tmem_wait_ld();
                if (row < NP) {
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        const int col = cg * 32 + c;
                        if (col < NP) {
                            // M[k] + M[j] - I in FP64, plus the tensor-core E[k] E[j]
                            const double exact = Araw[row * NP + col] + Braw[row * NP + col] - (row == col ? 1.0 : 0.0);
                            Araw[row * NP + col] = exact + ((double)__uint_as_float(hh[c]) + (double)__uint_as_float(cc[c]));
                        }
                    }
                }
            }
        }
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        if (*failed) break;
        for (int e = threadIdx.x; e < NP * NP; e += kThreads) Mk[e] = Araw[e];
        __syncthreads();  // the next pair's copies overwrite Araw
    }
    __syncthreads();
    if (*failed && threadIdx.x == 0) {
        // copies or MMAs of the pair that timed out may still be in flight:
        // wait for them, again with a bound, before the CTA leaves
        mbar_wait(&bars[0], phase, 1 << 20);
        mbar_wait(&bars[1], phase, 1 << 20);
    }
    fence_after_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tbase, 128);
}

template <int NP>
void compose_tc_t(double* M, double* V1, long d, long npairs, int sms, int* status, cudaStream_t s)
{
    const size_t smem = Lay<NP>::bytes;
    PARODE_CUDA(cudaFuncSetAttribute(k_compose_tc<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned grid = (unsigned)std::min<long>(npairs, sms);
    k_compose_tc<NP><<<grid, kThreads, smem, s>>>(M, V1, d, npairs, status);
    PARODE_CUDA(cudaGetLastError());
}

}  // namespace

bool compose_tc_supported(int NP) { return NP == 32 || NP == 64; }

void launch_compose_tc(int NP, double* M, double* V1, long d, long npairs, int sms, int* status, cudaStream_t s)
{
    switch (NP) {
    case 32: compose_tc_t<32>(M, V1, d, npairs, sms, status, s); break;
    case 64: compose_tc_t<64>(M, V1, d, npairs, sms, status, s); break;
    default: throw Error(kInvalidArgument, "tensor-core composition: NP must be 32 or 64");
    }
}

}  // namespace parode
