// kernels_ls_tc.cu -- mixed-precision (3xTF32 on tcgen05) level contraction
// of the level-synchronous scan, for scan dimensions above 64.
//
// One level computes dst(g, i) = sum_k P[i][k] src(g, k) + acc(g, i) for the
// columns g of the level (the reference's MVV up/down-sweep kernels,
// Kernels/MVVKernelScanUpsweep.cl:25-48, MVVKernelScanDownsweep.cl:25-48, as
// one contraction per level).  P rows sit on the MMA's M (128 per tile), the
// level's vectors on N (64 per tile), K runs over the scan dimension in
// slices of 32.  Operands stay FP64 in HBM; each slice is converted on the
// way into shared memory into TF32 hi/lo pairs (x = hi + lo) in the K-major
// no-swizzle canonical layout, and the tensor core forms hi*hi + hi*lo + lo*hi
// in FP32.  The FP32 partial sum of every K slice is drained from TMEM into
// FP64 registers (two TMEM accumulators in turn, so the next slice's MMAs run
// while the previous one drains): FP32 rounding is confined to 32-term sums.
#include "common.h"
#include "kernels.h"
#include "tc05.cuh"

#include <algorithm>

namespace parode {

namespace {

using namespace tc05;

constexpr int kThreads = 256;
constexpr int kBM = 128, kBN = 64, kBK = 32;
constexpr uint32_t kAHalf = kBM * kBK * 4;  // bytes of A hi (or lo) per stage
constexpr uint32_t kBHalf = kBN * kBK * 4;
constexpr uint32_t kStage = 2 * kAHalf + 2 * kBHalf;
constexpr uint32_t kSmem = 2 * kStage + 64;  // two stages + mbarrier + TMEM slot
constexpr uint32_t kTmemCols = 2 * kBN;      // two accumulators of 64 FP32 columns
constexpr long long kWaitLimit = 1LL << 31;

// K-major canonical offset inside a tile with kBK tf32 per row.
__device__ __forceinline__ uint32_t koff(int r, int k) { return kmajor_off(r, k, kBK); }

// Column of the 1 in row i of the exact part R (-1: no R).
__device__ __forceinline__ int r_col(const LevelArgs& a, int i)
{
    if (a.rn < 0) return -1;
    if (a.rn == 0) return i;
    const int b = i / a.rn;
    const int bt = b + a.rsh < 3 ? b + a.rsh : 3;
    return bt * a.rn + (i - b * a.rn);
}

// Slice s of the tile into shared-memory stage `st` (hi/lo TF32 pairs).
__device__ __forceinline__ void load_slice(const LevelArgs& a, int m0, long n0, int k0, unsigned char* st)
{
    const int tid = threadIdx.x;
    // A: 128 rows x 32 K; thread -> (row tid/2, 16 consecutive K)
    {
        const int r = tid >> 1, kb = (tid & 1) * 16;
        const int i = m0 + r;
        double v[16];
        if (i < a.Np && k0 + kb < a.Np) {
            const double2* p = reinterpret_cast<const double2*>(a.P + (long)i * a.ldp + k0 + kb);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const double2 t = (k0 + kb + 2 * q < a.Np) ? p[q] : make_double2(0.0, 0.0);
                v[2 * q] = t.x;
                v[2 * q + 1] = t.y;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = 0.0;
        }
        // P - R: the tensor cores only see the small remainder
        const int rc = i < a.Np ? r_col(a, i) - (k0 + kb) : -1;
#pragma unroll
        for (int q = 0; q < 16; ++q)
            if (q == rc) v[q] -= 1.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float4 h, l;
            split_tf32((float)v[4 * c + 0], h.x, l.x);
            split_tf32((float)v[4 * c + 1], h.y, l.y);
            split_tf32((float)v[4 * c + 2], h.z, l.z);
            split_tf32((float)v[4 * c + 3], h.w, l.w);
            // the FP32 rounding of x is itself split off: x - (float)x is
            // below 2^-24 |x| and is dropped, as in every 3xTF32 scheme
            *reinterpret_cast<float4*>(st + koff(r, kb + 4 * c)) = h;
            *reinterpret_cast<float4*>(st + kAHalf + koff(r, kb + 4 * c)) = l;
        }
    }
    // B: 64 vectors x 32 K; thread -> (vector tid/4, 8 consecutive K)
    {
        const int c = tid >> 2, kb = (tid & 3) * 8;
        const long g = n0 + c;
        double v[8];
        if (g < a.ncols && k0 + kb < a.Np) {
            const double2* p = reinterpret_cast<const double2*>(a.src + g * a.src_gs + k0 + kb);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double2 t = (k0 + kb + 2 * q < a.Np) ? p[q] : make_double2(0.0, 0.0);
                v[2 * q] = t.x;
                v[2 * q + 1] = t.y;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = 0.0;
        }
        unsigned char* b = st + 2 * kAHalf;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            float4 h, l;
            split_tf32((float)v[4 * q + 0], h.x, l.x);
            split_tf32((float)v[4 * q + 1], h.y, l.y);
            split_tf32((float)v[4 * q + 2], h.z, l.z);
            split_tf32((float)v[4 * q + 3], h.w, l.w);
            *reinterpret_cast<float4*>(b + koff(c, kb + 4 * q)) = h;
            *reinterpret_cast<float4*>(b + kBHalf + koff(c, kb + 4 * q)) = l;
        }
    }
}

// Thread 0: the 3xTF32 MMAs of one staged slice into TMEM column base `d`.
__device__ __forceinline__ void issue_slice(uint32_t d, uint32_t st)
{
    constexpr uint32_t SBO = kBK * 32;  // 8-row groups
    const uint64_t ah = make_desc(st, 128, SBO), al = make_desc(st + kAHalf, 128, SBO);
    const uint64_t bh = make_desc(st + 2 * kAHalf, 128, SBO), bl = make_desc(st + 2 * kAHalf + kBHalf, 128, SBO);
    const uint64_t A[3] = {ah, ah, al};
    const uint64_t B[3] = {bh, bl, bh};
    constexpr uint32_t idesc = make_idesc(kBM, kBN);
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int s = 0; s < kBK / 8; ++s)
            mma_tf32(d, A[q] + (uint64_t)(s * 16), B[q] + (uint64_t)(s * 16), idesc, (q == 0 && s == 0) ? 0u : 1u);
}

// Drain TMEM accumulator `d` (this warp's 32 lanes, 32 columns) into FP64.
__device__ __forceinline__ void drain(uint32_t taddr, double (&acc)[32])
{
    uint32_t r[32];
    tmem_ld32(taddr, r);
    tmem_wait_ld();
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[j] += (double)__uint_as_float(r[j]);
}

__device__ void tc_tile(const LevelArgs& a, long tile, unsigned char* sm, uint64_t* bar, uint32_t tbase,
                        uint32_t& phase, int* status)
{
    const int mt = (a.Np + kBM - 1) / kBM;
    const int m0 = (int)(tile % mt) * kBM;
    const long n0 = (tile / mt) * kBN;
    const int nk = (a.Np + kBK - 1) / kBK;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int quarter = warp & 3, half = warp >> 2;
    const uint32_t lane_addr = (uint32_t)(32 * quarter) << 16;
    const uint32_t base = smem_u32(sm);
    double acc[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[j] = 0.0;

    load_slice(a, m0, n0, 0, sm);
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
        fence_after_sync();
        issue_slice(tbase, base);
        mma_commit(bar);
    }
    for (int s = 0; s < nk; ++s) {
        if (s + 1 < nk) load_slice(a, m0, n0, (s + 1) * kBK, sm + ((s + 1) & 1) * kStage);
        // MMAs of slice s done: its stage may be refilled, its accumulator read
        if (!mbar_wait(bar, phase, kWaitLimit) && lane == 0) atomicExch(status, 1);
        phase ^= 1u;
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        if (threadIdx.x == 0 && s + 1 < nk) {
            fence_after_sync();
            issue_slice(tbase + (uint32_t)(((s + 1) & 1) * kBN), base + ((s + 1) & 1) * kStage);
            mma_commit(bar);
        }
        fence_after_sync();
        drain(tbase + lane_addr + (uint32_t)((s & 1) * kBN + half * 32), acc);
    }
    // results: row i of P, vectors g = n0 + 32 half + j
    const long i = m0 + 32 * quarter + lane;
    if (i < a.Np) {
        const int rc = r_col(a, (int)i);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const long g = n0 + 32 * half + j;
            if (g < a.ncols) {
                double v = acc[j];
                if (rc >= 0) v += a.src[g * a.src_gs + rc];  // R v, exact
                if (a.acc) v += a.acc[g * a.acc_gs + i * a.acc_is];
                a.dst[g * a.dst_gs + i * a.dst_is] = v;
            }
        }
    }
    // every thread's TMEM reads are complete before the next tile's MMAs
    fence_before_sync();
    __syncthreads();
}

// Persistent grouped kernel: CTAs walk the tiles of all entries.
__global__ void __launch_bounds__(kThreads, 1) k_level_tc(const LevelArgs* __restrict__ args,
                                                          const long* __restrict__ start, int nent, long tiles,
                                                          int* status)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 2 * kStage);
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + 2 * kStage + 16);
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    if ((threadIdx.x >> 5) == 0) tmem_alloc(slot, kTmemCols);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = *slot;
    uint32_t phase = 0;
    for (long t = blockIdx.x; t < tiles; t += gridDim.x) {
        int lo = 0, hi = nent - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (start[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const LevelArgs a = args[lo];
        tc_tile(a, t - start[lo], sm, bar, tbase, phase, status);
    }
    fence_after_sync();
    if ((threadIdx.x >> 5) == 0) tmem_dealloc(tbase, kTmemCols);
}

}  // namespace

long level_tc_tiles(const LevelArgs& a)
{
    return (long)((a.Np + kBM - 1) / kBM) * ((a.ncols + kBN - 1) / kBN);
}

bool level_tc_supported(const LevelArgs& a)
{
    // K-contiguous FP64 sources with 16-byte aligned rows, no in-place copy
    return a.cpy == nullptr && a.src_ks == 1 && (a.src_gs % 2) == 0 && (a.ldp % 2) == 0 && (a.Np % 8) == 0 &&
           a.Np > 64 && a.Np <= 1024 && (reinterpret_cast<uintptr_t>(a.src) & 15) == 0 &&
           (reinterpret_cast<uintptr_t>(a.P) & 15) == 0;
}

void launch_level_tc(const LevelArgs* dArgs, const long* dStart, int nent, long tiles, int sms, int* status,
                     cudaStream_t s)
{
    if (nent <= 0 || tiles <= 0) return;
    static bool attr_set = false;
    if (!attr_set) {
        PARODE_CUDA(cudaFuncSetAttribute(k_level_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
        attr_set = true;
    }
    const unsigned grid = (unsigned)std::min<long>(tiles, sms);
    k_level_tc<<<grid, kThreads, kSmem, s>>>(dArgs, dStart, nent, tiles, status);
    PARODE_CUDA(cudaGetLastError());
}

}  // namespace parode
