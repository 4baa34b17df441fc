// kernels_resp_tc.cu -- the mixed-precision (3xTF32, tcgen05) GEMMs of the
// block-response leaf: D = W x [sample windows], for the block aggregates
// (W's last NP rows) and the window part of the outputs (its B p output rows).
//
// The windows are the input samples read in place (window b starts
// `block_stride` samples after window b - 1; consecutive windows overlap), so
// the GEMM's N dimension walks the blocks and K the window.  The samples come
// pre-split into two TF32 planes (hi, lo = TF32(x - hi)) written by the
// sampler, so a K slice of 128 windows x 16 K arrives as one TMA box per
// plane, 64-byte swizzled, and goes to the tensor cores unconverted.  W is
// split once per plan into TF32 hi/lo blocks of 128 rows x 16 K in the MMA's
// no-swizzle K-major layout (k_split), one bulk copy per plane and slice.
//
// Tiles are 128 rows of W x 128 windows; K runs in slices of 16.  Warp roles
// around a ring of six 32 KB stages:
//   warp 0      producer: per slice the A hi/lo bulk copies (valid rows) and the
//               B hi/lo TMA boxes, completing on the stage's `full` mbarrier;
//   warp 1      one thread issues hi*hi into one of two TMEM drain buffers and
//               hi*lo + lo*hi into the tile's correction buffer, commits the
//               stage back to the producer and, after every kDrain slices,
//               the drain buffer to the epilogue;
//   warps 2-9   epilogue: two warps per TMEM lane quarter, one per half of the
//               tile's 128 columns; per drain unit FP32 -> FP64 running sums
//               in registers, after the tile's last unit also the corrections,
//               then the stores (rows of W at consecutive addresses of y or G).
// The hi*hi chains stay kDrain slices long (FP32 accumulation error grows
// with the chain; the FP64 sums across units do not).  Every wait is bounded;
// a wait that gives up sets the status word and an abort flag that makes
// every role leave its loop, and the CTA drains its copies (bounded) before
// it frees its TMEM and exits.
//
// The single-pass form (TF32 precision) reads only the hi halves and issues
// only hi*hi: a third of the tensor work and half of the operand traffic,
// with the TF32 rounding of both operands (about 2^-11 relative) left in.
#include "common.h"
#include "device_common.cuh"
#include "kernels.h"
#include "tc05.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

namespace parode {

namespace {

using namespace tc05;

constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;  // producer, MMA, epilogue
constexpr int kBM = 128, kBN = 128, kBK = 16;
constexpr int kS = 6;                          // ring stages
constexpr uint32_t kAHalf = kBM * kBK * 4;     // A hi (or lo) per slice: 8 KB
constexpr uint32_t kABlock = 2 * kAHalf;       // pre-split A block (hi | lo), as k_split writes it
constexpr uint32_t kBHalf = kBN * kBK * 4;     // B hi (or lo): 8 KB, 128 rows x 64 B, 64B swizzle
constexpr uint32_t kOffB = kABlock;
constexpr uint32_t kStage = kABlock + 2 * kBHalf;  // 32 KB
constexpr int kAcc = 2;                             // hi*hi drain buffers of kBN columns
// barriers: full[kS], empty[kS], acc_full[kAcc], acc_empty[kAcc], corr_empty[2]
constexpr uint32_t kNumBars = 2 * kS + 2 * kAcc + 2;
constexpr uint32_t kOffBars = kS * kStage;
constexpr uint32_t kOffSlot = kOffBars + 8 * kNumBars;
constexpr uint32_t kSmem = kOffSlot + 16;
constexpr uint32_t kTmemCols = 512;  // 2 drain buffers + 2 correction buffers of 128 columns
constexpr int kDrain = 8;
constexpr long long kWaitLimit = 1LL << 31;

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// 2D tensor load (this GPU's memory, no multicast) of the box at (x, y).
__device__ __forceinline__ void tma_load_2d(void* dst, const void* map, int x, int y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// SMEM descriptor of a K-major operand in the 64-byte swizzle layout the TMA
// writes with CU_TENSOR_MAP_SWIZZLE_64B: rows of 64 bytes (16 tf32 of K),
// 8-row groups 512 bytes apart; the leading offset is unused (1).
__device__ __forceinline__ uint64_t make_desc_sw64(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)((512 >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // version
    d |= (uint64_t)4 << 61;  // 64-byte swizzle
    return d;
}

__device__ __forceinline__ bool role_wait(uint64_t* bar, uint32_t parity, volatile int* abort, int* status)
{
    if (*abort) return false;
    if (mbar_wait(bar, parity, kWaitLimit)) return true;
    *abort = 1;
    atomicExch(status, 1);
    return false;
}


// Tile sequence of one CTA (entries found by a forward scan); the entry's
// arguments are read from global memory where used, not held in registers.
struct Cursor {
    const RespArgs* args;
    const long* start;
    int nent;
    int e;
    long next, end;
    __device__ void init(const RespArgs* ar, const long* st, int n, long t0, long t1)
    {
        args = ar;
        start = st;
        nent = n;
        e = 0;
        int hi = nent - 1;
        while (e < hi) {
            const int mid = (e + hi + 1) >> 1;
            if (start[mid] <= t0) e = mid;
            else hi = mid - 1;
        }
        end = t1;
        next = e + 1 < nent ? start[e + 1] : t1;
    }
    __device__ long seek(long t)
    {
        while (t >= next && e + 1 < nent) {
            ++e;
            next = e + 1 < nent ? start[e + 1] : end;
        }
        return t - start[e];
    }
    __device__ const RespArgs& a() const { return args[e]; }
};

__device__ __forceinline__ void tile_coords(const RespArgs& a, long lt, int& mi, int& m0, long& n0, int& nk)
{
    const int mt = (a.rows + kBM - 1) / kBM;
    mi = (int)(lt % mt);
    m0 = mi * kBM;
    n0 = (lt / mt) * kBN;
    nk = (a.K + kBK - 1) / kBK;
}

// kOne: the single-pass form, hi*hi only (no lo planes are read and no
// correction buffers used).
template <bool kOne>
__global__ void __launch_bounds__(kThreads, 1) k_resp_tc(const RespArgs* __restrict__ args,
                                                         const long* __restrict__ start, int nent,
                                                         const long* __restrict__ cta, int* status)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kOffBars);
    uint64_t* full = bars;
    uint64_t* empty = bars + kS;
    uint64_t* acc_full = bars + 2 * kS;
    uint64_t* acc_empty = bars + 2 * kS + kAcc;
    uint64_t* corr_empty = bars + 2 * kS + 2 * kAcc;
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + kOffSlot);
    volatile int* abort = reinterpret_cast<volatile int*>(sm + kOffSlot + 8);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int q = 0; q < kS; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], 1);
        }
        for (int q = 0; q < kAcc; ++q) {
            mbar_init(&acc_full[q], 1);
            mbar_init(&acc_empty[q], kEpiWarps);
        }
        for (int q = 0; q < 2; ++q) mbar_init(&corr_empty[q], kEpiWarps);
        *abort = 0;
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(slot, kTmemCols);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    // launched as a dependent of the sample kernel: the set-up above overlaps
    // its tail, the samples are read (and the outputs written) after this
    grid_dep_wait();
    const uint32_t tbase = *slot;
    const long t0 = cta[blockIdx.x], t1 = cta[blockIdx.x + 1];

    if (warp == 0) {
        // ---------------- producer ----------------
        Cursor c;
        c.init(args, start, nent, t0, t1);
        // ring position of the next slice: stage st in its use of parity ph
        // (kept as counters: a division by the six stages per slice cost the
        // single issuing threads more than the tensor work of a slice)
        int st = 0;
        uint32_t ph = 0;
        long slices = 0;
        for (long t = t0; t < t1 && !*abort; ++t) {
            const long lt = c.seek(t);
            const RespArgs& a = c.a();
            int mi, m0, nk;
            long n0;
            tile_coords(a, lt, mi, m0, n0, nk);
            const int rowsv = a.rows - m0 < kBM ? a.rows - m0 : kBM;
            const uint32_t abytes = (uint32_t)((rowsv + 7) / 8) * (uint32_t)(kBK * 32);
            for (int s = 0; s < nk && !*abort; ++s) {
                if (slices >= kS && !role_wait(&empty[st], ph ^ 1u, abort, status)) break;
                unsigned char* stg = sm + st * kStage;
                // test hook: CTA 0 issues nothing for its first slice
                const bool withhold = a.fault_withhold && blockIdx.x == 0 && slices == 0;
                if (lane == 0 && !withhold) {
                    const int sr = s;
                    const unsigned char* ab =
                        reinterpret_cast<const unsigned char*>(a.Ps) + ((size_t)mi * nk + sr) * kABlock;
                    const unsigned char* maps = reinterpret_cast<const unsigned char*>(a.maps);
                    mbar_arrive_tx(&full[st], kOne ? abytes + kBHalf : 2 * abytes + 2 * kBHalf);
                    bulk_g2s(stg, ab, abytes, &full[st]);
                    tma_load_2d(stg + kOffB, maps, sr * kBK, (int)n0, &full[st]);
                    if (!kOne) {
                        bulk_g2s(stg + kAHalf, ab + kAHalf, abytes, &full[st]);
                        tma_load_2d(stg + kOffB + kBHalf, maps + 128, sr * kBK, (int)n0, &full[st]);
                    }
                }
                __syncwarp();
                ++slices;
                if (++st == kS) {
                    st = 0;
                    ph ^= 1u;
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            Cursor c;
            c.init(args, start, nent, t0, t1);
            long u = 0, tt = 0;
            int st = 0;  // ring stage of the next slice and the parity of its fill
            uint32_t ph = 0;
            constexpr uint32_t SBO = kBK * 32;
            constexpr uint32_t idesc = make_idesc(kBM, kBN);
            bool ok = true;
            for (long t = t0; t < t1 && ok && !*abort; ++t, ++tt) {
                const long lt = c.seek(t);
                int mi, m0, nk;
                long n0;
                tile_coords(c.a(), lt, mi, m0, n0, nk);
                int ab = 0;
                uint32_t d = 0;
                const uint32_t dc = tbase + (uint32_t)(kAcc * kBN + (tt & 1) * kBN);
                if (!kOne && tt >= 2 &&
                    !role_wait(&corr_empty[tt & 1], (uint32_t)(((tt >> 1) - 1) & 1), abort, status)) {
                    ok = false;
                    break;
                }
                for (int s = 0; s < nk; ++s) {
                    if (s % kDrain == 0) {
                        ab = (int)(u % kAcc);
                        const long ause = u / kAcc;
                        if (ause >= 1 && !role_wait(&acc_empty[ab], (uint32_t)((ause - 1) & 1), abort, status)) {
                            ok = false;
                            break;
                        }
                        fence_after_sync();
                        d = tbase + (uint32_t)(ab * kBN);
                    }
                    if (!role_wait(&full[st], ph, abort, status)) {
                        ok = false;
                        break;
                    }
                    fence_after_sync();
                    const uint32_t stg = smem_u32(sm + st * kStage);
                    const uint64_t ah = make_desc(stg, 128, SBO), al = make_desc(stg + kAHalf, 128, SBO);
                    const uint64_t bh = make_desc_sw64(stg + kOffB), bl = make_desc_sw64(stg + kOffB + kBHalf);
                    const uint64_t A[3] = {ah, ah, al};
                    const uint64_t B[3] = {bh, bl, bh};
#pragma unroll
                    for (int q = 0; q < (kOne ? 1 : 3); ++q)
#pragma unroll
                        for (int k = 0; k < kBK / 8; ++k)
                            // A: next 8 K = two 16-byte chunks (256 bytes on); B: 32 bytes on in the swizzled row
                            mma_tf32(q == 0 ? d : dc, A[q] + (uint64_t)(k * 16), B[q] + (uint64_t)(k * 2), idesc,
                                     ((q == 0 && s % kDrain == 0) || (q == 1 && s == 0)) && k == 0 ? 0u : 1u);
                    mma_commit(&empty[st]);
                    if (++st == kS) {
                        st = 0;
                        ph ^= 1u;
                    }
                    if (s % kDrain == kDrain - 1 || s == nk - 1) {
                        mma_commit(&acc_full[ab]);
                        ++u;
                    }
                }
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue (warps 2-9) ----------------
        const int quarter = warp & 3;
        const int half = (warp - 2) >> 2;  // which 64 columns of the tile
        Cursor c;
        c.init(args, start, nent, t0, t1);
        long u = 0, tt = 0;
        bool ok = true;
        for (long t = t0; t < t1 && ok && !*abort; ++t, ++tt) {
            const long lt = c.seek(t);
            const RespArgs& a = c.a();
            int mi, m0, nk;
            long n0;
            tile_coords(a, lt, mi, m0, n0, nk);
            double sum[64];
#pragma unroll
            for (int q = 0; q < 64; ++q) sum[q] = 0.0;
            const int units = (nk + kDrain - 1) / kDrain;
            const uint32_t lanes = (uint32_t)(32 * quarter) << 16;
            for (int v = 0; v < units; ++v, ++u) {
                const int ab = (int)(u % kAcc);
                if (!role_wait(&acc_full[ab], (uint32_t)((u / kAcc) & 1), abort, status)) {
                    ok = false;
                    break;
                }
                fence_after_sync();
                // this unit's hi*hi, then at the tile's last unit the corrections,
                // 16 columns per load (few registers beside the 64 sums)
                const uint32_t cu = (uint32_t)(ab * kBN + half * 64);
                const uint32_t cc = (uint32_t)(kAcc * kBN + (tt & 1) * kBN + half * 64);
                const int passes = (!kOne && v == units - 1) ? 2 : 1;
                for (int ps = 0; ps < passes; ++ps) {
                    const uint32_t c0 = ps == 0 ? cu : cc;
#pragma unroll
                    for (int g = 0; g < 4; ++g) {
                        uint32_t r[16];
                        tmem_ld16(tbase + lanes + c0 + (uint32_t)(16 * g), r);
                        tmem_wait_ld();
#pragma unroll
                        for (int q = 0; q < 16; ++q) sum[16 * g + q] += (double)__uint_as_float(r[q]);
                    }
                }
                fence_before_sync();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&acc_empty[ab]);
                    if (!kOne && v == units - 1) mbar_arrive(&corr_empty[tt & 1]);
                }
            }
            if (!ok) break;
            const long i = m0 + 32 * quarter + lane;
            if (i < a.rows) {
                const long cbase = n0 + half * 64;
                int nvt = (int)std::max<long>(0, std::min<long>(64, a.ncols - cbase));
                if (a.dst_limit >= 0) {
                    const long lim = a.dst_limit - i * a.dst_is;
                    const long gmax = lim <= 0 ? cbase : (lim + a.dst_gs - 1) / a.dst_gs;
                    nvt = (int)std::max<long>(0, std::min<long>(nvt, gmax - cbase));
                }
                double* drow = a.dst + i * a.dst_is + cbase * a.dst_gs;
#pragma unroll
                for (int q = 0; q < 64; ++q)
                    if (q < nvt) drow[(long)q * a.dst_gs] = sum[q];
            }
        }
    }

    __syncthreads();
    if (*abort && threadIdx.x == 0) {
        for (int q = 0; q < kS; ++q) mbar_wait(&full[q], 0, 1 << 20);
    }
    fence_after_sync();
    if (warp == 0) tmem_dealloc(tbase, kTmemCols);
}

}  // namespace

long resp_tc_tiles(const RespArgs& a) { return (long)((a.rows + kBM - 1) / kBM) * ((a.ncols + kBN - 1) / kBN); }

std::vector<long> resp_tc_ranges(const std::vector<RespArgs>& ents, int ctas)
{
    std::vector<double> cost;
    double total = 0;
    for (const RespArgs& a : ents) {
        const long n = resp_tc_tiles(a);
        const double c = (a.K + kBK - 1) / kBK + 2.0;
        for (long t = 0; t < n; ++t) cost.push_back(c);
        total += c * n;
    }
    std::vector<long> r(ctas + 1, (long)cost.size());
    r[0] = 0;
    double acc = 0;
    int k = 1;
    for (long t = 0; t < (long)cost.size() && k < ctas; ++t) {
        acc += cost[t];
        while (k < ctas && acc >= total * k / ctas) r[k++] = t + 1;
    }
    for (; k < ctas; ++k) r[k] = (long)cost.size();
    return r;
}

void resp_encode_plane_maps(const float* hi, const float* lo, long ncols, int K, long block_stride, void* out)
{
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            fn = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if (!encode) throw Error(kDeviceError, "cuTensorMapEncodeTiled unavailable");
    const float* planes[2] = {hi, lo};
    for (int p = 0; p < (lo ? 2 : 1); ++p) {
        if ((reinterpret_cast<uintptr_t>(planes[p]) & 15) || ((block_stride * 4) & 15))
            throw Error(kInvalidArgument, "sample plane map: 16-byte alignment");
        CUtensorMap* m = reinterpret_cast<CUtensorMap*>(static_cast<unsigned char*>(out) + 128 * p);
        // K (padded to whole slices so that the last slice's box stays on the
        // map) x windows; rows overlap (block_stride < K)
        const cuuint64_t dims[2] = {(cuuint64_t)((K + kBK - 1) / kBK * kBK), (cuuint64_t)ncols};
        const cuuint64_t strides[1] = {(cuuint64_t)block_stride * 4};
        const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)kBN};
        const cuuint32_t estr[2] = {1, 1};
        CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(planes[p]), dims, strides, box,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) throw Error(kDeviceError, "cuTensorMapEncodeTiled (sample planes) failed");
    }
}

void launch_resp_tc(const RespArgs* dArgs, const long* dStart, int nent, const long* dCta, int ctas, int* status,
                    bool one_pass, cudaStream_t s)
{
    if (nent <= 0 || ctas <= 0) return;
    if (one_pass) {
        PARODE_CUDA(cudaFuncSetAttribute(k_resp_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
        launch_dependent(k_resp_tc<true>, (unsigned)ctas, kThreads, kSmem, s, dArgs, dStart, nent, dCta, status);
    } else {
        PARODE_CUDA(cudaFuncSetAttribute(k_resp_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
        launch_dependent(k_resp_tc<false>, (unsigned)ctas, kThreads, kSmem, s, dArgs, dStart, nent, dCta, status);
    }
}

}  // namespace parode
