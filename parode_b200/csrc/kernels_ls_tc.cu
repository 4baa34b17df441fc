// kernels_ls_tc.cu -- mixed-precision (3xTF32 on tcgen05) level contraction
// of the level-synchronous scan, for scan dimensions above 64.
//
// One level computes dst(g, i) = sum_k P[i][k] src(g, k) + acc(g, i) for the
// columns g of the level (the reference's MVV up/down-sweep kernels,
// Kernels/MVVKernelScanUpsweep.cl:25-48, MVVKernelScanDownsweep.cl:25-48, as
// one contraction per level).  P rows sit on the MMA's M (128 per tile), the
// level's vectors on N (64 per tile), K runs over the scan dimension in
// slices of 16.
//
// Exact part: P = R + E with R an exact 0/1 matrix, one 1 per row (I for RK4,
// the companion shift S^(2^l) for ABM).  Only E goes through the tensor
// cores; R v is added in FP64 in the epilogue.  For the lower levels E is
// small (P_l = Phi^(2^l) is within about 2^l h |A| of R_l), so the TF32
// representation error and the FP32 accumulation in TMEM are relative to
// |E v|, far below |v|.
//
// E is split once per level (k_split) into TF32 hi/lo blocks laid out as the
// MMA reads them (K-major, no swizzle).  The contraction kernel is
// warp-specialised around a ring of shared-memory stages:
//   warp 0      producer: per slice one bulk copy (TMA engine) of the 16 KB A
//               block and one 2D tensor load of B (64 vectors x 16 K, FP64),
//               completing on the stage's `full` mbarrier;
//   warps 2-3   converters: B FP64 -> TF32 hi/lo in the canonical layout,
//               then arrive on `conv`;
//   warp 1      one thread issues hi*hi into one of kAcc TMEM accumulators
//               and hi*lo + lo*hi into the tile's correction accumulator,
//               commits to `empty` (stage free) and, after every kDrain
//               slices (a drain unit), to `acc_full`;
//   warps 4-7   epilogue: per drain unit TMEM (FP32) -> FP64 running sums in
//               registers, arrive `acc_empty`; after a tile's last unit the
//               corrections too (arrive `corr_empty`), + R v + acc, store.
// The drains keep each FP32 accumulation chain of hi*hi to kDrain slices
// (2 kDrain MMAs), and the two corrections accumulate apart, over the whole
// tile, in a second accumulator read once per tile (they are about 2^-11 of
// hi*hi, so their FP32 roundings are that much smaller): the tensor cores'
// FP32 accumulation error grows with the chain, the FP64 sums across units
// do not.
// Every wait is bounded; a wait that gives up sets the status word and an
// abort flag that makes every role leave its loop.
#include "common.h"
#include "kernels.h"
#include "tc05.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

namespace parode {

namespace {

using namespace tc05;

constexpr int kThreads = 256;
constexpr int kBM = 128, kBN = 64, kBK = 16;
constexpr int kS = 5;                        // ring stages
constexpr uint32_t kAHalf = kBM * kBK * 4;   // A hi (or lo) per slice: 8 KB
constexpr uint32_t kBHalf = kBN * kBK * 4;   // B hi (or lo): 4 KB
constexpr uint32_t kABlock = 2 * kAHalf;     // pre-split A block (hi | lo)
constexpr uint32_t kBRaw = kBN * kBK * 8;    // B FP64, vector v at v * 128 bytes
constexpr uint32_t kOffRaw = kABlock;
constexpr uint32_t kOffConvB = kABlock + kBRaw;
constexpr uint32_t kStage = kABlock + kBRaw + 2 * kBHalf;  // 32 KB
constexpr uint32_t kOffBars = kS * kStage;
// TMEM: kAcc hi*hi drain buffers of kBN columns, then 2 per-tile correction buffers
constexpr int kAcc = 4;
// barriers: full[kS], conv[kS], empty[kS], acc_full[kAcc], acc_empty[kAcc], corr_empty[2]
constexpr uint32_t kNumBars = 3 * kS + 2 * kAcc + 2;
constexpr uint32_t kOffSlot = kOffBars + 8 * kNumBars;
constexpr uint32_t kSmem = kOffSlot + 16;
constexpr uint32_t kTmemCols = 512;  // hi*hi: kAcc drain buffers; corrections: 2 tile buffers (384 used)
constexpr int kDrain = 8;  // K slices per FP32 accumulation chain
constexpr long long kWaitLimit = 1LL << 31;

__host__ __device__ constexpr uint32_t koff(int r, int k) { return kmajor_off(r, k, kBK); }

// K elements of slice s (16, or fewer in the last slice).
__device__ __forceinline__ int slice_len(int K, int s)
{
    const int rest = K - s * kBK;
    return rest < kBK ? rest : kBK;
}

// Column of the 1 in row i of the exact part R (-1: no R).
__host__ __device__ inline int r_col(const LevelArgs& a, int i)
{
    if (a.rn < 0) return -1;
    if (a.rn == 0) return i;
    const int b = i / a.rn;
    const int bt = b + a.rsh < 3 ? b + a.rsh : 3;
    return bt * a.rn + (i - b * a.rn);
}

// ---------------------------------------------------------------------------
// E = P - R split into TF32 hi/lo blocks: block (mt, s) = rows [128 mt, +128),
// K [16 s, +16), hi then lo, each in the canonical K-major layout.  P is
// rows x K (level_rows, level_k), zero-padded to whole blocks.
// ---------------------------------------------------------------------------
__global__ void k_split(const LevelArgs* __restrict__ args)
{
    const LevelArgs& a = args[blockIdx.y];
    const int rows = level_rows(a), K = level_k(a);
    const int mt = (rows + kBM - 1) / kBM, nk = (K + kBK - 1) / kBK;
    const long total = (long)mt * kBM * nk * kBK;  // padded elements
    unsigned char* out = reinterpret_cast<unsigned char*>(const_cast<float*>(a.Ps));
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long kp = (long)nk * kBK;
        const int i = (int)(e / kp), k = (int)(e - (long)i * kp);
        double v = 0.0;
        if (i < rows && k < K) {
            v = a.P[(long)i * a.ldp + k];
            if (k == r_col(a, i)) v -= 1.0;
        }
        float hi, lo;
        split_tf32((float)v, hi, lo);
        const int mi = i / kBM, s = k / kBK;
        unsigned char* blk = out + ((size_t)mi * nk + s) * kABlock;
        *reinterpret_cast<float*>(blk + koff(i - mi * kBM, k - s * kBK)) = hi;
        *reinterpret_cast<float*>(blk + kAHalf + koff(i - mi * kBM, k - s * kBK)) = lo;
    }
}

// ---- mbarrier / bulk-copy helpers --------------------------------------------

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bulk copy (TMA engine, no tensor map) of `bytes` (multiple of 16, both
// addresses 16-byte aligned) into this CTA's shared memory.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// 2D tensor load (TMA, this GPU's memory, no multicast) of the box at
// coordinates (x, y) of the tensor map at device address `map`.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* map, int x, int y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Bounded wait shared by all roles: on time-out, record it and raise abort.
__device__ __forceinline__ bool role_wait(uint64_t* bar, uint32_t parity, volatile int* abort, int* status)
{
    if (*abort) return false;
    if (mbar_wait(bar, parity, kWaitLimit)) return true;
    *abort = 1;
    atomicExch(status, 1);
    return false;
}

// Tile sequence of one CTA: entries found by a forward scan.
struct Cursor {
    const LevelArgs* args;
    const long* start;
    int nent;
    int e;
    long next;
    LevelArgs a;
    __device__ void init(const LevelArgs* ar, const long* st, int n, long t0, long t1)
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
        a = args[e];
        next = e + 1 < nent ? start[e + 1] : t1;
        end = t1;
    }
    long end;
    // entry of tile t (t non-decreasing); returns the tile index inside it
    __device__ long seek(long t)
    {
        while (t >= next && e + 1 < nent) {
            ++e;
            a = args[e];
            next = e + 1 < nent ? start[e + 1] : end;
        }
        return t - start[e];
    }
};

__device__ __forceinline__ void tile_coords(const LevelArgs& a, long lt, int& mi, int& m0, long& n0, int& nk)
{
    const int mt = (level_rows(a) + kBM - 1) / kBM;
    mi = (int)(lt % mt);
    m0 = mi * kBM;
    n0 = (lt / mt) * kBN;
    nk = (level_k(a) + kBK - 1) / kBK;
}


// Persistent grouped kernel: CTA c walks tiles [cta[c], cta[c+1]) in order.
__global__ void __launch_bounds__(kThreads, 1) k_level_tc(const LevelArgs* __restrict__ args,
                                                          const long* __restrict__ start, int nent,
                                                          const long* __restrict__ cta, int* status)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kOffBars);
    uint64_t* full = bars;
    uint64_t* conv = bars + kS;
    uint64_t* empty = bars + 2 * kS;
    uint64_t* acc_full = bars + 3 * kS;
    uint64_t* acc_empty = bars + 3 * kS + kAcc;
    uint64_t* corr_empty = bars + 3 * kS + 2 * kAcc;
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + kOffSlot);
    volatile int* abort = reinterpret_cast<volatile int*>(sm + kOffSlot + 8);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int q = 0; q < kS; ++q) {
            mbar_init(&full[q], 1);  // the producer's expect-tx arrive; the copies complete the bytes
            mbar_init(&conv[q], 2);
            mbar_init(&empty[q], 1);
        }
        for (int q = 0; q < kAcc; ++q) {
            mbar_init(&acc_full[q], 1);
            mbar_init(&acc_empty[q], 4);
        }
        for (int q = 0; q < 2; ++q) mbar_init(&corr_empty[q], 4);
        *abort = 0;
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(slot, kTmemCols);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = *slot;
    const long t0 = cta[blockIdx.x], t1 = cta[blockIdx.x + 1];

    if (warp == 0) {
        // ---------------- producer ----------------
        Cursor c;
        c.init(args, start, nent, t0, t1);
        long j = 0;  // slice counter
        int pst = 0;  // its ring stage and the parity of that stage's use
        uint32_t pph = 0;
        for (long t = t0; t < t1 && !*abort; ++t) {
            const long lt = c.seek(t);
            const LevelArgs& a = c.a;
            int mi, m0, nk;
            long n0;
            tile_coords(a, lt, mi, m0, n0, nk);
            const int nv = (int)std::min<long>(kBN, a.ncols - n0);
            // the epilogue's acc rows of this tile into L2 ahead of time
            if (a.acc) {
                const int rows = level_rows(a) - m0 < kBM ? level_rows(a) - m0 : kBM;
                const int lines = (rows * 8 + 127) / 128;
                for (int q = lane; q < nv * lines; q += 32) {
                    const int v = q / lines, ln = q - v * lines;
                    const double* p = a.acc + (n0 + v) * a.acc_gs + (long)m0 * a.acc_is + ln * 16;
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
                }
            }
            for (int s = 0; s < nk && !*abort; ++s, ++j) {
                // ring position as counters (no per-slice division by kS)
                if (j >= kS && !role_wait(&empty[pst], pph ^ 1u, abort, status)) break;
                const int st = pst;
                unsigned char* stg = sm + st * kStage;
                // A: one 16 KB bulk copy; B: one 2D tensor load of 64 vectors x
                // 16 K (FP64; x = 16 s, a multiple of 16 bytes; the tails beyond
                // K or ncols are zero-filled by the TMA engine)
                // Only the M-tile's valid rows of A travel (8-row core-matrix
                // groups, hi and lo): the MMA's other rows read whatever the
                // stage held, and their results are never stored.
                // test hook: CTA 0 issues nothing for its first slice, so that
                // stage's waits run into their bound (no copy is in flight)
                const bool withhold = a.fault_withhold && blockIdx.x == 0 && j == 0;
                if (lane == 0 && !withhold) {
                    const int sr = s;
                    const int rowsv = level_rows(a) - m0 < kBM ? level_rows(a) - m0 : kBM;
                    const uint32_t abytes = (uint32_t)((rowsv + 7) / 8) * (uint32_t)(kBK * 32);
                    const unsigned char* ab = reinterpret_cast<const unsigned char*>(a.Ps) + ((size_t)mi * nk + sr) * kABlock;
                    mbar_arrive_tx(&full[st], 2 * abytes + kBRaw);
                    bulk_g2s(stg, ab, abytes, &full[st]);
                    bulk_g2s(stg + kAHalf, ab + kAHalf, abytes, &full[st]);
                    tma_load_2d(stg + kOffRaw, a.src_map, sr * kBK, (int)n0, &full[st]);
                }
                __syncwarp();
                if (++pst == kS) {
                    pst = 0;
                    pph ^= 1u;
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            Cursor c;
            c.init(args, start, nent, t0, t1);
            long u = 0, tt = 0;  // drain-unit and tile counters
            int mst = 0;         // ring stage of the next slice and its fill parity
            uint32_t mph = 0;
            constexpr uint32_t SBO = kBK * 32;
            constexpr uint32_t idesc = make_idesc(kBM, kBN);
            bool ok = true;
            for (long t = t0; t < t1 && ok && !*abort; ++t, ++tt) {
                const long lt = c.seek(t);
                int mi, m0, nk;
                long n0;
                tile_coords(c.a, lt, mi, m0, n0, nk);
                int ab = 0;
                uint32_t d = 0;
                // the corrections accumulate over the whole tile, in the
                // tile-parity buffer, once the epilogue has read it two tiles ago
                const uint32_t dc = tbase + (uint32_t)(kAcc * kBN + (tt & 1) * kBN);
                if (tt >= 2 && !role_wait(&corr_empty[tt & 1], (uint32_t)(((tt >> 1) - 1) & 1), abort, status)) {
                    ok = false;
                    break;
                }
                for (int s = 0; s < nk; ++s) {
                    if (s % kDrain == 0) {
                        // a new drain unit: wait until the epilogue has read this accumulator
                        ab = (int)(u % kAcc);
                        const long ause = u / kAcc;
                        if (ause >= 1 && !role_wait(&acc_empty[ab], (uint32_t)((ause - 1) & 1), abort, status)) {
                            ok = false;
                            break;
                        }
                        fence_after_sync();
                        d = tbase + (uint32_t)(ab * kBN);
                    }
                    const int st = mst;
                    // A landed (bulk copy) and B converted
                    if (!role_wait(&full[st], mph, abort, status) || !role_wait(&conv[st], mph, abort, status)) {
                        ok = false;
                        break;
                    }
                    fence_after_sync();
                    const uint32_t stg = smem_u32(sm + st * kStage);
                    const uint64_t ah = make_desc(stg, 128, SBO), al = make_desc(stg + kAHalf, 128, SBO);
                    const uint64_t bh = make_desc(stg + kOffConvB, 128, SBO);
                    const uint64_t bl = make_desc(stg + kOffConvB + kBHalf, 128, SBO);
                    const uint64_t A[3] = {ah, ah, al};
                    const uint64_t B[3] = {bh, bl, bh};
                    // hi*hi into the drain unit's accumulator (K/8 FP32
                    // roundings per unit in the large sum), the two
                    // corrections (about 2^-11 smaller) into the tile's
                    // correction accumulator, read once at the tile's end
#pragma unroll
                    for (int q = 0; q < 3; ++q)
#pragma unroll
                        for (int k = 0; k < kBK / 8; ++k)
                            mma_tf32(q == 0 ? d : dc, A[q] + (uint64_t)(k * 16), B[q] + (uint64_t)(k * 16), idesc,
                                     ((q == 0 && s % kDrain == 0) || (q == 1 && s == 0)) && k == 0 ? 0u : 1u);
                    mma_commit(&empty[st]);
                    if (++mst == kS) {
                        mst = 0;
                        mph ^= 1u;
                    }
                    if (s % kDrain == kDrain - 1 || s == nk - 1) {
                        mma_commit(&acc_full[ab]);
                        ++u;
                    }
                }
            }
        }
        __syncwarp();
    } else if (warp == 2 || warp == 3) {
        // ---------------- converters (64 threads) ----------------
        const int ct = threadIdx.x - 64;
        Cursor c;
        c.init(args, start, nent, t0, t1);
        int cst = 0;  // ring stage of the next slice and its fill parity
        uint32_t cph = 0;
        for (long t = t0; t < t1 && !*abort; ++t) {
            const long lt = c.seek(t);
            const LevelArgs& a = c.a;
            int mi, m0, nk;
            long n0;
            tile_coords(a, lt, mi, m0, n0, nk);
            bool ok = true;
            for (int s = 0; s < nk; ++s) {
                const int st = cst;
                if (!role_wait(&full[st], cph, abort, status)) {
                    ok = false;
                    break;
                }
                unsigned char* stg = sm + st * kStage;
                const double* raw = reinterpret_cast<const double*>(stg + kOffRaw);
                const int kl = slice_len(level_k(a), s);
                // 64 vectors x kBK/4 chunks of 4 K; item w -> vector w / (kBK/4),
                // chunk w % (kBK/4): a warp reads whole vectors and writes
                // contiguous core-matrix rows
                constexpr int kChunks = kBK / 4;
#pragma unroll
                for (int q = 0; q < kChunks; ++q) {
                    const int w = ct + 64 * q;
                    const int v = w / kChunks, kc = (w % kChunks) * 4;
                    const bool ok = n0 + v < a.ncols && kc < kl;
                    const double2* p = reinterpret_cast<const double2*>(raw + v * kBK + kc);
                    const double2 x0 = ok ? p[0] : make_double2(0.0, 0.0);
                    const double2 x1 = ok ? p[1] : make_double2(0.0, 0.0);
                    float4 h, l;
                    split_tf32((float)x0.x, h.x, l.x);
                    split_tf32((float)x0.y, h.y, l.y);
                    split_tf32((float)x1.x, h.z, l.z);
                    split_tf32((float)x1.y, h.w, l.w);
                    *reinterpret_cast<float4*>(stg + kOffConvB + koff(v, kc)) = h;
                    *reinterpret_cast<float4*>(stg + kOffConvB + kBHalf + koff(v, kc)) = l;
                }
                fence_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(&conv[st]);
                if (++cst == kS) {
                    cst = 0;
                    cph ^= 1u;
                }
            }
            if (!ok) break;
        }
    } else {
        // ---------------- epilogue (warps 4-7: TMEM lane quarters 0-3) ----------------
        const int quarter = warp & 3;
        Cursor c;
        c.init(args, start, nent, t0, t1);
        long u = 0, tt = 0;  // drain units, tiles
        bool ok = true;
        for (long t = t0; t < t1 && ok && !*abort; ++t, ++tt) {
            const long lt = c.seek(t);
            const LevelArgs& a = c.a;
            int mi, m0, nk;
            long n0;
            tile_coords(a, lt, mi, m0, n0, nk);
            // FP64 sums of this thread's row over the tile's drain units
            double sum[kBN];
#pragma unroll
            for (int q = 0; q < kBN; ++q) sum[q] = 0.0;
            const int units = (nk + kDrain - 1) / kDrain;
            for (int v = 0; v < units; ++v, ++u) {
                const int ab = (int)(u % kAcc);
                if (!role_wait(&acc_full[ab], (uint32_t)((u / kAcc) & 1), abort, status)) {
                    ok = false;
                    break;
                }
                fence_after_sync();
                // hi*hi of this unit; at the tile's last unit also the corrections
                // (read before the arrive below, so a later arrive implies them)
                const int halves = v == units - 1 ? 4 : 2;
                for (int h = 0; h < halves; ++h) {
                    const uint32_t col = h < 2 ? (uint32_t)(ab * kBN + h * 32)
                                               : (uint32_t)(kAcc * kBN + (tt & 1) * kBN + (h - 2) * 32);
                    uint32_t r[32];
                    tmem_ld32(tbase + ((uint32_t)(32 * quarter) << 16) + col, r);
                    tmem_wait_ld();
#pragma unroll
                    for (int q = 0; q < 32; ++q) {
                        if (h & 1) sum[32 + q] += (double)__uint_as_float(r[q]);
                        else sum[q] += (double)__uint_as_float(r[q]);
                    }
                }
                fence_before_sync();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&acc_empty[ab]);
                    if (v == units - 1) mbar_arrive(&corr_empty[tt & 1]);
                }
            }
            if (!ok) break;
            const long i = m0 + 32 * quarter + lane;
            const int rows = level_rows(a);
            const int rc = i < rows ? r_col(a, (int)i) : -1;
            // loop-invariant fields in registers
            const double* srow = a.src + (rc >= 0 ? rc : 0);
            const long sgs = a.src_gs;
            const double* arow = a.acc ? a.acc + i * a.acc_is : nullptr;
            const long ags = a.acc_gs;
            double* drow = a.dst + i * a.dst_is;
            const long dgs = a.dst_gs;
            int nvt = (int)std::min<long>(kBN, a.ncols - n0);
            if (a.dst_limit >= 0 && i < rows) {
                // columns whose result offset g dgs + i dst_is reaches the limit are dropped
                const long lim = a.dst_limit - i * a.dst_is;
                const long gmax = lim <= 0 ? n0 : (lim + dgs - 1) / dgs;  // first dropped column
                nvt = (int)std::max<long>(0, std::min<long>(nvt, gmax - n0));
            }
            const bool live = i < rows;
            if (live) {
                // 16 columns at a time: all loads in flight before the sums
#pragma unroll
                for (int c0 = 0; c0 < kBN; c0 += 16) {
                    double xa[16], xs[16];
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) {
                        const bool in = c0 + jj < nvt;
                        const long g = n0 + c0 + jj;
                        xs[jj] = (in && rc >= 0) ? srow[g * sgs] : 0.0;  // R v, exact
                        xa[jj] = (in && arow) ? arow[g * ags] : 0.0;
                    }
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj)
                        if (c0 + jj < nvt) drow[(n0 + c0 + jj) * dgs] = (sum[c0 + jj] + xs[jj]) + xa[jj];
                }
            }
        }
    }

    // all roles done (or aborted); bulk copies of an aborted producer are
    // drained by waiting on their stages (bounded) before the CTA exits
    __syncthreads();
    if (*abort && threadIdx.x == 0) {
        for (int q = 0; q < kS; ++q) mbar_wait(&full[q], 0, 1 << 20);
    }
    fence_after_sync();
    if (warp == 0) tmem_dealloc(tbase, kTmemCols);
}

}  // namespace

long level_tc_tiles(const LevelArgs& a)
{
    return (long)((level_rows(a) + kBM - 1) / kBM) * ((a.ncols + kBN - 1) / kBN);
}

size_t gemm_split_bytes(int rows, int K)
{
    return (size_t)((rows + kBM - 1) / kBM) * ((K + kBK - 1) / kBK) * kABlock;
}

size_t level_split_bytes(int Np) { return gemm_split_bytes(Np, Np); }

bool level_tc_supported(const LevelArgs& a)
{
    // K-contiguous FP64 sources with 16-byte aligned rows, no in-place copy,
    // one source; square levels of scan dimension 72..1024, or general shapes
    const bool general = a.M > 0 || a.K > 0;
    return a.cpy == nullptr && a.K1 == 0 && a.src_ks == 1 && (a.src_gs % 2) == 0 && (a.ldp % 2) == 0 &&
           (reinterpret_cast<uintptr_t>(a.src) & 15) == 0 &&
           (general ? (level_rows(a) > 0 && level_k(a) > 0) : ((a.Np % 8) == 0 && a.Np > 64 && a.Np <= 1024));
}

void launch_level_split(const LevelArgs* dArgs, int nent, long max_elems, cudaStream_t s)
{
    if (nent <= 0) return;
    const long elems = max_elems;
    dim3 grid((unsigned)std::max<long>(1, std::min<long>((elems + 255) / 256, 512)), (unsigned)nent);
    k_split<<<grid, 256, 0, s>>>(dArgs);
    PARODE_CUDA(cudaGetLastError());
}

void launch_level_tc(const LevelArgs* dArgs, const long* dStart, int nent, const long* dCta, int ctas, int* status,
                     cudaStream_t s)
{
    if (nent <= 0 || ctas <= 0) return;
    // set on every launch: per device, and safe with several host threads
    PARODE_CUDA(cudaFuncSetAttribute(k_level_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
    k_level_tc<<<(unsigned)ctas, kThreads, kSmem, s>>>(dArgs, dStart, nent, dCta, status);
    PARODE_CUDA(cudaGetLastError());
}

void level_encode_src_map(const LevelArgs& a, void* out)
{
    // resolved once (thread-safe static initialisation)
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            fn = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if (!encode) throw Error(kDeviceError, "cuTensorMapEncodeTiled unavailable");
    if ((reinterpret_cast<uintptr_t>(a.src) & 15) || ((a.src_gs * 8) & 15))
        throw Error(kInvalidArgument, "source map: 16-byte alignment");
    CUtensorMap* m = static_cast<CUtensorMap*>(out);
    const cuuint64_t dims[2] = {(cuuint64_t)level_k(a), (cuuint64_t)a.ncols};
    const cuuint64_t strides[1] = {(cuuint64_t)a.src_gs * 8};
    const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)kBN};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(a.src), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(kDeviceError, "cuTensorMapEncodeTiled failed");
}

// Host: tile ranges of `ctas` CTAs with about equal work (a tile costs its
// K slices plus a fixed overhead).
std::vector<long> level_tc_ranges(const std::vector<LevelArgs>& ents, int ctas)
{
    std::vector<double> cost;
    double total = 0;
    for (const LevelArgs& a : ents) {
        const long n = level_tc_tiles(a);
        const double c = (level_k(a) + kBK - 1) / kBK + 2.0;
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

}  // namespace parode
