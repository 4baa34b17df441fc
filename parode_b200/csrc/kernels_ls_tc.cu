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
// Data path: E is split once per level (k_split) into TF32 hi/lo tiles laid
// out exactly as the MMA reads them (K-major, no swizzle), so a slice of A is
// a 16 KB block that cp.async copies straight into shared memory; the
// level's vectors (B) are loaded as FP64 into registers two slices ahead and
// split into hi/lo on the way to shared memory.  A 3-stage operand ring lets
// one thread issue hi*hi + hi*lo + lo*hi for slice s while the CTA fills
// slice s+1; completion of each slice's MMAs frees its stage (mbarrier).
#include "common.h"
#include "kernels.h"
#include "tc05.cuh"

#include <algorithm>

namespace parode {

namespace {

using namespace tc05;

constexpr int kThreads = 256;
constexpr int kBM = 128, kBN = 64, kBK = 16;
constexpr int kStages = 3;
constexpr uint32_t kAHalf = kBM * kBK * 4;  // A hi (or lo) per slice: 8 KB
constexpr uint32_t kBHalf = kBN * kBK * 4;  // B hi (or lo): 4 KB
constexpr uint32_t kABlock = 2 * kAHalf;    // one pre-split A block (hi | lo)
constexpr uint32_t kStage = kABlock + 2 * kBHalf;
constexpr uint32_t kOffBar = kStages * kStage;
constexpr uint32_t kSmem = kOffBar + 64;    // + mbarriers + TMEM slot
constexpr uint32_t kTmemCols = kBN;
constexpr long long kWaitLimit = 1LL << 31;

__host__ __device__ constexpr uint32_t koff(int r, int k) { return kmajor_off(r, k, kBK); }

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
// K [16 s, +16), hi then lo, each in the canonical K-major layout.
// ---------------------------------------------------------------------------
__global__ void k_split(const LevelArgs* __restrict__ args)
{
    const LevelArgs& a = args[blockIdx.y];
    const int Np = a.Np;
    const int mt = (Np + kBM - 1) / kBM, nk = (Np + kBK - 1) / kBK;
    const long total = (long)mt * kBM * nk * kBK;  // padded elements
    unsigned char* out = reinterpret_cast<unsigned char*>(const_cast<float*>(a.Ps));
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        // e walks (row, k) of the padded matrix row-major
        const long kp = (long)nk * kBK;
        const int i = (int)(e / kp), k = (int)(e - (long)i * kp);
        double v = 0.0;
        if (i < Np && k < Np) {
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

__device__ __forceinline__ void cp16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// A block of slice s (16 KB, pre-split) into stage memory `st`.
__device__ __forceinline__ void fetch_a(const LevelArgs& a, int mi, int nk, int s, unsigned char* st)
{
    const unsigned char* src = reinterpret_cast<const unsigned char*>(a.Ps) + ((size_t)mi * nk + s) * kABlock;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int c = threadIdx.x + q * kThreads;  // 1024 chunks of 16 bytes
        cp16(st + c * 16, src + c * 16);
    }
}

// B values of slice s for this thread: vector tid/4, K [16 s + 4 (tid&3), +4).
__device__ __forceinline__ void load_b(const LevelArgs& a, long n0, int s, double (&b)[4])
{
    const int v = threadIdx.x >> 2, kb = s * kBK + (threadIdx.x & 3) * 4;
    const long g = n0 + v;
    if (g < a.ncols && kb < a.Np) {
        const double2* p = reinterpret_cast<const double2*>(a.src + g * a.src_gs + kb);
        const double2 t0 = p[0], t1 = p[1];
        b[0] = t0.x;
        b[1] = t0.y;
        b[2] = t1.x;
        b[3] = t1.y;
    } else {
        b[0] = b[1] = b[2] = b[3] = 0.0;
    }
}

__device__ __forceinline__ void store_b(const double (&b)[4], unsigned char* st)
{
    const int v = threadIdx.x >> 2, kb = (threadIdx.x & 3) * 4;
    float4 h, l;
    split_tf32((float)b[0], h.x, l.x);
    split_tf32((float)b[1], h.y, l.y);
    split_tf32((float)b[2], h.z, l.z);
    split_tf32((float)b[3], h.w, l.w);
    unsigned char* bb = st + kABlock;
    *reinterpret_cast<float4*>(bb + koff(v, kb)) = h;
    *reinterpret_cast<float4*>(bb + kBHalf + koff(v, kb)) = l;
}

// Thread 0: the 3xTF32 MMAs of one staged slice.
__device__ __forceinline__ void issue_slice(uint32_t d, uint32_t st, bool first)
{
    constexpr uint32_t SBO = kBK * 32;  // 8-row groups
    const uint64_t ah = make_desc(st, 128, SBO), al = make_desc(st + kAHalf, 128, SBO);
    const uint64_t bh = make_desc(st + kABlock, 128, SBO), bl = make_desc(st + kABlock + kBHalf, 128, SBO);
    const uint64_t A[3] = {ah, ah, al};
    const uint64_t B[3] = {bh, bl, bh};
    constexpr uint32_t idesc = make_idesc(kBM, kBN);
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int s = 0; s < kBK / 8; ++s)
            mma_tf32(d, A[q] + (uint64_t)(s * 16), B[q] + (uint64_t)(s * 16), idesc,
                     (first && q == 0 && s == 0) ? 0u : 1u);
}

struct Ring {
    uint32_t phase[kStages];
};

__device__ __forceinline__ void ring_wait(uint64_t* bar, Ring& r, int st, int* status)
{
    if (!mbar_wait(&bar[st], r.phase[st], kWaitLimit) && (threadIdx.x & 31) == 0) atomicExch(status, 1);
    r.phase[st] ^= 1u;
}

__device__ void tc_tile(const LevelArgs& a, long tile, unsigned char* sm, uint64_t* bar, uint32_t tbase, Ring& ring,
                        int* status)
{
    const int mt = (a.Np + kBM - 1) / kBM;
    const int mi = (int)(tile % mt);
    const int m0 = mi * kBM;
    const long n0 = (tile / mt) * kBN;
    const int nk = (a.Np + kBK - 1) / kBK;
    const uint32_t base = smem_u32(sm);

    // slice s uses stage s % 3; its MMAs commit to bar[s % 3]
    double b0[4], b1[4];
    load_b(a, n0, 0, b0);
    if (nk > 1) load_b(a, n0, 1, b1);
    fetch_a(a, mi, nk, 0, sm);
    cp_commit();
    for (int s = 0; s < nk; ++s) {
        const int st = s % kStages, nx = (s + 1) % kStages;
        // stage nx was last read by MMA(s - 2)
        if (s >= 2) ring_wait(bar, ring, nx, status);
        if (s + 1 < nk) fetch_a(a, mi, nk, s + 1, sm + nx * kStage);
        cp_commit();
        store_b(b0, sm + st * kStage);
#pragma unroll
        for (int q = 0; q < 4; ++q) b0[q] = b1[q];
        if (s + 2 < nk) load_b(a, n0, s + 2, b1);
        cp_wait1();  // A of slice s has landed (this thread's chunks)
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_after_sync();
            issue_slice(tbase, base + st * kStage, s == 0);
            mma_commit(&bar[st]);
        }
    }
    cp_wait0();
    // consume the completions not yet waited for: MMA(nk-2) (if any) and MMA(nk-1)
    for (int s = std::max(0, nk - 2); s < nk; ++s) ring_wait(bar, ring, s % kStages, status);
    fence_after_sync();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int quarter = warp & 3, half = warp >> 2;
    uint32_t r[32];
    tmem_ld32(tbase + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(half * 32), r);
    tmem_wait_ld();
    const long i = m0 + 32 * quarter + lane;
    if (i < a.Np) {
        const int rc = r_col(a, (int)i);
#pragma unroll 8
        for (int j = 0; j < 32; ++j) {
            const long g = n0 + 32 * half + j;
            if (g < a.ncols) {
                double v = (double)__uint_as_float(r[j]);
                if (rc >= 0) v += a.src[g * a.src_gs + rc];  // R v, exact
                if (a.acc) v += a.acc[g * a.acc_gs + i * a.acc_is];
                a.dst[g * a.dst_gs + i * a.dst_is] = v;
            }
        }
    }
    // TMEM reads complete before the next tile's first MMA overwrites it
    fence_before_sync();
    __syncthreads();
}

// Persistent grouped kernel: CTA c walks tiles [cta[c], cta[c+1]) in order
// (ranges balanced on the host); entries are found by a forward scan.
__global__ void __launch_bounds__(kThreads, 2) k_level_tc(const LevelArgs* __restrict__ args,
                                                          const long* __restrict__ start, int nent,
                                                          const long* __restrict__ cta, int* status)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kOffBar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + kOffBar + 32);
    if (threadIdx.x == 0) {
        for (int q = 0; q < kStages; ++q) mbar_init(&bar[q], 1);
        mbar_fence_init();
    }
    if ((threadIdx.x >> 5) == 0) tmem_alloc(slot, kTmemCols);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = *slot;
    Ring ring;
    for (int q = 0; q < kStages; ++q) ring.phase[q] = 0;
    const long t0 = cta[blockIdx.x], t1 = cta[blockIdx.x + 1];
    int e = 0;
    {
        int hi = nent - 1;
        while (e < hi) {
            const int mid = (e + hi + 1) >> 1;
            if (start[mid] <= t0) e = mid;
            else hi = mid - 1;
        }
    }
    LevelArgs a = args[e];
    long next = e + 1 < nent ? start[e + 1] : t1;
    for (long t = t0; t < t1; ++t) {
        while (t >= next) {
            ++e;
            a = args[e];
            next = e + 1 < nent ? start[e + 1] : t1;
        }
        tc_tile(a, t - start[e], sm, bar, tbase, ring, status);
    }
    fence_after_sync();
    if ((threadIdx.x >> 5) == 0) tmem_dealloc(tbase, kTmemCols);
}

}  // namespace

long level_tc_tiles(const LevelArgs& a)
{
    return (long)((a.Np + kBM - 1) / kBM) * ((a.ncols + kBN - 1) / kBN);
}

size_t level_split_bytes(int Np)
{
    return (size_t)((Np + kBM - 1) / kBM) * ((Np + kBK - 1) / kBK) * kABlock;
}

bool level_tc_supported(const LevelArgs& a)
{
    // K-contiguous FP64 sources with 16-byte aligned rows, no in-place copy
    return a.cpy == nullptr && a.src_ks == 1 && (a.src_gs % 2) == 0 && (a.ldp % 2) == 0 && (a.Np % 8) == 0 &&
           a.Np > 64 && a.Np <= 1024 && (reinterpret_cast<uintptr_t>(a.src) & 15) == 0;
}

void launch_level_split(const LevelArgs* dArgs, int nent, int max_np, cudaStream_t s)
{
    if (nent <= 0) return;
    const long elems = (long)level_split_bytes(max_np) / 8;
    dim3 grid((unsigned)std::max<long>(1, std::min<long>((elems + 255) / 256, 512)), (unsigned)nent);
    k_split<<<grid, 256, 0, s>>>(dArgs);
    PARODE_CUDA(cudaGetLastError());
}

void launch_level_tc(const LevelArgs* dArgs, const long* dStart, int nent, const long* dCta, int ctas, int* status,
                     cudaStream_t s)
{
    if (nent <= 0 || ctas <= 0) return;
    static bool attr_set = false;
    if (!attr_set) {
        PARODE_CUDA(cudaFuncSetAttribute(k_level_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
        attr_set = true;
    }
    k_level_tc<<<(unsigned)ctas, kThreads, kSmem, s>>>(dArgs, dStart, nent, dCta, status);
    PARODE_CUDA(cudaGetLastError());
}

// Host: tile ranges of `ctas` CTAs with about equal work (a tile costs its
// K slices plus a fixed overhead).
std::vector<long> level_tc_ranges(const std::vector<LevelArgs>& ents, int ctas)
{
    std::vector<double> cost;
    double total = 0;
    for (const LevelArgs& a : ents) {
        const long n = level_tc_tiles(a);
        const double c = (a.Np + kBK - 1) / kBK + 4.0;
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
