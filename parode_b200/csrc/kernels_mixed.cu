// kernels_mixed.cu -- leaf kernel of the mixed-precision blocked scan.
//
// Same tile structure as the FP64 leaf (kernels_blocked.cu): forcing, the R
// lowest Blelloch levels of every block in shared memory, zero-rooted
// down-sweep, y_local = C z + D u, block aggregates out.  The forcing and the
// level contractions V[right] += P_l V[left] run on the 5th-generation tensor
// cores (tcgen05.mma kind::tf32, accumulator in TMEM) in 3xTF32: every
// operand is split x = hi + lo with both parts rounded to TF32 and
// hi*hi + hi*lo + lo*hi is accumulated in FP32.  Vectors live in shared
// memory as FP32 hi/lo pairs; outputs run on the FP32 pipes.  The power
// table, the carry over block aggregates and the output fix-up stay in FP64
// (kernels_blocked.cu).
//
// Layout.  The tile's vectors are stored by Blelloch bucket: bucket l holds
// the positions whose (pos+1) has exactly l trailing zeros (the left children
// of level l), bucket R the block roots.  A level's left children are then
// consecutive rows, i.e. one K-major MMA operand (M = 128 rows per slice),
// while its right children are written back row by row from TMEM.  Input
// samples are stored as dense 16-byte rows (four inputs per chunk array), so
// the window term u_{2j+w} (RK4) or u_{j+w} (ABM) of every step is the same
// operand started w rows later.
#include "blocked.h"
#include "common.h"
#include "device_common.cuh"
#include "tc05.cuh"

#include <algorithm>

namespace parode {

namespace {

using namespace tc05;

constexpr int kTcThreads = 256;
constexpr long long kWaitLimit = 1LL << 31;  // SM cycles (about a second) before a wait gives up

struct TcLayout {
    int m4p;       // input chunks of 4, padded to a multiple of 2 (K = 8 per MMA)
    int rows;      // rows of each sample array
    int narr;      // sample arrays: RK4 even/odd samples, ABM all samples
    int W;         // window terms
    uint32_t vh, vl, ph, smp, bterm, cx, dx, bar, slot, total;
    __host__ __device__ uint32_t smp_chunk() const { return (uint32_t)rows * 16; }        // bytes per chunk array
    __host__ __device__ uint32_t smp_arr() const { return smp_chunk() * (uint32_t)m4p; }  // one array, one part
};

// Shared-memory layout (byte offsets).  Vl follows Vh and the power table
// follows Vl, so an M=128 operand slice that starts in a small bucket near
// the end of a vector array reads valid (ignored) rows.
__host__ __device__ inline TcLayout tc_layout(int NP, int R, int S, int n, int m, int p, int solver)
{
    TcLayout L;
    L.W = solver == 0 ? 3 : 5;
    L.narr = solver == 0 ? 2 : 1;
    const int m4 = (m + 3) / 4;
    L.m4p = m4 < 2 ? 2 : (m4 + 1) / 2 * 2;
    L.rows = (S + 8 + 7) / 8 * 8;
    uint32_t o = 0;
    L.vh = o;
    o += (uint32_t)S * NP * 4;
    L.vl = o;
    o += (uint32_t)S * NP * 4;
    L.ph = o;  // R levels x {hi, lo} x NP x NP
    o += (uint32_t)R * 2 * NP * NP * 4;
    L.smp = o;  // narr arrays x {hi, lo} x m4p chunks x rows x 16 B
    o += (uint32_t)L.narr * 2 * L.m4p * L.rows * 16;
    L.bterm = o;  // W terms x {hi, lo} x NP rows x (4 m4p) K
    o += (uint32_t)L.W * 2 * NP * L.m4p * 4 * 4;
    L.cx = o;  // Cext (p x NP) FP32
    o += (uint32_t)p * NP * 4;
    L.dx = o;  // D (p x m) FP32
    o += (uint32_t)p * (m > 0 ? m : 1) * 4;
    o = (o + 15) & ~15u;
    L.bar = o;
    o += 16;
    L.slot = o;
    o += 16;
    L.total = o;
    return L;
}

template <int NP>
__device__ __forceinline__ float* vptr(unsigned char* base, uint32_t off, int row, int k)
{
    return (float*)(base + off + kmajor_off(row, k, NP));
}

// Storage row of tile position pos (0 <= pos < S).
__device__ __forceinline__ int row_of(int pos, int R, int S)
{
    const int t = __ffs(pos + 1) - 1;
    if (t >= R) return (S - (S >> R)) + (pos >> R);
    return (S - (S >> t)) + ((pos + 1) >> (t + 1));
}

// Sample array element (array arr, hi/lo part, row r, input i).
__device__ __forceinline__ float* sptr(unsigned char* sm, const TcLayout& L, int arr, int part, int r, int i)
{
    return (float*)(sm + L.smp + (uint32_t)(arr * 2 + part) * L.smp_arr() + (uint32_t)(i >> 2) * L.smp_chunk() +
                    (uint32_t)r * 16 + (uint32_t)(i & 3) * 4);
}

// Issue D (+)= A B^T in 3xTF32 for K = 8 * ksteps: A hi/lo and B hi/lo are
// descriptor bases; a_step / b_step advance them by one K=8 slice.
__device__ __forceinline__ void mma3(uint32_t d, uint32_t ah, uint32_t al, uint32_t a_lbo, uint32_t a_sbo,
                                     uint32_t a_step, uint32_t bh, uint32_t bl, uint32_t b_lbo, uint32_t b_sbo,
                                     uint32_t b_step, int ksteps, uint32_t idesc, bool first)
{
    // descriptors are built once; a K step only moves the 14-bit start
    // address field (addresses < 256 KB, so the field never carries)
    const uint64_t dah = make_desc(ah, a_lbo, a_sbo), dal = make_desc(al, a_lbo, a_sbo);
    const uint64_t dbh = make_desc(bh, b_lbo, b_sbo), dbl = make_desc(bl, b_lbo, b_sbo);
    const uint64_t da[3] = {dah, dah, dal};
    const uint64_t db[3] = {dbh, dbl, dbh};
    const uint64_t sa = a_step >> 4, sb = b_step >> 4;
#pragma unroll
    for (int q = 0; q < 3; ++q)
        for (int s = 0; s < ksteps; ++s)
            mma_tf32(d, da[q] + sa * (uint64_t)s, db[q] + sb * (uint64_t)s, idesc, (first && q == 0 && s == 0) ? 0u : 1u);
}

// Wait for the round's MMAs (bounded), then make TMEM readable.
__device__ __forceinline__ void round_wait(uint64_t* bar, uint32_t& phase, int* status)
{
    if (!mbar_wait(bar, phase, kWaitLimit) && (threadIdx.x & 31) == 0) atomicExch(status, 1);
    phase ^= 1u;
    fence_after_sync();
}

__device__ __forceinline__ void round_end()
{
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
}

// Reads CPT TMEM columns of this thread's lane.
template <int CPT>
__device__ __forceinline__ void tmem_row(uint32_t taddr, uint32_t (&r)[CPT])
{
    if constexpr (CPT == 32) tmem_ld32(taddr, r);
    else tmem_ld16(taddr, r);
    tmem_wait_ld();
}

// One level: for every vector g < c of bucket l, V[right(g)] += P_l V[left(g)].
template <int NP>
__device__ void tc_level(unsigned char* sm, const TcLayout& L, uint64_t* bar, uint32_t tbase, int R, int S, int l,
                         uint32_t& phase, int* status)
{
    constexpr int CPT = NP < 32 ? NP : 32;  // TMEM columns per thread per slice
    constexpr int H = NP / CPT;             // column halves
    constexpr uint32_t SBO = NP * 32;
    const int c = S >> (l + 1);
    const int slices = (c + 127) >> 7;
    const int rs = S - (S >> l);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        fence_after_sync();
        const uint32_t base = smem_u32(sm);
        const uint32_t ph = base + L.ph + (uint32_t)l * 2 * NP * NP * 4;
        for (int z = 0; z < slices; ++z) {
            const uint32_t ro = (uint32_t)((rs + 128 * z) >> 3) * SBO;
            mma3(tbase + (uint32_t)(z * NP), base + L.vh + ro, base + L.vl + ro, 128, SBO, 256, ph,
                 ph + NP * NP * 4, 128, SBO, 256, NP / 8, make_idesc(128, NP), true);
        }
        mma_commit(bar);
    }
    __syncwarp();
    round_wait(bar, phase, status);
    const int sub = warp & 3, half = warp >> 2;
    if (half < H) {
        for (int z = 0; z < slices; ++z) {
            const int g = 128 * z + 32 * sub + lane;
            uint32_t r[CPT];
            tmem_row<CPT>(tbase + ((uint32_t)(32 * sub) << 16) + (uint32_t)(z * NP + half * CPT), r);
            if (g < c) {
                const int row = row_of(((g + 1) << (l + 1)) - 1, R, S);
#pragma unroll
                for (int k4 = 0; k4 < CPT; k4 += 4) {
                    const int k = half * CPT + k4;
                    float4* hp = (float4*)vptr<NP>(sm, L.vh, row, k);
                    float4* lp = (float4*)vptr<NP>(sm, L.vl, row, k);
                    const float4 hv = *hp, lv = *lp;
                    float4 ho, lo;
                    split_tf32(__uint_as_float(r[k4 + 0]) + (hv.x + lv.x), ho.x, lo.x);
                    split_tf32(__uint_as_float(r[k4 + 1]) + (hv.y + lv.y), ho.y, lo.y);
                    split_tf32(__uint_as_float(r[k4 + 2]) + (hv.z + lv.z), ho.z, lo.z);
                    split_tf32(__uint_as_float(r[k4 + 3]) + (hv.w + lv.w), ho.w, lo.w);
                    *hp = ho;
                    *lp = lo;
                }
            }
        }
    }
    round_end();
}

// Down-sweep bookkeeping of level l: V[left(g)] <-> V[right(g)] for g < c.
template <int NP>
__device__ void tc_swap(unsigned char* sm, const TcLayout& L, int R, int S, int l)
{
    const int c = S >> (l + 1);
    const int rs = S - (S >> l);
    // consecutive threads take consecutive vectors (rows) of the same 16-byte
    // chunk: a row's chunks are 128 bytes apart in the K-major layout, so
    // walking a row with neighbouring threads would hit one bank group
    for (int e = threadIdx.x; e < c * (NP / 4); e += kTcThreads) {
        const int k = 4 * (e / c), g = e - (k >> 2) * c;
        const int rl = rs + g, rr = row_of(((g + 1) << (l + 1)) - 1, R, S);
#pragma unroll
        for (int part = 0; part < 2; ++part) {
            const uint32_t off = part ? L.vl : L.vh;
            float4* a = (float4*)vptr<NP>(sm, off, rl, k);
            float4* b = (float4*)vptr<NP>(sm, off, rr, k);
            const float4 t = *a;
            *a = *b;
            *b = t;
        }
    }
    round_end();
}

template <int NP>
__global__ void __launch_bounds__(kTcThreads, 1) k_leaf_tc(LeafArgs a, int R, int S, int tcols)
{
    extern __shared__ __align__(128) unsigned char sm[];
    const TcLayout L = tc_layout(NP, R, S, a.n, a.m, a.p, a.solver);
    constexpr int CPT = NP < 32 ? NP : 32;
    constexpr int H = NP / CPT;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int B = 1 << R;
    const int m = a.m, n = a.n, p = a.p;
    const bool rk4 = a.solver == 0;
    const int mB = a.zeroB ? 0 : m;
    const int coff = rk4 ? 0 : 3 * n;
    const long nU = rk4 ? 2 * a.nScan + 1 : a.nScan + 4;
    uint64_t* bar = (uint64_t*)(sm + L.bar);
    uint32_t* slot = (uint32_t*)(sm + L.slot);
    float* sCx = (float*)(sm + L.cx);
    float* sD = (float*)(sm + L.dx);
    const int K4 = L.m4p * 4;  // padded input width of a window term

    // power table P_0..P_{R-1}: FP64 -> TF32 hi/lo, K-major (B operand rows = rows of P)
    for (int e = tid; e < R * NP * NP; e += kTcThreads) {
        const int l = e / (NP * NP), rem = e - l * NP * NP, r = rem / NP, k = rem - r * NP;
        const float hi = round_tf32((float)a.P[e]);
        const float lo = round_tf32((float)(a.P[e] - (double)hi));
        unsigned char* pb = sm + L.ph + (uint32_t)l * 2 * NP * NP * 4;
        *(float*)(pb + kmajor_off(r, k, NP)) = hi;
        *(float*)(pb + NP * NP * 4 + kmajor_off(r, k, NP)) = lo;
    }
    // forcing terms B_w (NP rows x K4), row coff+i = column block w of Bbar row i
    for (int e = tid; e < L.W * NP * K4; e += kTcThreads) {
        const int w = e / (NP * K4), rem = e - w * NP * K4, r = rem / K4, k = rem - r * K4;
        const int i = r - coff;
        double v = 0.0;
        if (mB > 0 && i >= 0 && i < n && k < m) v = a.Bbar[(long)i * L.W * m + w * m + k];
        const float hi = round_tf32((float)v);
        const float lo = round_tf32((float)(v - (double)hi));
        unsigned char* tb = sm + L.bterm + (uint32_t)w * 2 * NP * K4 * 4;
        *(float*)(tb + kmajor_off(r, k, K4)) = hi;
        *(float*)(tb + NP * K4 * 4 + kmajor_off(r, k, K4)) = lo;
    }
    for (int e = tid; e < p * NP; e += kTcThreads) {
        const int o = e / NP, k = e - o * NP, i = k - coff;
        float v = 0.f;
        if (a.zeroC && a.zeroD) v = (i == o) ? 1.f : 0.f;
        else if (!a.zeroC && i >= 0 && i < n) v = (float)a.C[(long)o * n + i];
        sCx[e] = v;
    }
    for (int e = tid; e < p * m; e += kTcThreads) sD[e] = a.zeroD ? 0.f : (float)a.D[e];
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(slot, (uint32_t)tcols);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = *slot;
    uint32_t phase = 0;

    for (long tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const long j0 = tile * S;
        // 1. input samples (hi/lo, 16-byte rows): RK4 arrays of even / odd
        //    half-step samples, ABM one array of whole-step samples
        for (int e = tid; e < L.narr * L.rows * K4; e += kTcThreads) {
            const int arr = e / (L.rows * K4), rem = e - arr * L.rows * K4, r = rem / K4, i = rem - r * K4;
            const long js = rk4 ? 2 * (j0 + r) + arr : j0 + r;
            double v = 0.0;
            if (i < m && js < nU) v = a.U[js * m + i];
            const float hi = round_tf32((float)v);
            const float lo = round_tf32((float)(v - (double)hi));
            *sptr(sm, L, arr, 0, r, i) = hi;
            *sptr(sm, L, arr, 1, r, i) = lo;
        }
        round_end();
        // 2. forcing on the tensor cores: Gamma (S x NP) = sum_w U_w B_w^T
        {
            const int slices = (S + 127) >> 7;
            if (tid == 0) {
                fence_after_sync();
                const uint32_t base = smem_u32(sm);
                const uint32_t idesc = make_idesc(128, NP);
                for (int z = 0; z < slices; ++z) {
                    for (int w = 0; w < L.W; ++w) {
                        const int arr = rk4 ? (w == 1 ? 1 : 0) : 0;
                        const int r0 = 128 * z + (rk4 ? (w == 2 ? 1 : 0) : w);
                        const uint32_t sa = base + L.smp + (uint32_t)(arr * 2) * L.smp_arr() + (uint32_t)r0 * 16;
                        const uint32_t tb = base + L.bterm + (uint32_t)w * 2 * NP * K4 * 4;
                        mma3(tbase + (uint32_t)(z * NP), sa, sa + L.smp_arr(), L.smp_chunk(), 128, 2 * L.smp_chunk(),
                             tb, tb + NP * K4 * 4, 128, (uint32_t)K4 * 32, 256, L.m4p / 2, idesc, w == 0);
                    }
                }
                mma_commit(bar);
            }
            __syncwarp();
            round_wait(bar, phase, a.status);
            const int sub = warp & 3, half = warp >> 2;
            if (half < H) {
                for (int z = 0; z < slices; ++z) {
                    const int j = 128 * z + 32 * sub + lane;
                    uint32_t r[CPT];
                    tmem_row<CPT>(tbase + ((uint32_t)(32 * sub) << 16) + (uint32_t)(z * NP + half * CPT), r);
                    if (j < S) {
                        const bool live = mB > 0 && j0 + j < a.nScan;
                        const int row = row_of(j, R, S);
#pragma unroll
                        for (int k4 = 0; k4 < CPT; k4 += 4) {
                            const int k = half * CPT + k4;
                            float4 ho, lo;
                            split_tf32(live ? __uint_as_float(r[k4 + 0]) : 0.f, ho.x, lo.x);
                            split_tf32(live ? __uint_as_float(r[k4 + 1]) : 0.f, ho.y, lo.y);
                            split_tf32(live ? __uint_as_float(r[k4 + 2]) : 0.f, ho.z, lo.z);
                            split_tf32(live ? __uint_as_float(r[k4 + 3]) : 0.f, ho.w, lo.w);
                            *(float4*)vptr<NP>(sm, L.vh, row, k) = ho;
                            *(float4*)vptr<NP>(sm, L.vl, row, k) = lo;
                        }
                    }
                }
            }
            round_end();
        }
        // 3. up-sweep on the tensor cores
        for (int l = 0; l < R; ++l) tc_level<NP>(sm, L, bar, tbase, R, S, l, phase, a.status);
        // 4. block aggregates (FP64) out, zero roots
        {
            const int rsR = S - (S >> R);
            for (int e = tid; e < (S / B) * NP; e += kTcThreads) {
                const int b = e / NP, k = e - b * NP;
                float* hp = vptr<NP>(sm, L.vh, rsR + b, k);
                float* lp = vptr<NP>(sm, L.vl, rsR + b, k);
                a.G[(tile * (S / B) + b) * NP + k] = (double)*hp + (double)*lp;
                *hp = 0.f;
                *lp = 0.f;
            }
            round_end();
        }
        // 5. down-sweep from the zero roots
        for (int l = R - 1; l >= 0; --l) {
            tc_swap<NP>(sm, L, R, S, l);
            if (l < R - 1) tc_level<NP>(sm, L, bar, tbase, R, S, l, phase, a.status);
        }
        // 6. y_local = Cext z + D u, FP32, one step per thread pair, FP64 out
        {
            const int ph = (p + 1) / 2;
            for (int jj = tid >> 1; jj < S; jj += kTcThreads / 2) {
                if (j0 + jj >= a.nScan) continue;
                const int row = row_of(jj, R, S);
                float z[NP];
#pragma unroll
                for (int k = 0; k < NP; k += 4) {
                    const float4 hv = *(const float4*)vptr<NP>(sm, L.vh, row, k);
                    const float4 lv = *(const float4*)vptr<NP>(sm, L.vl, row, k);
                    z[k] = hv.x + lv.x;
                    z[k + 1] = hv.y + lv.y;
                    z[k + 2] = hv.z + lv.z;
                    z[k + 3] = hv.w + lv.w;
                }
                const int urow = rk4 ? jj : jj + 3;  // RK4: even-sample array row jj = u_{2j}
                const int o0 = (tid & 1) * ph, o1 = min(p, o0 + ph);
                for (int o = o0; o < o1; ++o) {
                    const float* cr = sCx + o * NP;
                    float v = 0.f;
#pragma unroll
                    for (int k = 0; k < NP; k += 4) {
                        const float4 cv = *(const float4*)(cr + k);
                        v = fmaf(cv.x, z[k], v);
                        v = fmaf(cv.y, z[k + 1], v);
                        v = fmaf(cv.z, z[k + 2], v);
                        v = fmaf(cv.w, z[k + 3], v);
                    }
                    if (!a.zeroD)
                        for (int c = 0; c < m; ++c)
                            v = fmaf(sD[o * m + c], *sptr(sm, L, 0, 0, urow, c) + *sptr(sm, L, 0, 1, urow, c), v);
                    a.Y[(a.ybase + j0 + jj) * p + o] = (double)v;
                }
            }
        }
        __syncthreads();
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tbase, (uint32_t)tcols);
}

template <int NP>
void leaf_tc_t(const BlockedShape& sh, const LeafArgs& a, int grid, cudaStream_t s)
{
    const TcLayout L = tc_layout(NP, sh.R, sh.S, a.n, a.m, a.p, a.solver);
    const int slices = (sh.S + 127) >> 7;  // the forcing round covers all S rows
    int tcols = 32;
    while (tcols < slices * NP) tcols <<= 1;
    if (tcols > 512) throw Error(kInvalidArgument, "mixed leaf: TMEM columns exceed 512");
    PARODE_CUDA(cudaFuncSetAttribute(k_leaf_tc<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
    unsigned g = (unsigned)std::max<long>(1, std::min<long>(a.ntiles, grid));
    k_leaf_tc<NP><<<g, kTcThreads, L.total, s>>>(a, sh.R, sh.S, tcols);
    PARODE_CUDA(cudaGetLastError());
}

}  // namespace

size_t blocked_leaf_tc_bytes(const BlockedShape& sh, int n, int m, int p, int solver)
{
    if (sh.NP < 16) return 0;  // N = NP must be a multiple of 16 for M = 128
    if (sh.S < 128 || sh.S < 4 * sh.B || sh.S % sh.B != 0) return 0;
    if (((sh.S + 127) >> 7) * sh.NP > 512) return 0;
    TcLayout L = tc_layout(sh.NP, sh.R, sh.S, n, m, p, solver);
    return L.total <= 232448 - 1024 ? L.total : 0;
}

void launch_blocked_leaf_tc(const BlockedShape& sh, const LeafArgs& a, int grid, cudaStream_t s)
{
    switch (sh.NP) {
    case 16: leaf_tc_t<16>(sh, a, grid, s); break;
    case 32: leaf_tc_t<32>(sh, a, grid, s); break;
    case 64: leaf_tc_t<64>(sh, a, grid, s); break;
    default: throw Error(kInvalidArgument, "mixed leaf: unsupported NP");
    }
}

}  // namespace parode
