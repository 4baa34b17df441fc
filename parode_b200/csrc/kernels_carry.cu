// kernels_carry.cu -- exclusive scan of block aggregates for scan dimensions <= 64.
//
// The blocked and block-response leaves leave one aggregate G_b per block of
// B steps; the state entering block b is the exclusive scan
//   X_0 = x0,  X_{b+1} = Q X_b + G_b,  Q = Phi^B,
// which is the reference's Blelloch composition (Kernels/MVVKernelScanUpsweep.cl,
// MVVKernelScanDownsweep.cl) applied to the blocks.  Here it runs as a chunked
// scan: chunks of F = 16 items, each chunk's aggregate by 16 sequential steps
// (up), the chunk aggregates scanned one level higher with Q^16, and each
// chunk's items rewritten by 16 sequential steps from its carried-in state
// (down).  A CTA owns 8 chunks as the 8 columns of an NP x 8 tile: every step
// is one NP x NP x 8 product on the FP64 tensor cores (DMMA m8n8k4) with Q's
// fragments held in registers, so the sequential depth is 16 steps per level
// while the chunks spread over all SMs (narrow tiles keep the few-chunk upper
// levels short: a step's time is set by one SM's FP64 rate).  The flops equal
// the Blelloch up- plus down-sweep's (2 NP^2 per item each way).
//
// Above level 0 the chunks are few and every level is latency-bound, so each
// chunk runs at depth 4 instead of 16, with the doublings Q, Q^2, Q^4, Q^8 of
// the power table: its aggregate as a pairwise tree (15 products, the chain's
// count), its rewrite as a Kogge-Stone scan over [carry, item 0 .. item 14]
// (49 products).  The form depends on the level's global index only, so a
// time-partitioned solve takes the same steps on every level as the whole one.
#include "common.h"
#include "device_common.cuh"
#include "kernels.h"

#include <algorithm>

namespace parode {

namespace {

constexpr int kThreads = 256;
constexpr int kCols = 8;        // chunks per CTA (the tile's columns)
constexpr int kNT = kCols / 8;  // n-tiles of the tile
constexpr int kChunk = 16;      // items per chunk: Q^16 = 4 power-table levels up
constexpr int kLd = kCols + 4;  // shared-memory row pitch (doubles): conflict-free B fragments

// Warp roles: m-tile mt (8 rows of Q) and n-tiles nt0 .. nt0 + nts - 1 (8
// chunk columns each) of the NP x kCols tile.
template <int NP>
struct Roles {
    int g, t, mt, nt0, nts;
    bool active;
    __device__ Roles()
    {
        constexpr int MT = NP / 8, NT = kCols / 8, WPM = 8 / MT;
        constexpr int NTS = NT / WPM > 0 ? NT / WPM : 1;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        g = lane >> 2;
        t = lane & 3;
        mt = warp % MT;
        nts = NTS;
        nt0 = (warp / MT) * NTS;
        active = nt0 < NT;
    }
};

template <int NP>
__device__ __forceinline__ void load_q(const double* __restrict__ Q, const Roles<NP>& r, double (&qa)[NP / 4])
{
#pragma unroll
    for (int kk = 0; kk < NP / 4; ++kk) qa[kk] = Q[(r.mt * 8 + r.g) * NP + 4 * kk + r.t];
}

// G of step j for this lane's D-fragment positions: item (c0 + col) F + j, row.
template <int NP>
__device__ __forceinline__ void load_g(const double* __restrict__ items, long count, long c0, int F, int j,
                                       const Roles<NP>& r, double (&v)[kNT][2])
{
    const int row = r.mt * 8 + r.g;
#pragma unroll
    for (int u = 0; u < kNT; ++u)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const long item = (c0 + (r.nt0 + u) * 8 + 2 * r.t + e) * F + j;
            v[u][e] = (u < r.nts && item < count) ? items[item * NP + row] : 0.0;
        }
}

// acc += Q X on the tile (X in shared memory, row pitch kLd).  The K
// products go to kSplit independent partial sums, so the dependent MMA chain
// (the step's latency) is NP / 4 / kSplit long.
template <int NP>
__device__ __forceinline__ void step_mma(const double* X, const double (&qa)[NP / 4], double (&acc)[kNT][2],
                                         const Roles<NP>& r)
{
    constexpr int kSplit = NP / 4 < 4 ? NP / 4 : 4;
    double part[kSplit][kNT][2];
#pragma unroll
    for (int q = 0; q < kSplit; ++q)
#pragma unroll
        for (int u = 0; u < kNT; ++u) part[q][u][0] = part[q][u][1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < NP / 4; ++kk) {
        const double* xr = X + (4 * kk + r.t) * kLd + r.g;
#pragma unroll
        for (int u = 0; u < kNT; ++u)
            if (u < r.nts) dmma_m8n8k4(part[kk % kSplit][u][0], part[kk % kSplit][u][1], qa[kk], xr[(r.nt0 + u) * 8]);
    }
#pragma unroll
    for (int u = 0; u < kNT; ++u)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            double v = acc[u][e];
#pragma unroll
            for (int q = 0; q < kSplit; ++q) v += part[q][u][e];
            acc[u][e] = v;
        }
}

// This lane's D-fragment positions of the states into item slot j.
template <int NP>
__device__ __forceinline__ void store_g(double* __restrict__ items, long count, long c0, int F, int j,
                                        const Roles<NP>& r, const double (&v)[kNT][2])
{
    const int row = r.mt * 8 + r.g;
#pragma unroll
    for (int u = 0; u < kNT; ++u)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const long item = (c0 + (r.nt0 + u) * 8 + 2 * r.t + e) * F + j;
            if (u < r.nts && item < count) items[item * NP + row] = v[u][e];
        }
}

template <int NP>
__device__ __forceinline__ void store_tile(double* X, const double (&acc)[kNT][2], const Roles<NP>& r)
{
    const int row = r.mt * 8 + r.g;
#pragma unroll
    for (int u = 0; u < kNT; ++u)
        if (u < r.nts) {
            X[row * kLd + (r.nt0 + u) * 8 + 2 * r.t] = acc[u][0];
            X[row * kLd + (r.nt0 + u) * 8 + 2 * r.t + 1] = acc[u][1];
        }
}

// Chunk aggregates of one tile (kCols chunks from c0 = tile * kCols):
// next[c] = sum_{j<16} Q^(15-j) items[16 c + j] (items past count are zero;
// the last chunk's aggregate is never read by the scan).  Xs: 2 NP x kLd
// doubles of shared memory.  Every thread of the CTA takes part.
template <int NP>
__device__ __forceinline__ void chunk_up_tile(const double* __restrict__ items, long count,
                                              const double* __restrict__ Q, double* __restrict__ next, long tile,
                                              double* Xs0, double* Xs1)
{
    const Roles<NP> r;
    const long c0 = tile * kCols;
    const long nchunks = (count + kChunk - 1) / kChunk;
    double* Xs[2] = {Xs0, Xs1};
    double qa[NP / 4];
    load_q<NP>(Q, r, qa);
    for (int e = threadIdx.x; e < NP * kLd; e += kThreads) Xs[0][e] = 0.0;
    grid_dep_wait();  // the items are the previous kernel's
    grid_dep_trigger();  // the next level's CTAs may start loading their powers
    double pre[kNT][2];
    if (r.active) load_g<NP>(items, count, c0, kChunk, 0, r, pre);
    __syncthreads();
    int cur = 0;
    for (int j = 0; j < kChunk; ++j) {
        if (r.active) {
            double acc[kNT][2];
#pragma unroll
            for (int u = 0; u < kNT; ++u) acc[u][0] = pre[u][0], acc[u][1] = pre[u][1];
            if (j + 1 < kChunk) load_g<NP>(items, count, c0, kChunk, j + 1, r, pre);
            step_mma<NP>(Xs[cur], qa, acc, r);
            store_tile<NP>(Xs[cur ^ 1], acc, r);
        }
        __syncthreads();
        cur ^= 1;
    }
    for (int e = threadIdx.x; e < NP * kCols; e += kThreads) {
        const int col = e / NP, row = e - col * NP;
        if (c0 + col < nchunks) next[(c0 + col) * NP + row] = Xs[cur][row * kLd + col];
    }
    __syncthreads();  // Xs is reused by the CTA's next tile
}

template <int NP>
__global__ void __launch_bounds__(kThreads) k_chunk_up(const double* __restrict__ items, long count,
                                                        const double* __restrict__ Q, double* __restrict__ next)
{
    __shared__ double Xs[2][NP * kLd];
    chunk_up_tile<NP>(items, count, Q, next, blockIdx.x, Xs[0], Xs[1]);
}

// Chunk rewrite of one tile: from the chunk's carried-in state
// x = carries[c], items [F c, F c + F) become the states entering them (x,
// then Q x + item, ...).  Each lane reads item j + 1 (its D-fragment
// positions) before it writes the state into the same positions, so slots
// need no barrier.
template <int NP>
__device__ __forceinline__ void chunk_down_tile(double* __restrict__ items, long count,
                                                const double* __restrict__ Q, const double* __restrict__ carries,
                                                int F, long tile, double* Xs0, double* Xs1)
{
    const Roles<NP> r;
    const long c0 = tile * kCols;
    const long nchunks = (count + F - 1) / F;
    double* Xs[2] = {Xs0, Xs1};
    double qa[NP / 4];
    load_q<NP>(Q, r, qa);
    grid_dep_wait();  // the carries and items are the previous kernels'
    grid_dep_trigger();  // the next level's CTAs may start loading their powers
    for (int e = threadIdx.x; e < NP * kLd; e += kThreads) {
        const int row = e / kLd, col = e - row * kLd;
        Xs[0][e] = (col < kCols && c0 + col < nchunks) ? carries[(c0 + col) * NP + row] : 0.0;
    }
    double pre[kNT][2];
    if (r.active) load_g<NP>(items, count, c0, F, 0, r, pre);
    __syncthreads();
    if (r.active) {
        // slot 0 <- the carried-in state (item 0 is already in pre)
        double x0[kNT][2];
        const int row = r.mt * 8 + r.g;
#pragma unroll
        for (int u = 0; u < kNT; ++u)
#pragma unroll
            for (int e = 0; e < 2; ++e) x0[u][e] = Xs[0][row * kLd + (r.nt0 + u) * 8 + 2 * r.t + e];
        store_g<NP>(items, count, c0, F, 0, r, x0);
    }
    int cur = 0;
    for (int j = 0; j + 1 < F; ++j) {
        if (r.active) {
            double acc[kNT][2];
#pragma unroll
            for (int u = 0; u < kNT; ++u) acc[u][0] = pre[u][0], acc[u][1] = pre[u][1];
            load_g<NP>(items, count, c0, F, j + 1, r, pre);
            step_mma<NP>(Xs[cur], qa, acc, r);
            store_tile<NP>(Xs[cur ^ 1], acc, r);
            store_g<NP>(items, count, c0, F, j + 1, r, acc);
        }
        __syncthreads();
        cur ^= 1;
    }
    __syncthreads();  // Xs is reused by the CTA's next tile
}

template <int NP>
__global__ void __launch_bounds__(kThreads) k_chunk_down(double* __restrict__ items, long count,
                                                          const double* __restrict__ Q,
                                                          const double* __restrict__ carries, int F)
{
    __shared__ double Xs[2][NP * kLd];
    chunk_down_tile<NP>(items, count, Q, carries, F, blockIdx.x, Xs[0], Xs[1]);
}

// ---- depth-4 forms of the levels above 0 ------------------------------------
constexpr int kTP = 20;  // row pitch (doubles) of a chunk's 16-column tile: conflict-free B fragments

// Warp w: m-tile w % MT of the chunks grp + WPC k (k < CPW), grp = w / MT;
// a CTA holds CC = WPC CPW chunks.  (Two chunks per warp, interleaving their
// products in half the CTAs, measured slower on cfg2's levels: 134 against
// 122 us for the whole carry.)
template <int NP>
struct TreeRoles {
    static constexpr int MT = NP / 8;
    static constexpr int WPC = MT >= 8 ? 1 : 8 / MT;
    static constexpr int CPW = 1;
    static constexpr int CC = WPC * CPW;
    int g, t, mt, grp;
    bool active;
    __device__ TreeRoles()
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        g = lane >> 2;
        t = lane & 3;
        mt = warp % MT;
        grp = warp / MT;
        active = grp < WPC;
    }
    __device__ int chunk(int k) const { return grp + WPC * k; }
};

// A fragments of Q, Q^2, Q^4, Q^8 (P: Q's level of the power table).
template <int NP>
__device__ __forceinline__ void load_q4(const double* __restrict__ P, const TreeRoles<NP>& r,
                                        double (&qa)[4][NP / 4])
{
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int kk = 0; kk < NP / 4; ++kk) qa[i][kk] = P[(long)i * NP * NP + (r.mt * 8 + r.g) * NP + 4 * kk + r.t];
}

// acc[u] (this lane's D fragment of 8-column tile u) += Q S_u[:, col_u], col_u
// this lane's B column of tile u (< 0: a zero column); the NT tiles' chains
// interleave.
template <int NP, int NT>
__device__ __forceinline__ void tiles_mma(const double (&qa)[NP / 4], const double* const (&S)[NT],
                                          const int (&col)[NT], int t, double (&acc)[NT][2])
{
    constexpr int kSplit = NP / 4 < 4 ? NP / 4 : 4;
    double part[kSplit][NT][2];
#pragma unroll
    for (int q = 0; q < kSplit; ++q)
#pragma unroll
        for (int u = 0; u < NT; ++u) part[q][u][0] = part[q][u][1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < NP / 4; ++kk)
#pragma unroll
        for (int u = 0; u < NT; ++u) {
            const double b = col[u] >= 0 ? S[u][(4 * kk + t) * kTP + col[u]] : 0.0;
            dmma_m8n8k4(part[kk % kSplit][u][0], part[kk % kSplit][u][1], qa[kk], b);
        }
#pragma unroll
    for (int u = 0; u < NT; ++u)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            double v = acc[u][e];
#pragma unroll
            for (int q = 0; q < kSplit; ++q) v += part[q][u][e];
            acc[u][e] = v;
        }
}

// Chunk aggregates as pairwise trees: step s combines neighbours 2^s items
// apart, Y[p] = Q^(2^s) X[2p] + X[2p+1].  P points at Q's table level.
template <int NP>
__global__ void __launch_bounds__(kThreads) k_chunk_tree_up(const double* __restrict__ items, long count,
                                                             const double* __restrict__ P, double* __restrict__ next)
{
    using R = TreeRoles<NP>;
    constexpr int CPW = R::CPW;
    __shared__ double Xs[2][R::CC][NP * kTP];
    const R r;
    const long c0 = (long)blockIdx.x * R::CC;
    const long nchunks = (count + kChunk - 1) / kChunk;
    double qa[4][NP / 4];
    if (r.active) load_q4<NP>(P, r, qa);
    grid_dep_wait();  // the items are the previous kernel's
    grid_dep_trigger();  // the next level's CTAs may start loading their powers
    for (int e = threadIdx.x; e < R::CC * kChunk * NP; e += kThreads) {
        const int cl = e / (kChunk * NP), rem = e - cl * kChunk * NP, j = rem / NP, row = rem - j * NP;
        const long item = (c0 + cl) * kChunk + j;
        Xs[0][cl][row * kTP + j] = item < count ? items[item * NP + row] : 0.0;
    }
    __syncthreads();
    const int row = r.mt * 8 + r.g;
#pragma unroll
    for (int st = 0; st < 4; ++st) {
        const int ncol = 8 >> st;  // this step's outputs
        if (r.active) {
            const double* S[CPW];
            int col[CPW];
            double acc[CPW][2];
#pragma unroll
            for (int k = 0; k < CPW; ++k) {
                S[k] = Xs[st & 1][r.chunk(k)];
                col[k] = r.g < ncol ? 2 * r.g : -1;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int p = 2 * r.t + e;
                    acc[k][e] = p < ncol ? S[k][row * kTP + 2 * p + 1] : 0.0;
                }
            }
            tiles_mma<NP, CPW>(qa[st], S, col, r.t, acc);
#pragma unroll
            for (int k = 0; k < CPW; ++k)
#pragma unroll
                for (int e = 0; e < 2; ++e)
                    if (2 * r.t + e < ncol) Xs[(st & 1) ^ 1][r.chunk(k)][row * kTP + 2 * r.t + e] = acc[k][e];
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < R::CC * NP; e += kThreads) {
        const int cl = e / NP, row2 = e - cl * NP;
        if (c0 + cl < nchunks) next[(c0 + cl) * NP + row2] = Xs[0][cl][row2 * kTP];
    }
}

// Chunk rewrite as a Kogge-Stone scan: E = [carry, item 0 .. item F-2], step
// s adds Q^(2^s) E[j - 2^s] to E[j]; slot j then holds the state entering
// item j.  F items per chunk (16, or the top's count).
template <int NP>
__global__ void __launch_bounds__(kThreads) k_chunk_ks_down(double* __restrict__ items, long count,
                                                             const double* __restrict__ P,
                                                             const double* __restrict__ carries, int F)
{
    using R = TreeRoles<NP>;
    constexpr int CPW = R::CPW;
    __shared__ double Es[2][R::CC][NP * kTP];
    const R r;
    const long c0 = (long)blockIdx.x * R::CC;
    const long nchunks = (count + F - 1) / F;
    double qa[4][NP / 4];
    if (r.active) load_q4<NP>(P, r, qa);
    grid_dep_wait();  // the carries and items are the previous kernels'
    grid_dep_trigger();  // the next level's CTAs may start loading their powers
    for (int e = threadIdx.x; e < R::CC * kChunk * NP; e += kThreads) {
        const int cl = e / (kChunk * NP), rem = e - cl * kChunk * NP, j = rem / NP, row = rem - j * NP;
        const long c = c0 + cl;
        double v = 0.0;
        if (c < nchunks) {
            if (j == 0) v = carries[c * NP + row];
            else if (j - 1 < F - 1 && c * F + j - 1 < count) v = items[(c * F + j - 1) * NP + row];
        }
        Es[0][cl][row * kTP + j] = v;
    }
    __syncthreads();
    const int row = r.mt * 8 + r.g;
    int cur = 0;
#pragma unroll
    for (int st = 0; st < 4; ++st) {
        const int d = 1 << st;
        if (d >= F) break;  // no slot below F reads further back
        if (r.active) {
            // tiles (chunk k, columns 8u .. 8u + 7); columns below d keep their value
            if (d < 8) {
                const double* S[2 * CPW];
                int col[2 * CPW];
                double acc[2 * CPW][2];
#pragma unroll
                for (int k = 0; k < CPW; ++k)
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        S[2 * k + u] = Es[cur][r.chunk(k)];
                        col[2 * k + u] = 8 * u + r.g - d;
#pragma unroll
                        for (int e = 0; e < 2; ++e) acc[2 * k + u][e] = S[2 * k + u][row * kTP + 8 * u + 2 * r.t + e];
                    }
                tiles_mma<NP, 2 * CPW>(qa[st], S, col, r.t, acc);
#pragma unroll
                for (int k = 0; k < CPW; ++k)
#pragma unroll
                    for (int u = 0; u < 2; ++u)
#pragma unroll
                        for (int e = 0; e < 2; ++e)
                            Es[cur ^ 1][r.chunk(k)][row * kTP + 8 * u + 2 * r.t + e] = acc[2 * k + u][e];
            } else {
                const double* S[CPW];
                int col[CPW];
                double acc[CPW][2];
#pragma unroll
                for (int k = 0; k < CPW; ++k) {
                    S[k] = Es[cur][r.chunk(k)];
                    col[k] = r.g;  // 8 + g - 8
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        acc[k][e] = S[k][row * kTP + 8 + 2 * r.t + e];
                        Es[cur ^ 1][r.chunk(k)][row * kTP + 2 * r.t + e] = S[k][row * kTP + 2 * r.t + e];
                    }
                }
                tiles_mma<NP, CPW>(qa[st], S, col, r.t, acc);
#pragma unroll
                for (int k = 0; k < CPW; ++k)
#pragma unroll
                    for (int e = 0; e < 2; ++e) Es[cur ^ 1][r.chunk(k)][row * kTP + 8 + 2 * r.t + e] = acc[k][e];
            }
        }
        __syncthreads();
        cur ^= 1;
    }
    for (int e = threadIdx.x; e < R::CC * kChunk * NP; e += kThreads) {
        const int cl = e / (kChunk * NP), rem = e - cl * kChunk * NP, j = rem / NP, row2 = rem - j * NP;
        const long c = c0 + cl, item = c * F + j;
        if (c < nchunks && j < F && item < count) items[item * NP + row2] = Es[cur][cl][row2 * kTP + j];
    }
}

// ---------------------------------------------------------------------------
template <int NP>
unsigned tree_grid(long nchunks)
{
    constexpr int CC = TreeRoles<NP>::CC;
    return (unsigned)((nchunks + CC - 1) / CC);
}

template <int NP>
int chunk_up_t(double* items, long count, const double* P, int l0, int h0, double* work, int levels, ChunkLevels* L,
               cudaStream_t s)
{
    const long mat = (long)NP * NP;
    L->arr[0] = items;
    L->cnt[0] = count;
    int h = 0;
    double* w = work;
    int launches = 0;
    while (levels < 0 ? L->cnt[h] > kChunk : h < levels) {
        if (h + 1 >= 16) throw Error(kInvalidArgument, "chunk carry: too many levels");
        const long nc = (L->cnt[h] + kChunk - 1) / kChunk;
        if (h0 + h == 0) {
            const unsigned grid = (unsigned)((nc + kCols - 1) / kCols);
            launch_dependent(k_chunk_up<NP>, grid, kThreads, 0, s, (const double*)L->arr[h], L->cnt[h],
                             P + (long)(l0 + 4 * h) * mat, w);
        } else {
            launch_dependent(k_chunk_tree_up<NP>, tree_grid<NP>(nc), kThreads, 0, s, (const double*)L->arr[h],
                             L->cnt[h], P + (long)(l0 + 4 * h) * mat, w);
        }
        ++launches;
        L->arr[h + 1] = w;
        L->cnt[h + 1] = nc;
        w += nc * NP;
        ++h;
    }
    L->h = h;
    return launches;
}

template <int NP>
int chunk_down_t(const ChunkLevels& L, const double* P, int l0, int h0, cudaStream_t s)
{
    const long mat = (long)NP * NP;
    for (int k = L.h - 1; k >= 0; --k) {
        const long nc = (L.cnt[k] + kChunk - 1) / kChunk;
        if (h0 + k == 0) {
            const unsigned grid = (unsigned)((nc + kCols - 1) / kCols);
            launch_dependent(k_chunk_down<NP>, grid, kThreads, 0, s, L.arr[k], L.cnt[k], P + (long)(l0 + 4 * k) * mat,
                             (const double*)L.arr[k + 1], kChunk);
        } else {
            launch_dependent(k_chunk_ks_down<NP>, tree_grid<NP>(nc), kThreads, 0, s, L.arr[k], L.cnt[k],
                             P + (long)(l0 + 4 * k) * mat, (const double*)L.arr[k + 1], kChunk);
        }
    }
    return L.h;
}

template <int NP>
int chunk_top_t(double* items, long count, const double* Q, const double* X0, cudaStream_t s)
{
    // one chunk of at most 16 items, entered with X0 (Q's table level and the
    // three above it: Q^2, Q^4, Q^8)
    launch_dependent(k_chunk_ks_down<NP>, 1, kThreads, 0, s, items, count, Q, X0, (int)count);
    return 1;
}

template <int NP>
int chunk_carry_t(double* items, long count, const double* P, int l0, int h0, const double* X0, double* work,
                  cudaStream_t s)
{
    ChunkLevels L;
    int launches = chunk_up_t<NP>(items, count, P, l0, h0, work, -1, &L, s);
    launches += chunk_top_t<NP>(L.arr[L.h], L.cnt[L.h], P + (long)(l0 + 4 * L.h) * NP * NP, X0, s);
    launches += chunk_down_t<NP>(L, P, l0, h0, s);
    return launches;
}

}  // namespace

int chunk_carry_table_levels(long count) { return 4 * chunk_carry_levels(count) + 4; }

int chunk_carry_levels(long count)
{
    int h = 0;
    while (count > kChunk) {
        count = (count + kChunk - 1) / kChunk;
        ++h;
    }
    return h;
}

long chunk_carry_scratch(long count)
{
    long total = 0;
    while (count > kChunk) {
        count = (count + kChunk - 1) / kChunk;
        total += count;
    }
    return total;
}

#define PARODE_NP_SWITCH(NP, CALL)                                                             \
    switch (NP) {                                                                              \
    case 8: return CALL(8);                                                                    \
    case 16: return CALL(16);                                                                  \
    case 24: return CALL(24);                                                                  \
    case 32: return CALL(32);                                                                  \
    case 40: return CALL(40);                                                                  \
    case 48: return CALL(48);                                                                  \
    case 56: return CALL(56);                                                                  \
    case 64: return CALL(64);                                                                  \
    default: throw Error(kInvalidArgument, "chunk carry: NP must be a multiple of 8 up to 64"); \
    }

int launch_chunk_up(int NP, double* items, long count, const double* P, int l0, double* work, int levels,
                    ChunkLevels* L, cudaStream_t s)
{
#define PARODE_UP(K) chunk_up_t<K>(items, count, P, l0, 0, work, levels, L, s)
    PARODE_NP_SWITCH(NP, PARODE_UP)
#undef PARODE_UP
}

int launch_chunk_down(int NP, const ChunkLevels& L, const double* P, int l0, cudaStream_t s)
{
#define PARODE_DOWN(K) chunk_down_t<K>(L, P, l0, 0, s)
    PARODE_NP_SWITCH(NP, PARODE_DOWN)
#undef PARODE_DOWN
}

int launch_chunk_carry(int NP, double* items, long count, const double* P, int l0, int h0, const double* X0,
                       double* work, cudaStream_t s)
{
    if (count <= 0) return 0;
#define PARODE_CARRY(K) chunk_carry_t<K>(items, count, P, l0, h0, X0, work, s)
    PARODE_NP_SWITCH(NP, PARODE_CARRY)
#undef PARODE_CARRY
}

}  // namespace parode
