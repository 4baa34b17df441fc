// kernels_ls.cu -- FP64 kernels of the level-synchronous Blelloch scan.
//
// The reference runs every Blelloch level as a separate set of OpenCL
// launches over (M, v) pairs (Sources/GPUFixedStepIterative.cpp:236-398).
// Here the matrix part of the sweep is the power table P_l = Phi^(2^l) (all
// up-sweep matrices of level l are equal for an LTI system, and the matrix
// down-sweep is never read for the outputs), so each level is one batched
// contraction P_l x [vectors] on the FP64 tensor cores (DMMA m8n8k4), with
// the vector add / left-right copy of the reference's MVV and RootCopy
// kernels fused into its epilogue.
#include "device_common.cuh"
#include "kernels.h"
#include "common.h"

#include <algorithm>

namespace parode {

namespace {

constexpr int kThreads = 256;

// K-slice of the staged operands for a contraction length Np.
__host__ __device__ inline int level_ks(int Np)
{
    int ks = 8192 / Np;
    ks = ks < 4 ? 4 : (ks > 32 ? 32 : ks);
    return ks & ~3;
}

// One CTA owns NC = 8*FC*CW columns and all Np rows of the result; each warp
// owns an FR x FC block of 8x8 fragments.  P and the source columns are
// staged through shared memory in K slices of KS (row pitch KS+4 doubles,
// which spreads the 8 fragment rows over distinct bank groups).
template <int FR, int FC>
__device__ void affine_level_body(const LevelArgs& a, long tile, int CW, int KS, double* smem);

template <int FR, int FC>
__global__ void __launch_bounds__(kThreads) k_affine_level(LevelArgs a, int CW, int KS)
{
    extern __shared__ double smem[];
    affine_level_body<FR, FC>(a, blockIdx.x, CW, KS, smem);
}

// Grouped form: entry e owns tiles [start[e], start[e+1]) of the grid; each
// CTA finds its entry by binary search.  KS follows each entry's Np.
template <int FR, int FC>
__global__ void __launch_bounds__(kThreads) k_affine_level_grouped(const LevelArgs* __restrict__ args,
                                                                   const long* __restrict__ start, int nent, int CW)
{
    extern __shared__ double smem[];
    const long t = blockIdx.x;
    int lo = 0, hi = nent - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    const LevelArgs a = args[lo];
    affine_level_body<FR, FC>(a, t - start[lo], CW, level_ks(a.Np), smem);
}

template <int FR, int FC>
__device__ void affine_level_body(const LevelArgs& a, long tile, int CW, int KS, double* smem)
{
    const int ldk = KS + 4;
    double* sP = smem;
    const int NC = 8 * FC * CW;
    double* sV = smem + (long)a.Np * ldk;
    const long g0 = tile * NC;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = warp / CW, wc = warp % CW;
    const int gq = lane >> 2, tq = lane & 3;
    const int rf = a.Np >> 3;

    double acc[FR][FC][2];
#pragma unroll
    for (int r = 0; r < FR; ++r)
#pragma unroll
        for (int b = 0; b < FC; ++b) acc[r][b][0] = acc[r][b][1] = 0.0;

    for (int k0 = 0; k0 < a.Np; k0 += KS) {
        const int kl = min(KS, a.Np - k0);
        for (int e = tid; e < a.Np * kl; e += kThreads) {
            int r = e / kl, kk = e - r * kl;
            sP[r * ldk + kk] = a.P[(long)r * a.ldp + k0 + kk];
        }
        for (int e = tid; e < NC * kl; e += kThreads) {
            int c = e / kl, kk = e - c * kl;
            long g = g0 + c;
            sV[c * ldk + kk] = (g < a.ncols) ? a.src[g * a.src_gs + (long)(k0 + kk) * a.src_ks] : 0.0;
        }
        __syncthreads();
        for (int kk = 0; kk < kl; kk += 4) {
            double bf[FC];
#pragma unroll
            for (int b = 0; b < FC; ++b) bf[b] = sV[((wc * FC + b) * 8 + gq) * ldk + kk + tq];
#pragma unroll
            for (int r = 0; r < FR; ++r) {
                const int rb = wr * FR + r;
                if (rb < rf) {
                    double af = sP[(rb * 8 + gq) * ldk + kk + tq];
#pragma unroll
                    for (int b = 0; b < FC; ++b) dmma_m8n8k4(acc[r][b][0], acc[r][b][1], af, bf[b]);
                }
            }
        }
        __syncthreads();
    }

#pragma unroll
    for (int r = 0; r < FR; ++r) {
        const int rb = wr * FR + r;
        if (rb >= rf) continue;
        const long i = rb * 8 + gq;
#pragma unroll
        for (int b = 0; b < FC; ++b)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const long g = g0 + (wc * FC + b) * 8 + 2 * tq + e;
                if (g >= a.ncols) continue;
                double v = acc[r][b][e];
                double old_src = 0.0;
                if (a.cpy) old_src = a.src[g * a.src_gs + i * a.src_ks];
                if (a.acc) v += a.acc[g * a.acc_gs + i * a.acc_is];
                if (a.cpy) a.cpy[g * a.cpy_gs + i * a.cpy_is] = old_src;
                a.dst[g * a.dst_gs + i * a.dst_is] = v;
            }
    }
}

// ---------------------------------------------------------------------------
// Tiled level contraction for contraction lengths above 64: CTA tile of
// 64 rows x 64 columns, K slices of 32 staged by cp.async in a 3-stage ring,
// 8 warps of 32 x 16 (eight independent m8n8k4 DMMA accumulators each).
// The result must not alias the source (the down-sweep swaps first).
// kTileKC: the source columns are K-contiguous (src_ks == 1, the sweeps);
// otherwise N-contiguous (src_gs == 1, the power-table squaring).
// ---------------------------------------------------------------------------

constexpr int kTM = 64, kTN = 64, kTK = 32, kTStages = 3;
constexpr int kLdA = kTK + 4;   // A tile [64 rows][36]: rows g and g+4 of a fragment in distinct bank halves
constexpr int kLdBk = kTK + 4;  // B tile, K-contiguous: [64 cols][36]
constexpr int kLdBn = kTN + 4;  // B tile, N-contiguous: [32 k][68]
constexpr int kStageA = kTM * kLdA;
constexpr int kStageB = (kTN * kLdBk > kTK * kLdBn) ? kTN * kLdBk : kTK * kLdBn;
constexpr size_t kTiledSmem = (size_t)kTStages * (kStageA + kStageB) * sizeof(double);

__device__ __forceinline__ void cp_async16(double* dst, const double* src, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    const int bytes = valid ? 16 : 0;  // 0: the 16 bytes are zero-filled and src is not read
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <bool kKC>
__device__ void tiled_load(const LevelArgs& a, int m0, long n0, int k0, double* sA, double* sB)
{
    const int tid = threadIdx.x;
    const int rows = level_rows(a), K = level_k(a);  // K even: a 2-double chunk is wholly in or out
    const long scols = a.src_cols > 0 ? a.src_cols : a.ncols;
    // A: 64 rows x 32 doubles = 1024 chunks of 16 bytes
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int c = tid + q * 256;
        const int r = c >> 4, kc = (c & 15) * 2;
        const bool ok = (m0 + r < rows) && (k0 + kc < K);
        const double* src = ok ? a.P + (long)(m0 + r) * a.ldp + k0 + kc : a.P;
        cp_async16(sA + r * kLdA + kc, src, ok);
    }
    if (kKC) {
        // B: 64 columns x 32 doubles of K, each column contiguous in K
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = tid + q * 256;
            const int col = c >> 4, kc = (c & 15) * 2;
            const long g = n0 + col;
            const int k = k0 + kc;
            const bool ok = (g < scols) && (k < K);
            const double* src = !ok ? a.src
                                    : (a.K1 > 0 && k >= a.K1) ? a.src2 + g * a.src2_gs + (k - a.K1)
                                                              : a.src + g * a.src_gs + k;
            cp_async16(sB + col * kLdBk + kc, src, ok);
        }
    } else {
        // B: 32 rows of K x 64 columns, each row contiguous in N
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = tid + q * 256;
            const int kr = c >> 5, nc = (c & 31) * 2;
            const long g = n0 + nc;
            const bool ok = (g < scols) && (k0 + kr < K);
            const double* src = ok ? a.src + (long)(k0 + kr) * a.src_ks + g : a.src;
            cp_async16(sB + kr * kLdBn + nc, src, ok);
        }
    }
}

template <bool kKC>
__device__ void tiled_level_body(const LevelArgs& a, long tile, double* smem)
{
    const int rows = level_rows(a);
    const int mt = (rows + kTM - 1) / kTM;
    const int m0 = (int)(tile % mt) * kTM;
    const long n0 = (tile / mt) * kTN;
    double* sA = smem;
    double* sB = smem + kTStages * kStageA;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int gq = lane >> 2, tq = lane & 3;
    // a tile wholly beyond the source columns only writes acc (or zeros)
    const long scols = a.src_cols > 0 ? a.src_cols : a.ncols;
    const int nk = n0 >= scols ? 0 : (level_k(a) + kTK - 1) / kTK;

    double acc[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < kTStages - 1; ++s) {
        if (s < nk) tiled_load<kKC>(a, m0, n0, s * kTK, sA + s * kStageA, sB + s * kStageB);
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<kTStages - 2>();
        __syncthreads();
        {
            const int nx = kt + kTStages - 1;
            const int st = nx % kTStages;
            if (nx < nk) tiled_load<kKC>(a, m0, n0, nx * kTK, sA + st * kStageA, sB + st * kStageB);
            cp_async_commit();
        }
        const double* A = sA + (kt % kTStages) * kStageA;
        const double* B = sB + (kt % kTStages) * kStageB;
#pragma unroll
        for (int kk = 0; kk < kTK; kk += 4) {
            double af[4], bf[2];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = A[(wm * 32 + i * 8 + gq) * kLdA + kk + tq];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int col = wn * 16 + j * 8 + gq;
                bf[j] = kKC ? B[col * kLdBk + kk + tq] : B[(kk + tq) * kLdBn + col];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) dmma_m8n8k4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
    }
    cp_async_wait<0>();

    // acc may be dst itself (in place): every acc value is loaded before the
    // first store, so the sixteen loads go out together instead of each
    // waiting behind the store before it
    if (a.acc) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const long r = m0 + wm * 32 + i * 8 + gq;
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const long g = n0 + wn * 16 + j * 8 + 2 * tq + e;
                    const long o = g * a.dst_gs + r * a.dst_is;
                    // exactly the elements stored below (acc past dst_limit may lie past its buffer)
                    if (r < rows && g < a.ncols && !(a.dst_limit >= 0 && o >= a.dst_limit))
                        acc[i][j][e] += a.acc[g * a.acc_gs + r * a.acc_is];
                }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const long r = m0 + wm * 32 + i * 8 + gq;
        if (r >= rows) continue;
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const long g = n0 + wn * 16 + j * 8 + 2 * tq + e;
                if (g >= a.ncols) continue;
                const long o = g * a.dst_gs + r * a.dst_is;
                if (a.dst_limit >= 0 && o >= a.dst_limit) continue;
                a.dst[o] = acc[i][j][e];
            }
    }
}

template <bool kKC>
__global__ void __launch_bounds__(kThreads, 2) k_level_tiled(LevelArgs a)
{
    extern __shared__ double smem[];
    tiled_level_body<kKC>(a, blockIdx.x, smem);
}

template <bool kKC>
__global__ void __launch_bounds__(kThreads, 2) k_level_tiled_grouped(const LevelArgs* __restrict__ args,
                                                                     const long* __restrict__ start, int nent)
{
    extern __shared__ double smem[];
    const long t = blockIdx.x;
    int lo = 0, hi = nent - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    const LevelArgs a = args[lo];
    tiled_level_body<kKC>(a, t - start[lo], smem);
}

// Down-sweep bookkeeping before a tiled level: cpy(g, i) <-> dst(g, i).
__device__ void swap_body(const LevelArgs& a)
{
    const long total = a.ncols * (long)a.Np;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long g = e / a.Np;
        const long i = e - g * a.Np;
        double* x = a.cpy + g * a.cpy_gs + i * a.cpy_is;
        double* y = a.dst + g * a.dst_gs + i * a.dst_is;
        const double t = *x;
        *x = *y;
        *y = t;
    }
}

__global__ void k_swap(LevelArgs a) { swap_body(a); }

// Grouped form: blockIdx.y selects the entry.
__global__ void k_swap_grouped(const LevelArgs* __restrict__ args)
{
    const LevelArgs a = args[blockIdx.y];
    swap_body(a);
}

// One thread per (run of kSampleRun samples, channel); channels fastest.
template <int KMAX>
__global__ void k_sinusoid_samples(double* U, int m, int K, const double* a, const double* f, const double* phi,
                                   double base, double dt, long count, long joff)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long runs = (count + kSampleRun - 1) / kSampleRun;
    if (e >= runs * m) return;
    const long r = e / m;
    const int i = (int)(e - r * m);
    const long j0 = r * kSampleRun;
    sinusoid_run<kSampleRun, KMAX>(a, f, phi, K, i, base, dt, j0, count, SampleOut64{U + j0 * m + i, m}, joff);
}

// The same samples as TF32 hi / lo planes (the tensor-core GEMMs' operands),
// by the plain rotation (sinusoid_rot: the planes' own rounding is 2^-22).
template <int KMAX>
__global__ void k_sinusoid_planes(float* hi, float* lo, int m, int K, const double* a, const double* f,
                                  const double* phi, double base, double dt, long count, long joff)
{
    grid_dep_trigger();  // the response GEMMs may set up meanwhile (they wait for these samples)
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long runs = (count + kSampleRun - 1) / kSampleRun;
    if (e >= runs * m) return;
    const long r = e / m;
    const int i = (int)(e - r * m);
    const long j0 = r * kSampleRun;
    sinusoid_rot<kSampleRun, KMAX>(a, f, phi, K, i, base, dt, j0, count,
                                   SampleOutSplit{hi + j0 * m + i, lo ? lo + j0 * m + i : nullptr, m}, joff);
}

// FP64 samples (any input function) into TF32 hi / lo planes.
__global__ void k_split_planes(const double* __restrict__ U, float* __restrict__ hi, float* __restrict__ lo, long n)
{
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
        SampleOutSplit{hi, lo, 1}(e, U[e]);
}

// V[k][i] = Gamma_k[i]; RK4: Gamma_k = Bbar [u_2k; u_2k+1; u_2k+2] in rows
// 0..n-1 (Kernels/BTimesURK4thOrder.cl:15-37 of the reference); ABM:
// Gamma_k = [0; 0; 0; Bbar [u_k .. u_k+4]] (Kernels/BTimesUAdamsMoulton.cl:17-38).
__global__ void k_forcing(double* V, int Np, int n, int m, int solver, const double* Bbar, const double* U,
                          long T, long Tp)
{
    long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Tp * (long)Np) return;
    long k = e / Np;
    int i = (int)(e - k * Np);
    double v = 0.0;
    if (k < T && m > 0) {
        if (solver == 0) {
            if (i < n) {
                const double* b = Bbar + (long)i * 3 * m;
                const double* u = U + 2 * k * m;
                for (int q = 0; q < 3 * m; ++q) v = fma(b[q], u[q], v);
            }
        } else if (i >= 3 * n && i < 4 * n) {
            const double* b = Bbar + (long)(i - 3 * n) * 5 * m;
            const double* u = U + k * m;
            for (int q = 0; q < 5 * m; ++q) v = fma(b[q], u[q], v);
        }
    }
    V[e] = v;
}

// y_k = C x_k + D u_k (Kernels/SystemOutput.cl:28-59 of the reference), or
// y_k = x_k when C and D are both absent.
__global__ void k_output(double* Y, const double* V, int Np, int xoff, int n, int m, int p, const double* C,
                         const double* D, int zeroC, int zeroD, const double* U, int ustride, int uoff, long count,
                         long ybase)
{
    long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count * (long)p) return;
    long k = e / p;
    int o = (int)(e - k * p);
    const double* x = V + k * Np + xoff;
    double v = 0.0;
    if (zeroC && zeroD) {
        v = x[o];
    } else {
        if (!zeroC)
            for (int c = 0; c < n; ++c) v = fma(C[(long)o * n + c], x[c], v);
        if (!zeroD && m > 0) {
            const double* u = U + (k * ustride + uoff) * m;
            for (int c = 0; c < m; ++c) v = fma(D[(long)o * m + c], u[c], v);
        }
    }
    Y[(ybase + k) * p + o] = v;
}

__global__ void k_copy(double* dst, const double* src, long N)
{
    long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < N) dst[e] = src[e];
}

// Batched element kernels: blockIdx.y selects the job, the x dimension
// strides over its elements; each element is computed as by the single-system
// kernels above.
template <int KMAX>
__global__ void k_samples_batch(const SampleJob* __restrict__ jobs)
{
    const SampleJob J = jobs[blockIdx.y];
    const long runs = (J.count + kSampleRun - 1) / kSampleRun;
    const long total = runs * J.m;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long r = e / J.m;
        const int i = (int)(e - r * J.m);
        const long j0 = r * kSampleRun;
        sinusoid_run<kSampleRun, KMAX>(J.a, J.f, J.phi, J.K, i, J.base, J.dt, j0, J.count,
                                       SampleOut64{J.U + j0 * J.m + i, J.m});
    }
}

// Rows (steps) are dealt to the CTAs of the job; a row's components to the
// threads (no per-element division).  Forcing rows: RK4 0..n-1, ABM 3n..4n-1.
__global__ void k_forcing_batch(const ForcingJob* __restrict__ jobs)
{
    const ForcingJob& J = jobs[blockIdx.y];
    const int n = J.n, m = J.m, Np = J.Np;
    const bool rk4 = J.solver == 0;
    const int lo = rk4 ? 0 : 3 * n, W = rk4 ? 3 : 5;
    const long ustep = rk4 ? 2L * m : (long)m;
    for (long k = blockIdx.x; k < J.Tp; k += gridDim.x) {
        double* row = J.V + k * Np;
        const double* u = J.U + k * ustep;
        for (int i = threadIdx.x; i < Np; i += blockDim.x) {
            double v = 0.0;
            if (k < J.T && m > 0 && i >= lo && i < lo + n) {
                const double* b = J.BbarT + (i - lo);  // consecutive threads, consecutive addresses
                for (int q = 0; q < W * m; ++q) v = fma(b[(long)q * n], u[q], v);
            }
            row[i] = v;
        }
    }
}

// Output rows: a CTA covers blockDim/p rows at a time, thread (r, o) one output.
__global__ void k_output_batch(const OutputJob* __restrict__ jobs)
{
    const OutputJob& J = jobs[blockIdx.y];
    const int p = J.p, n = J.n, m = J.m;
    const int rows = p <= (int)blockDim.x ? (int)blockDim.x / p : 1;
    const int r = p <= (int)blockDim.x ? (int)threadIdx.x / p : 0;
    if (r >= rows) return;
    const int o0 = p <= (int)blockDim.x ? (int)threadIdx.x - r * p : (int)threadIdx.x;
    const int ostep = p <= (int)blockDim.x ? p : (int)blockDim.x;
    for (long k = (long)blockIdx.x * rows + r; k < J.count; k += (long)gridDim.x * rows) {
        const double* x = J.V + k * J.Np + J.xoff;
        const double* u = (!J.zeroD && m > 0) ? J.U + (k * J.ustride + J.uoff) * m : nullptr;
        for (int o = o0; o < p; o += ostep) {
            double v = 0.0;
            if (J.zeroC && J.zeroD) {
                v = x[o];
            } else {
                if (!J.zeroC)
                    for (int c = 0; c < n; ++c) v = fma(J.CT[(long)c * p + o], x[c], v);
                if (u)
                    for (int c = 0; c < m; ++c) v = fma(J.DT[(long)c * p + o], u[c], v);
            }
            J.Y[(J.ybase + k) * p + o] = v;
        }
    }
}

__global__ void k_copy_batch(const CopyJob* __restrict__ jobs)
{
    const CopyJob J = jobs[blockIdx.y];
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < J.N; e += (long)gridDim.x * blockDim.x)
        J.dst[e] = J.src ? J.src[e] : 0.0;
}

__global__ void k_phi_batch(const PhiJob* __restrict__ jobs)
{
    const PhiJob J = jobs[blockIdx.y];
    const long total = (long)J.Np * J.Np;
    const int n = J.n;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const int r = (int)(e / J.Np), c = (int)(e - (long)r * J.Np);
        double v = 0.0;
        if (J.solver == 0) {
            if (r < n && c < n) v = J.src[(long)r * n + c];
        } else if (r < 3 * n) {
            v = (c == r + n) ? 1.0 : 0.0;
        } else if (r < 4 * n && c < 4 * n) {
            v = J.src[(long)(r - 3 * n) * (4 * n) + c];
        }
        J.dst[e] = v;
    }
}

inline unsigned blocks_for(long n, int t) { return (unsigned)((n + t - 1) / t); }

// x extent of a batched launch (y = jobs): `cap` CTAs per job, raised so
// that the whole grid has about 2048 CTAs when the jobs are few, and never
// more than the largest job needs.
inline unsigned batch_grid_x(long max_elems, int per_cta, int cap, int njobs)
{
    const long want = std::max<long>(cap, (2048 + njobs - 1) / njobs);
    return (unsigned)std::max<long>(1, std::min<long>(blocks_for(max_elems, per_cta), want));
}

// Arguments of the tiled contraction for a level: the down-sweep (cpy set)
// becomes, after the swap, right = P left + right.
LevelArgs tiled_args(const LevelArgs& a)
{
    LevelArgs b = a;
    if (a.cpy) {
        b.src = a.cpy;
        b.src_gs = a.cpy_gs;
        b.src_ks = a.cpy_is;
        b.acc = a.dst;
        b.acc_gs = a.dst_gs;
        b.acc_is = a.dst_is;
        b.cpy = nullptr;
    }
    if (b.src_ks != 1 && b.src_gs != 1) throw Error(kInvalidArgument, "tiled level: source neither K- nor N-contiguous");
    return b;
}

long tiled_tiles(const LevelArgs& b)
{
    return (long)((level_rows(b) + kTM - 1) / kTM) * ((b.ncols + kTN - 1) / kTN);
}

template <int FR, int FC>
void launch_level_t(const LevelArgs& a, int CW, cudaStream_t s)
{
    const int KS = level_ks(a.Np);
    const int NC = 8 * FC * CW;
    size_t smem = (size_t)(a.Np + NC) * (KS + 4) * sizeof(double);
    // set on every launch: per device, and safe with several host threads
    PARODE_CUDA(cudaFuncSetAttribute(k_affine_level<FR, FC>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    unsigned grid = blocks_for(a.ncols, NC);
    k_affine_level<FR, FC><<<grid, kThreads, smem, s>>>(a, CW, KS);
    PARODE_CUDA(cudaGetLastError());
}

}  // namespace

void launch_affine_level(const LevelArgs& a, cudaStream_t s)
{
    if (a.ncols <= 0) return;
    if (a.Np <= 0 || (a.Np & 7) != 0 || a.Np > 1024)
        throw Error(kInvalidArgument, "scan dimension must be a positive multiple of 8 up to 1024");
    if (a.Np > 64) {
        // tiled contraction; the down-sweep first swaps (left, right), then
        // right = P left + right (the tile's result must not alias its source)
        LevelArgs b = tiled_args(a);
        if (a.cpy) {
            k_swap<<<(unsigned)std::min<long>(blocks_for(a.ncols * (long)a.Np, 256), 4096), 256, 0, s>>>(a);
            PARODE_CUDA(cudaGetLastError());
        }
        PARODE_CUDA(cudaFuncSetAttribute(k_level_tiled<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTiledSmem));
        PARODE_CUDA(cudaFuncSetAttribute(k_level_tiled<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTiledSmem));
        const long tiles = tiled_tiles(b);
        if (b.src_ks == 1) k_level_tiled<true><<<(unsigned)tiles, kThreads, kTiledSmem, s>>>(b);
        else k_level_tiled<false><<<(unsigned)tiles, kThreads, kTiledSmem, s>>>(b);
        PARODE_CUDA(cudaGetLastError());
        return;
    }
    const int rf = a.Np / 8;
    if (rf <= 8) {
        int RW = 1;
        while (RW < rf) RW <<= 1;
        launch_level_t<1, 4>(a, 8 / RW, s);
    } else if (rf <= 16) {
        launch_level_t<2, 4>(a, 1, s);
    } else if (rf <= 32) {
        launch_level_t<4, 4>(a, 1, s);
    } else if (rf <= 64) {
        launch_level_t<8, 2>(a, 1, s);
    } else {
        launch_level_t<16, 1>(a, 1, s);
    }
}

void launch_sinusoid_samples(double* U, int m, int K, const double* a, const double* f, const double* phi,
                             double base, double dt, long count, cudaStream_t s, long joff)
{
    if (count <= 0 || m <= 0) return;
    const long total = (count + kSampleRun - 1) / kSampleRun * m;
    const unsigned g = (unsigned)blocks_for(total, 256);
    switch (sample_kmax(K)) {
    case 1: k_sinusoid_samples<1><<<g, 256, 0, s>>>(U, m, K, a, f, phi, base, dt, count, joff); break;
    case 2: k_sinusoid_samples<2><<<g, 256, 0, s>>>(U, m, K, a, f, phi, base, dt, count, joff); break;
    case 3: k_sinusoid_samples<3><<<g, 256, 0, s>>>(U, m, K, a, f, phi, base, dt, count, joff); break;
    default: k_sinusoid_samples<4><<<g, 256, 0, s>>>(U, m, K, a, f, phi, base, dt, count, joff); break;
    }
    PARODE_CUDA(cudaGetLastError());
}

void launch_sinusoid_planes(float* hi, float* lo, int m, int K, const double* a, const double* f, const double* phi,
                            double base, double dt, long count, cudaStream_t s, long joff)
{
    if (count <= 0 || m <= 0) return;
    const long total = (count + kSampleRun - 1) / kSampleRun * m;
    const unsigned g = (unsigned)blocks_for(total, 256);
    switch (sample_kmax(K)) {
    case 1: k_sinusoid_planes<1><<<g, 256, 0, s>>>(hi, lo, m, K, a, f, phi, base, dt, count, joff); break;
    case 2: k_sinusoid_planes<2><<<g, 256, 0, s>>>(hi, lo, m, K, a, f, phi, base, dt, count, joff); break;
    case 3: k_sinusoid_planes<3><<<g, 256, 0, s>>>(hi, lo, m, K, a, f, phi, base, dt, count, joff); break;
    default: k_sinusoid_planes<4><<<g, 256, 0, s>>>(hi, lo, m, K, a, f, phi, base, dt, count, joff); break;
    }
    PARODE_CUDA(cudaGetLastError());
}

// y rounded to float (the reference C ABI's output arrays), two per thread
__global__ void k_to_float(const double* __restrict__ src, float* __restrict__ dst, long n)
{
    for (long i = 2 * ((long)blockIdx.x * blockDim.x + threadIdx.x); i < n; i += 2L * gridDim.x * blockDim.x) {
        dst[i] = (float)src[i];
        if (i + 1 < n) dst[i + 1] = (float)src[i + 1];
    }
}

void launch_to_float(const double* src, float* dst, long n, cudaStream_t s)
{
    if (n <= 0) return;
    k_to_float<<<(unsigned)std::min<long>((n / 2 + 255) / 256 + 1, 148L * 16), 256, 0, s>>>(src, dst, n);
    PARODE_CUDA(cudaGetLastError());
}

void launch_split_planes(const double* U, float* hi, float* lo, long n, cudaStream_t s)
{
    if (n <= 0) return;
    k_split_planes<<<(unsigned)std::min<long>((n + 255) / 256, 148L * 16), 256, 0, s>>>(U, hi, lo, n);
    PARODE_CUDA(cudaGetLastError());
}

void launch_forcing(double* V, int Np, int n, int m, int solver, const double* Bbar, const double* U, long T,
                    long Tp, cudaStream_t s)
{
    long total = Tp * (long)Np;
    k_forcing<<<blocks_for(total, 256), 256, 0, s>>>(V, Np, n, m, solver, Bbar, U, T, Tp);
    PARODE_CUDA(cudaGetLastError());
}

void launch_output(double* Y, const double* V, int Np, int xoff, int n, int m, int p, const double* C,
                   const double* D, int zeroC, int zeroD, const double* U, int ustride, int uoff, long count,
                   long ybase, cudaStream_t s)
{
    long total = count * (long)p;
    if (total <= 0) return;
    k_output<<<blocks_for(total, 256), 256, 0, s>>>(Y, V, Np, xoff, n, m, p, C, D, zeroC, zeroD, U, ustride, uoff,
                                                    count, ybase);
    PARODE_CUDA(cudaGetLastError());
}

void launch_copy(double* dst, const double* src, long N, cudaStream_t s)
{
    if (N <= 0) return;
    k_copy<<<blocks_for(N, 256), 256, 0, s>>>(dst, src, N);
    PARODE_CUDA(cudaGetLastError());
}

int launches_per_level() { return 1; }

// ---------------------------------------------------------------------------
// grouped / batched launchers
// ---------------------------------------------------------------------------

LevelConfig level_config(const LevelArgs& a)
{
    LevelConfig c;
    const int Np = a.Np;
    if (Np > 64 || a.M > 0 || a.K > 0) {
        const LevelArgs b = tiled_args(a);
        c.id = b.src_ks == 1 ? 5 : 6;
        c.NC = kTN;
        c.smem = kTiledSmem;
        return c;
    }
    const int rf = Np / 8;
    if (rf <= 8) {
        int RW = 1;
        while (RW < rf) RW <<= 1;
        c.id = 0;
        c.CW = 8 / RW;
    } else if (rf <= 16) {
        c.id = 1;
    } else if (rf <= 32) {
        c.id = 2;
    } else if (rf <= 64) {
        c.id = 3;
    } else {
        c.id = 4;
    }
    static const int fc[5] = {4, 4, 4, 2, 1};
    c.NC = 8 * fc[c.id] * c.CW;
    c.smem = (size_t)(Np + c.NC) * (level_ks(Np) + 4) * sizeof(double);
    return c;
}

namespace {
template <int FR, int FC>
void grouped_t(const LevelConfig& c, const LevelArgs* args, const long* start, int nent, long tiles, size_t smem,
               cudaStream_t s)
{
    PARODE_CUDA(cudaFuncSetAttribute(k_affine_level_grouped<FR, FC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     200 * 1024));
    k_affine_level_grouped<FR, FC><<<(unsigned)tiles, kThreads, smem, s>>>(args, start, nent, c.CW);
    PARODE_CUDA(cudaGetLastError());
}
}  // namespace

void launch_affine_level_grouped(const LevelConfig& c, const LevelArgs* dArgs, const long* dStart, int nent,
                                 long tiles, size_t smem, cudaStream_t s)
{
    if (nent <= 0 || tiles <= 0) return;
    if (c.id >= 5) {
        PARODE_CUDA(cudaFuncSetAttribute(k_level_tiled_grouped<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTiledSmem));
        PARODE_CUDA(cudaFuncSetAttribute(k_level_tiled_grouped<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTiledSmem));
        if (c.id == 5) k_level_tiled_grouped<true><<<(unsigned)tiles, kThreads, kTiledSmem, s>>>(dArgs, dStart, nent);
        else k_level_tiled_grouped<false><<<(unsigned)tiles, kThreads, kTiledSmem, s>>>(dArgs, dStart, nent);
        PARODE_CUDA(cudaGetLastError());
        return;
    }
    if (smem > 200 * 1024) throw Error(kInvalidArgument, "grouped level: shared memory above 200 KB");
    switch (c.id) {
    case 0: grouped_t<1, 4>(c, dArgs, dStart, nent, tiles, smem, s); break;
    case 1: grouped_t<2, 4>(c, dArgs, dStart, nent, tiles, smem, s); break;
    case 2: grouped_t<4, 4>(c, dArgs, dStart, nent, tiles, smem, s); break;
    case 3: grouped_t<8, 2>(c, dArgs, dStart, nent, tiles, smem, s); break;
    default: grouped_t<16, 1>(c, dArgs, dStart, nent, tiles, smem, s); break;
    }
}

LevelArgs level_grouped_args(const LevelArgs& a) { return (a.Np > 64 || a.M > 0 || a.K > 0) ? tiled_args(a) : a; }

void launch_gemm_tiled(const LevelArgs& a, cudaStream_t s)
{
    if (a.ncols <= 0) return;
    if (level_k(a) <= 0 || (level_k(a) & 1) || level_rows(a) <= 0 || (a.src_ks != 1 && a.src_gs != 1) ||
        (a.ldp & 1) || a.cpy)
        throw Error(kInvalidArgument, "tiled GEMM: even K, even ldp, K- or N-contiguous source, no copy");
    if (a.K1 > 0 && ((a.K1 & 1) || a.K1 >= level_k(a) || a.src_ks != 1 || !a.src2 || (a.src2_gs & 1) ||
                     (a.src_gs & 1)))
        throw Error(kInvalidArgument, "tiled GEMM: two-part source needs even K1 < K, K-contiguous, even strides");
    PARODE_CUDA(cudaFuncSetAttribute(k_level_tiled<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kTiledSmem));
    PARODE_CUDA(cudaFuncSetAttribute(k_level_tiled<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kTiledSmem));
    const long tiles = tiled_tiles(a);
    if (a.src_ks == 1) k_level_tiled<true><<<(unsigned)tiles, kThreads, kTiledSmem, s>>>(a);
    else k_level_tiled<false><<<(unsigned)tiles, kThreads, kTiledSmem, s>>>(a);
    PARODE_CUDA(cudaGetLastError());
}

long level_tiles(const LevelConfig& c, const LevelArgs& stored)
{
    if (c.id >= 5) return tiled_tiles(stored);
    return (stored.ncols + c.NC - 1) / c.NC;
}

void launch_swap_grouped(const LevelArgs* dArgs, int nent, long max_elems, cudaStream_t s)
{
    if (nent <= 0 || max_elems <= 0) return;
    dim3 grid((unsigned)std::min<long>(blocks_for(max_elems, 256), 64), (unsigned)nent);
    k_swap_grouped<<<grid, 256, 0, s>>>(dArgs);
    PARODE_CUDA(cudaGetLastError());
}

void launch_samples_batch(const SampleJob* dJobs, int njobs, long max_elems, int max_terms, cudaStream_t s)
{
    if (njobs <= 0 || max_elems <= 0) return;
    dim3 grid(batch_grid_x(max_elems, 256, 64, njobs), (unsigned)njobs);
    switch (sample_kmax(max_terms)) {
    case 1: k_samples_batch<1><<<grid, 256, 0, s>>>(dJobs); break;
    case 2: k_samples_batch<2><<<grid, 256, 0, s>>>(dJobs); break;
    case 3: k_samples_batch<3><<<grid, 256, 0, s>>>(dJobs); break;
    default: k_samples_batch<4><<<grid, 256, 0, s>>>(dJobs); break;
    }
    PARODE_CUDA(cudaGetLastError());
}

void launch_forcing_batch(const ForcingJob* dJobs, int njobs, long max_elems, cudaStream_t s)
{
    if (njobs <= 0 || max_elems <= 0) return;
    // max_elems: the largest Tp x Np; a CTA of 128 threads walks rows
    dim3 grid(batch_grid_x(max_elems, 1024, 256, njobs), (unsigned)njobs);
    k_forcing_batch<<<grid, 128, 0, s>>>(dJobs);
    PARODE_CUDA(cudaGetLastError());
}

void launch_output_batch(const OutputJob* dJobs, int njobs, long max_elems, cudaStream_t s)
{
    if (njobs <= 0 || max_elems <= 0) return;
    dim3 grid(batch_grid_x(max_elems, 2048, 128, njobs), (unsigned)njobs);
    k_output_batch<<<grid, 256, 0, s>>>(dJobs);
    PARODE_CUDA(cudaGetLastError());
}

void launch_copy_batch(const CopyJob* dJobs, int njobs, long max_elems, cudaStream_t s)
{
    if (njobs <= 0 || max_elems <= 0) return;
    dim3 grid(batch_grid_x(max_elems, 256, 16, njobs), (unsigned)njobs);
    k_copy_batch<<<grid, 256, 0, s>>>(dJobs);
    PARODE_CUDA(cudaGetLastError());
}

void launch_phi_batch(const PhiJob* dJobs, int njobs, long max_elems, cudaStream_t s)
{
    if (njobs <= 0 || max_elems <= 0) return;
    dim3 grid(batch_grid_x(max_elems, 256, 16, njobs), (unsigned)njobs);
    k_phi_batch<<<grid, 256, 0, s>>>(dJobs);
    PARODE_CUDA(cudaGetLastError());
}

}  // namespace parode
