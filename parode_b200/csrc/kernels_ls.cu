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

__global__ void k_sinusoid_samples(double* U, int m, int K, const double* a, const double* f, const double* phi,
                                   double base, double dt, long count)
{
    long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long total = count * m;
    if (e >= total) return;
    long j = e / m;
    int i = (int)(e - j * m);
    U[e] = sinusoid_value(a, f, phi, K, i, sample_time(base, dt, j));
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
__global__ void k_samples_batch(const SampleJob* __restrict__ jobs)
{
    const SampleJob J = jobs[blockIdx.y];
    const long total = J.count * J.m;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long j = e / J.m;
        const int i = (int)(e - j * J.m);
        J.U[e] = sinusoid_value(J.a, J.f, J.phi, J.K, i, sample_time(J.base, J.dt, j));
    }
}

__global__ void k_forcing_batch(const ForcingJob* __restrict__ jobs)
{
    const ForcingJob J = jobs[blockIdx.y];
    const long total = J.Tp * (long)J.Np;
    const int n = J.n, m = J.m;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long k = e / J.Np;
        const int i = (int)(e - k * J.Np);
        double v = 0.0;
        if (k < J.T && m > 0) {
            if (J.solver == 0) {
                if (i < n) {
                    const double* b = J.Bbar + (long)i * 3 * m;
                    const double* u = J.U + 2 * k * m;
                    for (int q = 0; q < 3 * m; ++q) v = fma(b[q], u[q], v);
                }
            } else if (i >= 3 * n && i < 4 * n) {
                const double* b = J.Bbar + (long)(i - 3 * n) * 5 * m;
                const double* u = J.U + k * m;
                for (int q = 0; q < 5 * m; ++q) v = fma(b[q], u[q], v);
            }
        }
        J.V[e] = v;
    }
}

__global__ void k_output_batch(const OutputJob* __restrict__ jobs)
{
    const OutputJob J = jobs[blockIdx.y];
    const int p = J.p, n = J.n, m = J.m;
    const long total = J.count * (long)p;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long k = e / p;
        const int o = (int)(e - k * p);
        const double* x = J.V + k * J.Np + J.xoff;
        double v = 0.0;
        if (J.zeroC && J.zeroD) {
            v = x[o];
        } else {
            if (!J.zeroC)
                for (int c = 0; c < n; ++c) v = fma(J.C[(long)o * n + c], x[c], v);
            if (!J.zeroD && m > 0) {
                const double* u = J.U + (k * J.ustride + J.uoff) * m;
                for (int c = 0; c < m; ++c) v = fma(J.D[(long)o * m + c], u[c], v);
            }
        }
        J.Y[(J.ybase + k) * p + o] = v;
    }
}

__global__ void k_copy_batch(const CopyJob* __restrict__ jobs)
{
    const CopyJob J = jobs[blockIdx.y];
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < J.N; e += (long)gridDim.x * blockDim.x)
        J.dst[e] = J.src[e];
}

inline unsigned blocks_for(long n, int t) { return (unsigned)((n + t - 1) / t); }

template <int FR, int FC>
void launch_level_t(const LevelArgs& a, int CW, cudaStream_t s)
{
    const int KS = level_ks(a.Np);
    const int NC = 8 * FC * CW;
    size_t smem = (size_t)(a.Np + NC) * (KS + 4) * sizeof(double);
    static bool attr_set = false;
    if (!attr_set) {
        PARODE_CUDA(cudaFuncSetAttribute(k_affine_level<FR, FC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         200 * 1024));
        attr_set = true;
    }
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
                             double base, double dt, long count, cudaStream_t s)
{
    long total = count * m;
    if (total <= 0) return;
    k_sinusoid_samples<<<blocks_for(total, 256), 256, 0, s>>>(U, m, K, a, f, phi, base, dt, count);
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

LevelConfig level_config(int Np)
{
    LevelConfig c;
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
    static bool attr_set = false;
    if (!attr_set) {
        PARODE_CUDA(cudaFuncSetAttribute(k_affine_level_grouped<FR, FC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr_set = true;
    }
    k_affine_level_grouped<FR, FC><<<(unsigned)tiles, kThreads, smem, s>>>(args, start, nent, c.CW);
    PARODE_CUDA(cudaGetLastError());
}
}  // namespace

void launch_affine_level_grouped(const LevelConfig& c, const LevelArgs* dArgs, const long* dStart, int nent,
                                 long tiles, size_t smem, cudaStream_t s)
{
    if (nent <= 0 || tiles <= 0) return;
    if (smem > 200 * 1024) throw Error(kInvalidArgument, "grouped level: shared memory above 200 KB");
    switch (c.id) {
    case 0: grouped_t<1, 4>(c, dArgs, dStart, nent, tiles, smem, s); break;
    case 1: grouped_t<2, 4>(c, dArgs, dStart, nent, tiles, smem, s); break;
    case 2: grouped_t<4, 4>(c, dArgs, dStart, nent, tiles, smem, s); break;
    case 3: grouped_t<8, 2>(c, dArgs, dStart, nent, tiles, smem, s); break;
    default: grouped_t<16, 1>(c, dArgs, dStart, nent, tiles, smem, s); break;
    }
}

void launch_samples_batch(const SampleJob* dJobs, int njobs, long max_elems, cudaStream_t s)
{
    if (njobs <= 0 || max_elems <= 0) return;
    dim3 grid((unsigned)std::min<long>(blocks_for(max_elems, 256), 64), (unsigned)njobs);
    k_samples_batch<<<grid, 256, 0, s>>>(dJobs);
    PARODE_CUDA(cudaGetLastError());
}

void launch_forcing_batch(const ForcingJob* dJobs, int njobs, long max_elems, cudaStream_t s)
{
    if (njobs <= 0 || max_elems <= 0) return;
    dim3 grid((unsigned)std::min<long>(blocks_for(max_elems, 256), 64), (unsigned)njobs);
    k_forcing_batch<<<grid, 256, 0, s>>>(dJobs);
    PARODE_CUDA(cudaGetLastError());
}

void launch_output_batch(const OutputJob* dJobs, int njobs, long max_elems, cudaStream_t s)
{
    if (njobs <= 0 || max_elems <= 0) return;
    dim3 grid((unsigned)std::min<long>(blocks_for(max_elems, 256), 64), (unsigned)njobs);
    k_output_batch<<<grid, 256, 0, s>>>(dJobs);
    PARODE_CUDA(cudaGetLastError());
}

void launch_copy_batch(const CopyJob* dJobs, int njobs, long max_elems, cudaStream_t s)
{
    if (njobs <= 0 || max_elems <= 0) return;
    dim3 grid((unsigned)std::min<long>(blocks_for(max_elems, 256), 16), (unsigned)njobs);
    k_copy_batch<<<grid, 256, 0, s>>>(dJobs);
    PARODE_CUDA(cudaGetLastError());
}

}  // namespace parode
