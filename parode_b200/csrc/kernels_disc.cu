// kernels_disc.cu -- the batch's discretisation on the device: per system the
// RK4 Phi / Bbar (reference Sources/RungeKutta4thOrder.cpp:36-70) or the ABM
// companion map's last block row and Bbar (Sources/AdamsMoulton.cpp:238-316),
// and ||Phi - R||_inf over the stored rows (R the exact 0/1 part: I for RK4,
// the companion shift for ABM).
//
// The matrix products (A^2, A^3, A^4 and A B, A^2 B, A^3 B; ABM needs A^2 and
// A B) run as grouped GEMMs over 32 x 32 output tiles of every system, one
// launch per dependency stage, so a large system spreads over many SMs; one
// CTA per system then forms Phi, Bbar, the transpose and the distance.  Every
// product and sum is taken in the order of the host restatement (host_math.cpp:
// discretise_rk4, discretise_abm_last; its GEMM accumulates each element over
// the inner index in order, built without FMA contraction): explicit
// __dmul_rn / __dadd_rn keep the device from contracting, and a tile's sum
// runs over the inner index in order from zero, so the device gives the host's
// bits and the batch's layout (which the distance to R sizes) is the same
// either way.
#include "common.h"
#include "kernels.h"

#include <algorithm>

namespace parode {

namespace {

constexpr int kThreads = 128;
constexpr int kTile = 32;       // output tile edge and inner-index chunk
constexpr int kPitch = kTile + 1;

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }

// Grouped tile GEMM: thread (ty, tx) owns rows ty + 16 v (v < 2) and columns
// tx + 8 u (u < 4) of its tile, eight independent in-order sums.
__global__ void __launch_bounds__(kThreads) k_disc_gemm(const DiscTile* __restrict__ tiles, long ntiles)
{
    __shared__ double Xs[kTile * kPitch];  // [row][inner]
    __shared__ double Ys[kTile * kPitch];  // [inner][col]
    const int tx = threadIdx.x & 7, ty = threadIdx.x >> 3;
    for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const DiscTile tl = tiles[t];
        double s[2][4];
#pragma unroll
        for (int v = 0; v < 2; ++v)
#pragma unroll
            for (int u = 0; u < 4; ++u) s[v][u] = 0.0;
        for (int kc = 0; kc < tl.k; kc += kTile) {
            const int kn = min(kTile, tl.k - kc);
            for (int e = threadIdx.x; e < kTile * kTile; e += kThreads) {
                const int a = e >> 5, b = e & 31;
                const int xi = tl.i0 + a, yj = tl.j0 + b;
                Xs[a * kPitch + b] = (xi < tl.r && b < kn) ? tl.X[(long)xi * tl.k + kc + b] : 0.0;
                Ys[a * kPitch + b] = (a < kn && yj < tl.c) ? tl.Y[(long)(kc + a) * tl.c + yj] : 0.0;
            }
            __syncthreads();
            // only the chunk's real inner indices: no padded products join a sum
            for (int q = 0; q < kn; ++q) {
                double x[2], y[4];
#pragma unroll
                for (int v = 0; v < 2; ++v) x[v] = Xs[(ty + 16 * v) * kPitch + q];
#pragma unroll
                for (int u = 0; u < 4; ++u) y[u] = Ys[q * kPitch + tx + 8 * u];
#pragma unroll
                for (int v = 0; v < 2; ++v)
#pragma unroll
                    for (int u = 0; u < 4; ++u) s[v][u] = add(s[v][u], mul(x[v], y[u]));
            }
            __syncthreads();
        }
#pragma unroll
        for (int v = 0; v < 2; ++v)
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = tl.i0 + ty + 16 * v, j = tl.j0 + tx + 8 * u;
                if (i < tl.r && j < tl.c) tl.Z[(long)i * tl.c + j] = s[v][u];
            }
    }
}

// Per system: Phi, Bbar (and its transpose) from the products, then the
// distance to R.  gridDim.y CTAs share a system's elementwise part (only for
// jobs without a transpose or a distance, which read all of it).
__global__ void __launch_bounds__(kThreads) k_discretise_finish(const DiscJob* __restrict__ jobs)
{
    const DiscJob jb = jobs[blockIdx.x];
    const int n = jb.n, m = jb.m, N = jb.solver == 0 ? n : 4 * n;
    const int tid = blockIdx.y * kThreads + threadIdx.x, nthr = gridDim.y * kThreads;
    const double h = jb.h, h2 = mul(h, h);
    const double* A = jb.A;
    const double* B = jb.B;
    const double* A2 = jb.work;
    const double* A3 = A2 + (long)n * n;
    const double* A4 = A3 + (long)n * n;
    const double* AB = A4 + (long)n * n;
    const double* A2B = AB + (long)n * max(m, 1);
    const double* A3B = A2B + (long)n * max(m, 1);
    const int W = jb.solver == 0 ? 3 : 5;
    // a system without B has a zero Bbar; with B every slot is written below
    if (m == 0)
        for (int e = tid; e < n * W; e += nthr) jb.bbar[e] = 0.0;
    if (jb.solver == 0) {
        const double h3 = mul(mul(h, h), h), h4 = mul(mul(mul(h, h), h), h);
        const double c2 = mul(0.5, h2), c3 = mul(1.0 / 6.0, h3), c4 = mul(1.0 / 24.0, h4);
        for (int q = tid; q < n * n; q += nthr) {
            const int i = q / n, j = q - i * n;
            double v = add(i == j ? 1.0 : 0.0, mul(h, A[q]));
            v = add(v, mul(c2, A2[q]));
            v = add(v, mul(c3, A3[q]));
            jb.phi[q] = add(v, mul(c4, A4[q]));
        }
        if (m > 0) {
            const double b1 = mul(0.5, h3), b2 = mul(0.25, h4), b3 = mul(4.0, h), b4 = mul(2.0, h2);
            const double sixth = 1.0 / 6.0, b5 = mul(sixth, h);
            for (int q = tid; q < n * m; q += nthr) {
                const int i = q / m, j = q - i * m;
                double* row = jb.bbar + (long)i * 3 * m;
                const double u = add(add(add(mul(h, B[q]), mul(h2, AB[q])), mul(b1, A2B[q])), mul(b2, A3B[q]));
                row[j] = mul(sixth, u);
                row[m + j] = mul(sixth, add(add(mul(b3, B[q]), mul(b4, AB[q])), mul(b1, A2B[q])));
                row[2 * m + j] = mul(b5, B[q]);
            }
        }
    } else {
        // the companion map's last block row [A3 A2 A1 A0]
        const double k81 = -81.0 * h2 / 576.0, k333 = 333.0 * h2 / 576.0, k531 = -531.0 * h2 / 576.0,
                     k495 = 495.0 * h2 / 576.0;
        const double k1 = 1.0 * h / 24.0, k5 = -5.0 * h / 24.0, k28 = 28.0 * h / 24.0;
        for (int q = tid; q < n * n; q += nthr) {
            const int r = q / n, c = q - r * n;
            double* last = jb.phi + (long)r * N;
            last[c] = mul(k81, A2[q]);
            last[n + c] = add(mul(k1, A[q]), mul(k333, A2[q]));
            last[2 * n + c] = add(mul(k5, A[q]), mul(k531, A2[q]));
            last[3 * n + c] = add(add(r == c ? 1.0 : 0.0, mul(k28, A[q])), mul(k495, A2[q]));
        }
        if (m > 0) {
            const double kb1 = h / 24.0, kb19 = 19.0 * h / 24.0, kb9 = 9.0 * h / 24.0;
            for (int q = tid; q < n * m; q += nthr) {
                const int r = q / m, c = q - r * m;
                double* row = jb.bbar + (long)r * 5 * m;
                row[c] = mul(k81, AB[q]);
                row[m + c] = add(mul(kb1, B[q]), mul(k333, AB[q]));
                row[2 * m + c] = add(mul(k5, B[q]), mul(k531, AB[q]));
                row[3 * m + c] = add(mul(kb19, B[q]), mul(k495, AB[q]));
                row[4 * m + c] = mul(kb9, B[q]);
            }
        }
    }
    __syncthreads();
    // Bbar transposed (level-synchronous systems' coalesced forcing kernel)
    if (jb.bbarT) {
        const int Wm = W * m;
        for (int e = threadIdx.x; e < max(Wm, 1) * n; e += kThreads) jb.bbarT[e] = 0.0;
        __syncthreads();
        for (int e = threadIdx.x; e < n * Wm; e += kThreads) {
            const int r = e / Wm, c = e - r * Wm;
            jb.bbarT[(long)c * n + r] = jb.bbar[e];
        }
    }
    // ||Phi - R||_inf over the stored rows (each row summed in order), when
    // asked for (a batch sizes its layout with it; a single plan does not)
    if (!jb.delta) return;
    __shared__ double rowmax[kThreads];
    const int d0 = jb.solver == 0 ? 0 : 3 * n;
    double dmax = 0.0;
    for (int r = threadIdx.x; r < n; r += kThreads) {
        double sum = 0.0;
        for (int c = 0; c < N; ++c) sum = add(sum, fabs(add(jb.phi[(long)r * N + c], -(c == d0 + r ? 1.0 : 0.0))));
        dmax = fmax(dmax, sum);
    }
    rowmax[threadIdx.x] = dmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int t = 0; t < kThreads; ++t) v = fmax(v, rowmax[t]);
        *jb.delta = v;
    }
}

void push_tiles(const double* X, const double* Y, double* Z, int r, int k, int c, std::vector<DiscTile>& out)
{
    for (int i0 = 0; i0 < r; i0 += kTile)
        for (int j0 = 0; j0 < c; j0 += kTile) {
            DiscTile t;
            t.X = X;
            t.Y = Y;
            t.Z = Z;
            t.r = r;
            t.k = k;
            t.c = c;
            t.i0 = i0;
            t.j0 = j0;
            out.push_back(t);
        }
}

}  // namespace

long discretise_work_doubles(int n, int m) { return 3L * n * n + 3L * n * std::max(m, 1); }

void discretise_tiles(const DiscJob& j, int stage, std::vector<DiscTile>& out)
{
    const int n = j.n, m = j.m;
    double* A2 = j.work;
    double* A3 = A2 + (long)n * n;
    double* A4 = A3 + (long)n * n;
    double* AB = A4 + (long)n * n;
    double* A2B = AB + (long)n * std::max(m, 1);
    double* A3B = A2B + (long)n * std::max(m, 1);
    if (stage == 0) {
        push_tiles(j.A, j.A, A2, n, n, n, out);
        if (m > 0) push_tiles(j.A, j.B, AB, n, n, m, out);
    } else if (j.solver == 0 && stage == 1) {
        push_tiles(A2, j.A, A3, n, n, n, out);
        if (m > 0) push_tiles(A2, j.B, A2B, n, n, m, out);
    } else if (j.solver == 0 && stage == 2) {
        push_tiles(j.A, A3, A4, n, n, n, out);
        if (m > 0) push_tiles(A3, j.B, A3B, n, n, m, out);
    }
}

void launch_discretise_batch(const DiscJob* jobs, int njobs, const DiscTile* const tiles[3], const long ntiles[3],
                             int sms, cudaStream_t s, int parts)
{
    for (int st = 0; st < 3; ++st) {
        if (ntiles[st] <= 0) continue;
        const long grid = std::min<long>(ntiles[st], (long)std::max(sms, 1) * 8);
        k_disc_gemm<<<(unsigned)grid, kThreads, 0, s>>>(tiles[st], ntiles[st]);
        PARODE_CUDA(cudaGetLastError());
    }
    for (int k = 0; k < njobs; k += 65535) {
        const int cnt = std::min(65535, njobs - k);
        k_discretise_finish<<<dim3((unsigned)cnt, (unsigned)std::max(parts, 1)), kThreads, 0, s>>>(jobs + k);
        PARODE_CUDA(cudaGetLastError());
    }
}

}  // namespace parode
