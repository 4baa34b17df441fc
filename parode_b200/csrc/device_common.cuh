// device_common.cuh -- device helpers shared by the scan kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <utility>

#include "common.h"

namespace parode {

// Programmatic dependent launch (a kernel launched by launch_dependent may
// start while the kernel before it in the stream finishes): grid_dep_wait()
// returns once the grids it depends on have completed and their memory is
// visible (at once for a kernel launched the ordinary way); every read of
// their results, and every write, comes after it.  grid_dep_trigger() lets
// the dependent grid's CTAs be scheduled once every CTA of this grid has
// called it (or exited), so the dependents' own prologue (loads of data no
// kernel in flight writes) overlaps this grid's work.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void grid_dep_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

template <typename... K, typename... A>
void launch_dependent(void (*kernel)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    PARODE_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
}

// D(8x8) += A(8x4, row) * B(4x8, col), FP64 tensor-core MMA.
// Fragments (PTX ISA, mma.m8n8k4 .f64): lane = 4*g + t with g = lane>>2,
// t = lane&3; A holds A[g][t], B holds B[t][g], D holds D[g][2t], D[g][2t+1].
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Sum-of-sinusoids input with an explicit operation order (no contraction),
// matching the host-side evaluation order a * sin((2 pi f) t + phi).
__device__ __forceinline__ double sinusoid_value(const double* a, const double* f, const double* phi, int K,
                                                 int i, double t)
{
    const double two_pi = 6.283185307179586476925286766559;
    double v = 0.0;
    for (int k = 0; k < K; ++k) {
        int q = i * K + k;
        double arg = __dadd_rn(__dmul_rn(__dmul_rn(two_pi, f[q]), t), phi[q]);
        v = __dadd_rn(v, __dmul_rn(a[q], sin(arg)));
    }
    return v;
}

// Where a sampler puts sample j of its run: FP64 at out[j * stride], or
// split into two TF32 planes (hi = TF32(x), lo = TF32(x - hi) with
// x = float(v), both rounded to nearest) for the tensor-core GEMMs.
struct SampleOut64 {
    double* out;
    long stride;
    __device__ __forceinline__ void operator()(long j, double v) const { out[j * stride] = v; }
};

// x rounded to TF32 (10 mantissa bits), to nearest with ties away from zero:
// half a unit of the kept last bit added to the magnitude, the 13 dropped
// bits cleared (for finite x the result of cvt.rna.tf32.f32, in two integer
// operations instead of a conversion).
__device__ __forceinline__ float tf32_rna(float x)
{
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

struct SampleOutSplit {
    float* hi;
    float* lo;
    long stride;
    __device__ __forceinline__ void operator()(long j, double v) const
    {
        const float x = (float)v;
        const float h = tf32_rna(x);
        hi[j * stride] = h;
        if (lo) lo[j * stride] = tf32_rna(x - h);  // no lo plane in the single-pass form
    }
};

// Sample time t_j = base + dt * j, rounded as the host computes it.
__device__ __forceinline__ double sample_time(double base, double dt, long j)
{
    return __dadd_rn(base, __dmul_rn(dt, (double)j));
}

// Samples j0 .. j0 + L - 1 (those below count) of channel i of the sum-of-
// sinusoid input, into out[(j - j0) * stride]: the values sinusoid_value
// gives, at a fraction of its cost.  Every argument is rounded exactly as
// sinusoid_value rounds it; each term starts from sincos at j0 and advances
// by the rotation through the difference d of consecutive arguments.  d is
// the nominal step delta = w dt plus a residue e from the roundings of t_j
// and of the arguments (|e| is a few units in the last place of the
// argument, below 1e-10 for arguments up to 1e5), so sin d and cos d come
// from sincos(delta), once per term, corrected to first order in e (the
// neglected e^2 / 2 is below 1e-20; a residue above 1e-8 takes sincos of the
// argument instead).  Both differences are exact for
// arguments of one sign within a factor 2.  The rotations add a few units in
// the last place per step: about 2e-14 of the amplitude after 64 steps.  The
// terms (a compile-time count, so that each has its own registers) advance
// side by side as independent chains and are summed in sinusoid_value's
// order; inputs with more than 4 terms per channel take sinusoid_value per
// sample.
template <int L, int KT, class Out>
__device__ __forceinline__ void sinusoid_run_terms(const double* a, const double* f, const double* phi, int i,
                                                   double base, double dt, long j0, int n, const Out& out,
                                                   long joff)
{
    const double two_pi = 6.283185307179586476925286766559;
    double w[KT], ph[KT], amp[KT], prev[KT], s[KT], c[KT], dl[KT], sdl[KT], cdl[KT];
    double v = 0.0;
#pragma unroll
    for (int q = 0; q < KT; ++q) {
        w[q] = __dmul_rn(two_pi, f[i * KT + q]);
        ph[q] = phi[i * KT + q];
        amp[q] = a[i * KT + q];
        prev[q] = __dadd_rn(__dmul_rn(w[q], sample_time(base, dt, joff + j0)), ph[q]);
        sincos(prev[q], &s[q], &c[q]);
        dl[q] = __dmul_rn(w[q], dt);
        sincos(dl[q], &sdl[q], &cdl[q]);
        v = __dadd_rn(v, __dmul_rn(amp[q], s[q]));
    }
    if (n > 0) out(0, v);
    for (int j = 1; j < n; ++j) {
        const double t = sample_time(base, dt, joff + j0 + j);
        v = 0.0;
#pragma unroll
        for (int q = 0; q < KT; ++q) {
            const double arg = __dadd_rn(__dmul_rn(w[q], t), ph[q]);
            const double e = (arg - prev[q]) - dl[q];
            prev[q] = arg;
            if (fabs(e) <= 1e-8) {
                const double sd = fma(e, cdl[q], sdl[q]);
                const double cd = fma(-e, sdl[q], cdl[q]);
                const double sn = fma(s[q], cd, c[q] * sd);
                c[q] = fma(c[q], cd, -(s[q] * sd));
                s[q] = sn;
            } else {
                sincos(arg, &s[q], &c[q]);  // arguments too large for the first-order step
            }
            v = __dadd_rn(v, __dmul_rn(amp[q], s[q]));
        }
        out(j, v);
    }
}

// The plain rotation: each term from sincos at the run's first sample, then
// rotated by sincos of the nominal step w dt, with no correction for the
// rounding of the sample times.  Against the rounded arguments the phase
// drifts by at most w ulp(t) plus ~64 roundings over a run (about 1e-13 of
// the amplitude at the benchmark's times): for the TF32 sample planes, whose
// own rounding is 2^-22, not for the FP64 samples.  5 FP64 operations per
// term and sample instead of ~14.
template <int L, int KT, class Out>
__device__ __forceinline__ void sinusoid_rot_terms(const double* a, const double* f, const double* phi, int i,
                                                   double base, double dt, long j0, int n, const Out& out, long joff)
{
    const double two_pi = 6.283185307179586476925286766559;
    double amp[KT], s[KT], c[KT], sdl[KT], cdl[KT];
    double v = 0.0;
    const double t0 = sample_time(base, dt, joff + j0);
#pragma unroll
    for (int q = 0; q < KT; ++q) {
        const double w = __dmul_rn(two_pi, f[i * KT + q]);
        amp[q] = a[i * KT + q];
        sincos(__dadd_rn(__dmul_rn(w, t0), phi[i * KT + q]), &s[q], &c[q]);
        sincos(__dmul_rn(w, dt), &sdl[q], &cdl[q]);
        v = fma(amp[q], s[q], v);
    }
    if (n > 0) out(0, v);
    for (int j = 1; j < n; ++j) {
        v = 0.0;
#pragma unroll
        for (int q = 0; q < KT; ++q) {
            const double sn = fma(s[q], cdl[q], c[q] * sdl[q]);
            c[q] = fma(c[q], cdl[q], -(s[q] * sdl[q]));
            s[q] = sn;
            v = fma(amp[q], s[q], v);
        }
        out(j, v);
    }
}

template <int L, int KMAX, class Out>
__device__ __forceinline__ void sinusoid_rot(const double* a, const double* f, const double* phi, int K, int i,
                                             double base, double dt, long j0, long count, const Out& out, long joff)
{
    const long rest = count - j0;
    const int n = rest < L ? (int)rest : L;
    if (K == 1) sinusoid_rot_terms<L, 1>(a, f, phi, i, base, dt, j0, n, out, joff);
    else if (KMAX >= 2 && K == 2) sinusoid_rot_terms<L, (KMAX >= 2 ? 2 : 1)>(a, f, phi, i, base, dt, j0, n, out, joff);
    else if (KMAX >= 3 && K == 3) sinusoid_rot_terms<L, (KMAX >= 3 ? 3 : 1)>(a, f, phi, i, base, dt, j0, n, out, joff);
    else if (KMAX >= 4 && K == 4) sinusoid_rot_terms<L, (KMAX >= 4 ? 4 : 1)>(a, f, phi, i, base, dt, j0, n, out, joff);
    else
        for (int j = 0; j < n; ++j) out(j, sinusoid_value(a, f, phi, K, i, sample_time(base, dt, joff + j0 + j)));
}

// KMAX (1..4): the largest term count given its own chains; a kernel's
// registers follow the largest variant it contains.  Sample j of the run is
// written at out(j) and taken at the time of sample joff + j0 + j (joff: the
// index of the buffer's first sample on the whole horizon).
template <int L, int KMAX, class Out>
__device__ __forceinline__ void sinusoid_run(const double* a, const double* f, const double* phi, int K, int i,
                                             double base, double dt, long j0, long count, const Out& out,
                                             long joff = 0)
{
    const long rest = count - j0;
    const int n = rest < L ? (int)rest : L;
    if (K == 1) {
        sinusoid_run_terms<L, 1>(a, f, phi, i, base, dt, j0, n, out, joff);
    } else if (KMAX >= 2 && K == 2) {
        sinusoid_run_terms<L, (KMAX >= 2 ? 2 : 1)>(a, f, phi, i, base, dt, j0, n, out, joff);
    } else if (KMAX >= 3 && K == 3) {
        sinusoid_run_terms<L, (KMAX >= 3 ? 3 : 1)>(a, f, phi, i, base, dt, j0, n, out, joff);
    } else if (KMAX >= 4 && K == 4) {
        sinusoid_run_terms<L, (KMAX >= 4 ? 4 : 1)>(a, f, phi, i, base, dt, j0, n, out, joff);
    } else {
        for (int j = 0; j < n; ++j) out(j, sinusoid_value(a, f, phi, K, i, sample_time(base, dt, joff + j0 + j)));
    }
}

// The sampling kernels' KMAX for inputs of up to max_terms terms per channel.
inline int sample_kmax(int max_terms) { return max_terms < 1 ? 1 : (max_terms > 4 ? 4 : max_terms); }

}  // namespace parode
