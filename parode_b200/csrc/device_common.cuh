// device_common.cuh -- device helpers shared by the scan kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace parode {

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

// Sample time t_j = base + dt * j, rounded as the host computes it.
__device__ __forceinline__ double sample_time(double base, double dt, long j)
{
    return __dadd_rn(base, __dmul_rn(dt, (double)j));
}

}  // namespace parode
