// general.h -- the general affine scan over per-step maps (kernels_general.cu,
// kernels_general_tc.cu, general.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace parode {

// Padded scan dimension of the general scan (8, 16, 32 or 64).
int general_padded_dim(int ns);
// Device bytes of its scan buffers for `count` maps.
size_t general_scan_bytes(int ns, long count);

// Caller arrays into / out of the padded in-place layout (general.h).
void launch_general_in(double* Mp, double* Vp, const double* M, const double* V, const double* x0, int ns, int NP,
                       long count, long Tp, int sms, cudaStream_t s);
void launch_general_out(double* X, const double* Vp, int ns, int NP, long count, int sms, cudaStream_t s);
// Ms[k] = Phi (NP x NP) for k < count.
void launch_distribute(double* Ms, const double* Phi, int NP, long count, int sms, cudaStream_t s);

// Up-sweep level with distance d over npairs pairs: V1[k] += M[k] V1[k-d],
// M[k] <- M[k] M[k-d] for k = q 2d + 2d - 1 (V1 = slot 0).  precision kMixed
// runs the products on tcgen05 (3xTF32) where compose_tc_supported(NP).
void launch_compose(int NP, int precision, double* M, double* V1, long d, long npairs, int sms, int* status,
                    cudaStream_t s);
bool compose_tc_supported(int NP);
void launch_compose_tc(int NP, double* M, double* V1, long d, long npairs, int sms, int* status, cudaStream_t s);
// Down-sweep level: V1[L] += M[L] V1[p], L = q 2d + d - 1, p = q 2d - 1.
void launch_down_general(int NP, const double* M, double* V1, long d, long npairs, int sms, cudaStream_t s);

// The whole scan on device data: x_0 = x0 (nullptr: 0), x_{k+1} = M_k x_k +
// V_k (V nullptr: 0), X[k] = x_k for k < count; M count x ns x ns, V and X
// count x ns, row-major FP64.  Scratch from the stream-ordered pool; returns
// after enqueueing (status: device word the tensor-core kernel sets on a
// time-out, nullptr for the FP64 form).
void general_scan(const double* M, const double* V, const double* x0, int ns, long count, int precision,
                  double* X, int* status, cudaStream_t s);

}  // namespace parode
