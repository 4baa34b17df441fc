// general.cpp -- host driver of the general affine scan (general.h).
//
// The reference's scan driver (Sources/GPUFixedStepIterative.cpp:236-398)
// with its matrix products kept: a level-synchronous up-sweep that composes
// the pairs of each level (matrices and vectors), then a down-sweep that
// passes the prefixes down through the left subtrees' compositions, in place.
// Pairs whose span starts past the last map are skipped (the padding up to
// the next power of two is never read for an output).
#include "general.h"

#include "common.h"
#include "kernels.h"

#include <algorithm>

namespace parode {

void general_scan(const double* M, const double* V, const double* x0, int ns, long count, int precision,
                  double* X, int* status, cudaStream_t s)
{
    if (!M || !X) throw Error(kInvalidArgument, "general scan: M and X must be device pointers");
    if (ns < 1 || ns > 64) throw Error(kInvalidArgument, "general scan: scan dimension must be in [1, 64]");
    if (count < 1) throw Error(kInvalidArgument, "general scan: count must be >= 1");
    if (precision != kFP64 && precision != kMixed) throw Error(kInvalidArgument, "unknown precision");
    int dev = 0, sms = 148;
    PARODE_CUDA(cudaGetDevice(&dev));
    PARODE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int NP = general_padded_dim(ns);
    const long Tp = next_pow2(count);
    double* buf = nullptr;
    if (fault_alloc_now()) throw Error(kNotEnoughResources, "general scan: device allocation failed (injected)");
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&buf), general_scan_bytes(ns, count), s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(kNotEnoughResources, "general scan: device allocation failed");
    }
    double* Mp = buf;
    double* Vp = Mp + Tp * (long)NP * NP;  // slot -1
    double* V1 = Vp + NP;                  // slot 0
    try {
        launch_general_in(Mp, Vp, M, V, x0, ns, NP, count, Tp, sms, s);
        const int levels = ilog2(Tp);
        for (int l = 0; l < levels; ++l) {
            const long d = 1L << l;
            // mixed form: the top four levels compose in FP64, as the mixed
            // level-synchronous scan keeps its high powers (few pairs, and
            // their products carry the whole horizon)
            const int prec = l < levels - 4 ? precision : (int)kFP64;
            launch_compose(NP, prec, Mp, V1, d, sweep_columns(count, Tp, d), sms, status, s);
        }
        for (int l = levels - 1; l >= 0; --l) {
            const long d = 1L << l;
            launch_down_general(NP, Mp, V1, d, sweep_columns(count, Tp, d), sms, s);
        }
        launch_general_out(X, Vp, ns, NP, count, sms, s);
    } catch (...) {
        cudaFreeAsync(buf, s);
        throw;
    }
    PARODE_CUDA(cudaFreeAsync(buf, s));
}

}  // namespace parode
