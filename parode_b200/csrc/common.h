// common.h -- shared definitions of the ParODE B200 library (host and device).
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

namespace parode {

// Error codes: ParODEEnums.h (-1..-7) and parode_ext.h (-8..-10).
enum Err : int {
    kOK = 0,
    kNoGPU = -1,
    kNotInitialized = -2,
    kCouldNotCreateGPUKernels = -3,
    kNotEnoughResources = -4,
    kInvalidDeviceId = -5,
    kInvalidSystem = -6,
    kInvalidSolverType = -7,
    kInvalidInput = -8,
    kInvalidArgument = -9,
    kDeviceError = -10,
};

// Exception carrying an API error code; never crosses the C ABI.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

#define PARODE_CUDA(call)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            if (e_ == cudaErrorMemoryAllocation)                                                   \
                throw ::parode::Error(::parode::kNotEnoughResources,                               \
                                      std::string(#call ": ") + cudaGetErrorString(e_));           \
            throw ::parode::Error(::parode::kDeviceError, std::string(#call ": ") + cudaGetErrorString(e_)); \
        }                                                                                          \
    } while (0)

// Host-side fault injection for tests (PARODE_OPT_FAULT_ALLOC): true when the
// device allocation being made now is the one set to fail.  Every allocation
// site of the solve paths asks before allocating.
bool fault_alloc_now();

enum Solver : int { kRK4 = 0, kABM = 1 };
// kTF32: the single-pass form of the mixed response GEMMs (hi*hi only); the
// other tensor-core stages run their 3xTF32 form under it.
enum Precision : int { kFP64 = 0, kMixed = 1, kTF32 = 2 };

inline long round_up(long v, long q) { return (v + q - 1) / q * q; }
inline long next_pow2(long v)
{
    long p = 1;
    while (p < v) p <<= 1;
    return p;
}
inline int ilog2(long v)
{
    int l = 0;
    while ((1L << l) < v) ++l;
    return l;
}

}  // namespace parode
