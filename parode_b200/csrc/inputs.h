// inputs.h -- registry of input functions u(t) (the reference's u-kernels).
//
// The reference compiles the user's `fType UFunc(fType t, int nInputIndex)`
// into an OpenCL kernel per device at RegisterInput time
// (Sources/ParODE.cpp:410-466, Kernels/u.cl:6-11).  Here a user function is
// compiled with NVRTC into a CUDA kernel that fills the input-sample buffer;
// the built-in sum-of-sinusoids input needs no compilation.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace parode {

struct InputEntry {
    enum Kind { kUser, kSinusoid } kind = kUser;
    // user function
    std::string source;
    cudaLibrary_t lib[2] = {nullptr, nullptr};  // [0] fType = float, [1] fType = double
    cudaKernel_t kern[2] = {nullptr, nullptr};
    // sinusoids
    int m = 0, K = 0;
    std::vector<double> a, f, phi;
    std::vector<double*> dparams;  // per device: a | f | phi, 3*m*K doubles
};

class InputRegistry {
public:
    ~InputRegistry();
    // Compiles (for fType = float, the reference's ABI type) and registers a
    // user function; returns its index.  Throws Error on a compile failure.
    int add_user(const std::string& source);
    int add_sinusoid(int m, int K, const double* a, const double* f, const double* phi);
    InputEntry* get(int idx);
    void clear();
    int size() const { return (int)entries_.size(); }

    // U[j*m + i] = u_i(base + dt*(joff + j)) for j < count, i < m, enqueued
    // on `s` (joff: the first sample's index on the whole horizon, for a time
    // shard).  `double_type` selects the fType = double variant of a user
    // function.
    void fill(InputEntry* e, int device, double* U, int m, double base, double dt, long count, bool double_type,
              cudaStream_t s, long joff = 0);
    // The same samples as TF32 hi / lo planes (hi[j*m + i], lo[j*m + i]; lo
    // may be null): the sinusoid input writes them directly; a user function
    // fills `scratch` (count*m doubles) first.
    void fill_planes(InputEntry* e, int device, float* hi, float* lo, double* scratch, int m, double base,
                     double dt, long count, bool double_type, cudaStream_t s, long joff = 0);
    // Device copy of a sinusoid input's parameters: a | f | phi, m*K each.
    const double* sinusoid_device(InputEntry* e, int device);

private:
    void compile(InputEntry* e, int variant);
    std::vector<std::unique_ptr<InputEntry>> entries_;
};

}  // namespace parode
