// inputs.cpp -- input-function registry: NVRTC-compiled user functions and
// the built-in sum-of-sinusoids input (see inputs.h).
#include "inputs.h"

#include "common.h"
#include "kernels.h"

#include <nvrtc.h>

#include <cstring>

namespace parode {

namespace {

// Kernel wrapped around the user's UFunc: the same role as the reference's
// Kernels/u.cl:6-11 (one value per (sample, input)), with the sample time
// formed in FP64 before the conversion to fType.
const char* kUKernelTail = R"(
extern "C" __global__ void parode_u_samples(double* U, int m, double base, double dt, long long count,
                                            long long joff)
{
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count * (long long)m) return;
    long long j = e / m;
    int i = (int)(e - j * m);
    double t = __dadd_rn(base, __dmul_rn(dt, (double)(joff + j)));
    U[e] = (double)UFunc((fType)t, i);
}
)";

std::string nvrtc_log(nvrtcProgram prog)
{
    size_t n = 0;
    nvrtcGetProgramLogSize(prog, &n);
    std::string log(n, '\0');
    if (n) nvrtcGetProgramLog(prog, &log[0]);
    return log;
}

}  // namespace

InputRegistry::~InputRegistry() { clear(); }

void InputRegistry::clear()
{
    for (auto& e : entries_) {
        for (int v = 0; v < 2; ++v)
            if (e->lib[v]) cudaLibraryUnload(e->lib[v]);
        for (double* p : e->dparams)
            if (p) cudaFree(p);
    }
    entries_.clear();
}

void InputRegistry::compile(InputEntry* e, int variant)
{
    std::string src = variant ? "typedef double fType;\n" : "typedef float fType;\n";
    src += "#line 1 \"UFunc\"\n";
    src += e->source;
    src += "\n";
    src += kUKernelTail;
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "parode_input.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
        throw Error(kCouldNotCreateGPUKernels, "nvrtcCreateProgram failed");
    const char* opts[] = {"--gpu-architecture=sm_100a", "-default-device", "-std=c++17"};
    nvrtcResult r = nvrtcCompileProgram(prog, 3, opts);
    if (r != NVRTC_SUCCESS) {
        std::string log = nvrtc_log(prog);
        nvrtcDestroyProgram(&prog);
        throw Error(kCouldNotCreateGPUKernels, "input function does not compile:\n" + log);
    }
    size_t n = 0;
    nvrtcGetCUBINSize(prog, &n);
    std::vector<char> cubin(n);
    nvrtcGetCUBIN(prog, cubin.data());
    nvrtcDestroyProgram(&prog);
    cudaLibrary_t lib = nullptr;
    PARODE_CUDA(cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
    cudaKernel_t k = nullptr;
    cudaError_t ge = cudaLibraryGetKernel(&k, lib, "parode_u_samples");
    if (ge != cudaSuccess) {
        cudaLibraryUnload(lib);
        throw Error(kCouldNotCreateGPUKernels, "input kernel missing after compilation");
    }
    e->lib[variant] = lib;
    e->kern[variant] = k;
}

int InputRegistry::add_user(const std::string& source)
{
    auto e = std::make_unique<InputEntry>();
    e->kind = InputEntry::kUser;
    e->source = source;
    compile(e.get(), 0);
    entries_.push_back(std::move(e));
    return (int)entries_.size() - 1;
}

int InputRegistry::add_sinusoid(int m, int K, const double* a, const double* f, const double* phi)
{
    if (m <= 0 || K <= 0 || !a || !f || !phi) throw Error(kInvalidArgument, "bad sinusoid input description");
    auto e = std::make_unique<InputEntry>();
    e->kind = InputEntry::kSinusoid;
    e->m = m;
    e->K = K;
    e->a.assign(a, a + (long)m * K);
    e->f.assign(f, f + (long)m * K);
    e->phi.assign(phi, phi + (long)m * K);
    entries_.push_back(std::move(e));
    return (int)entries_.size() - 1;
}

const double* InputRegistry::sinusoid_device(InputEntry* e, int device)
{
    if ((int)e->dparams.size() <= device) e->dparams.resize(device + 1, nullptr);
    if (!e->dparams[device]) {
        long q = (long)e->m * e->K;
        double* d = nullptr;
        PARODE_CUDA(cudaMalloc(&d, sizeof(double) * 3 * q));
        std::vector<double> h(3 * q);
        std::memcpy(h.data(), e->a.data(), sizeof(double) * q);
        std::memcpy(h.data() + q, e->f.data(), sizeof(double) * q);
        std::memcpy(h.data() + 2 * q, e->phi.data(), sizeof(double) * q);
        PARODE_CUDA(cudaMemcpy(d, h.data(), sizeof(double) * 3 * q, cudaMemcpyHostToDevice));
        e->dparams[device] = d;
    }
    return e->dparams[device];
}

InputEntry* InputRegistry::get(int idx)
{
    if (idx < 0 || idx >= (int)entries_.size()) return nullptr;
    return entries_[idx].get();
}

void InputRegistry::fill(InputEntry* e, int device, double* U, int m, double base, double dt, long count,
                         bool double_type, cudaStream_t s, long joff)
{
    if (m <= 0 || count <= 0) return;
    if (e->kind == InputEntry::kSinusoid) {
        if (e->m < m) throw Error(kInvalidInput, "sinusoid input has fewer channels than the system");
        long q = (long)e->m * e->K;
        const double* d = sinusoid_device(e, device);
        // the kernel indexes parameters as i*K + k for i < m, so a sinusoid
        // input wider than the system is read from its first m channels
        launch_sinusoid_samples(U, m, e->K, d, d + q, d + 2 * q, base, dt, count, s, joff);
        return;
    }
    int v = double_type ? 1 : 0;
    if (!e->kern[v]) compile(e, v);
    long long cnt = count, off = joff;
    void* args[] = {&U, &m, &base, &dt, &cnt, &off};
    long total = count * m;
    unsigned grid = (unsigned)((total + 255) / 256);
    PARODE_CUDA(cudaLaunchKernel((const void*)e->kern[v], dim3(grid), dim3(256), args, 0, s));
}

void InputRegistry::fill_planes(InputEntry* e, int device, float* hi, float* lo, double* scratch, int m, double base,
                                double dt, long count, bool double_type, cudaStream_t s, long joff)
{
    if (m <= 0 || count <= 0) return;
    if (e->kind == InputEntry::kSinusoid) {
        if (e->m < m) throw Error(kInvalidInput, "sinusoid input has fewer channels than the system");
        const long q = (long)e->m * e->K;
        const double* d = sinusoid_device(e, device);
        launch_sinusoid_planes(hi, lo, m, e->K, d, d + q, d + 2 * q, base, dt, count, s, joff);
        return;
    }
    if (!scratch) throw Error(kInvalidArgument, "a user input function needs FP64 scratch for its samples");
    fill(e, device, scratch, m, base, dt, count, double_type, s, joff);
    launch_split_planes(scratch, hi, lo, count * m, s);
}

}  // namespace parode
