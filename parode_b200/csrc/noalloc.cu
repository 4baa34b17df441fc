// noalloc.cu -- the affine scan over caller device buffers, with no allocation.
//
// ParODE_AffineScanDevice runs the device carry scan of the blocked path
// (power-table squaring, then the FP64 items up / top / down hierarchy) on a
// caller's Phi, Gamma and x0 without allocating anything: its scratch is one
// file-scope __device__ array, so no cudaMalloc / cudaFree (and no allocating
// library routine) runs on any call.  It serves callers that cannot allocate:
//  - a caller that has reserved the whole device for its own pool (an
//    allocation would fail or evict its working set),
//  - a caller issuing work on a stream while other streams run, where a
//    cudaMalloc / cudaFree would synchronise the device and stall them,
//  - a fixed-memory, fixed-latency loop that must not hit the allocator.
//
// Set-up, once per device with that device current: look up the scratch
// array's device address with cudaGetSymbolAddress, check the return code and
// cache the pointer; and load every kernel the entry point launches.  With
// the CUDA runtime's lazy module loading (the default since CUDA 12.2) that
// set-up is what loads the array's module and maps its device memory, and a
// kernel's module is otherwise loaded at its first launch.  InitializeAllGPUs
// and InitializeSelectedGPUs run the set-up for every device they select; a
// caller that skips them gets it on its first call on a device.  Either must
// come before the caller reserves the device's memory for itself, and before
// any stream capture is started on the device.  The cached pointer belongs to
// the device's primary context: after cudaDeviceReset, or under another
// context made current by the caller, the address is stale.
//
// The scratch is shared by all calls on a device: calls whose work overlaps
// on the GPU (two streams, or two host threads with no ordering between them)
// race on it.  Issue the calls on one stream, or order them with events.
//
// Nothing in the scratch has to start at zero: every word a call reads is
// written earlier by the same call (the padding of Phi, Gamma and x0 is
// written as zeros by the padding kernel).
#include "blocked.h"
#include "common.h"
#include "parode_ext.h"

#include <algorithm>
#include <cstdio>
#include <mutex>

namespace parode {
namespace {

// 16 MiB of FP64 scratch per device.  A call with scan dimension ns
// (NP = the power of two >= max(8, ns)) and `count` items needs
//   levels * NP^2 + NP + count * NP + items_scratch(count) * NP
// doubles (levels ~ log2(count) + 1; items_scratch ~ count / (B - 1)), e.g.
// count <= 29,000 at ns = 64 and count <= 230,000 at ns = 8.
constexpr long kScratchDoubles = 2L << 20;
__device__ __align__(256) double g_scan_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};

constexpr int kPadThreads = 256;

// dst (rows x NP, row-major) <- src (rows x ns) with zero columns ns..NP-1;
// src == nullptr writes zeros.
__global__ void k_pad_rows(double* dst, const double* src, long rows, int ns, int NP)
{
    const long total = rows * NP;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long r = e / NP;
        const int k = (int)(e - r * NP);
        dst[e] = (src != nullptr && k < ns) ? src[r * ns + k] : 0.0;
    }
}

// Phi (ns x ns) into the NP x NP level-0 table entry, zero elsewhere.
__global__ void k_pad_matrix(double* dst, const double* src, int ns, int NP)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < NP * NP; e += gridDim.x * blockDim.x) {
        const int r = e / NP, k = e - r * NP;
        dst[e] = (r < ns && k < ns) ? src[r * ns + k] : 0.0;
    }
}

// dst (rows x ns) <- the first ns columns of src (rows x NP).
__global__ void k_unpad_rows(double* dst, const double* src, long rows, int ns, int NP)
{
    const long total = rows * ns;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long r = e / ns;
        const int k = (int)(e - r * ns);
        dst[e] = src[r * NP + k];
    }
}

unsigned grid_for(long work, int sms)
{
    return (unsigned)std::max<long>(1, std::min<long>((work + kPadThreads - 1) / kPadThreads, 8L * sms));
}

// Per-device set-up (see the file comment); idempotent.  Caller holds g_mu.
void setup_device_locked(int dev)
{
    if (g_scratch_ptr[dev] != nullptr) return;
    void* p = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&p, g_scan_scratch);
    if (rc != cudaSuccess || p == nullptr) {
        cudaGetLastError();
        throw Error(kDeviceError, std::string("cudaGetSymbolAddress(scan scratch): ") + cudaGetErrorString(rc));
    }
    cudaFuncAttributes fa;
    PARODE_CUDA(cudaFuncGetAttributes(&fa, k_pad_rows));
    PARODE_CUDA(cudaFuncGetAttributes(&fa, k_pad_matrix));
    PARODE_CUDA(cudaFuncGetAttributes(&fa, k_unpad_rows));
    preload_blocked_carry_kernels();
    int n = 0;
    PARODE_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    g_sms[dev] = n;
    g_scratch_ptr[dev] = static_cast<double*>(p);
}

// Scratch pointer and SM count of the current device (set-up on first use).
double* scratch_for_current_device(int* sms)
{
    int dev = -1;
    PARODE_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(kInvalidDeviceId, "device id out of range");
    std::lock_guard<std::mutex> g(g_mu);
    setup_device_locked(dev);
    *sms = g_sms[dev];
    return g_scratch_ptr[dev];
}

// Levels of the power table the carry hierarchy reads for `count` items
// starting at level 0 (as the blocked solve sizes it).
int carry_levels(const BlockedShape& sh, long count)
{
    long c = count;
    int lev = 0;
    while (c > sh.S_items) {
        c = (c + sh.B - 1) / sh.B;
        lev += sh.R;
    }
    return std::max(lev + ilog2(next_pow2(c)), sh.R);
}

void affine_scan_device(const double* dPhi, const double* dGamma, const double* dX0, int ns, long count,
                        double* dX, cudaStream_t s)
{
    if (dPhi == nullptr || dX == nullptr) throw Error(kInvalidArgument, "Phi and X must be device pointers");
    if (ns < 1 || ns > 64) throw Error(kInvalidArgument, "scan dimension must be in [1, 64]");
    if (count < 1) throw Error(kInvalidArgument, "count must be >= 1");
    BlockedShape sh;
    if (!blocked_shape(ns, 1, 0, &sh)) throw Error(kInvalidArgument, "scan dimension not supported");
    const long NP = sh.NP;
    const int levels = carry_levels(sh, count);
    const long need = (long)levels * NP * NP + NP + count * NP + blocked_items_scratch(sh, count) * NP;
    if (need > kScratchDoubles) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "affine scan needs %ld scratch doubles; the static scratch holds %ld", need,
                      kScratchDoubles);
        throw Error(kNotEnoughResources, msg);
    }
    int sms = 0;
    double* base = scratch_for_current_device(&sms);
    double* P = base;
    double* X0 = P + (long)levels * NP * NP;
    double* items = X0 + NP;
    double* work = items + count * NP;

    k_pad_matrix<<<grid_for(NP * NP, sms), kPadThreads, 0, s>>>(P, dPhi, ns, (int)NP);
    PARODE_CUDA(cudaGetLastError());
    k_pad_rows<<<1, kPadThreads, 0, s>>>(X0, dX0, 1, ns, (int)NP);
    PARODE_CUDA(cudaGetLastError());
    k_pad_rows<<<grid_for(count * NP, sms), kPadThreads, 0, s>>>(items, dGamma, count, ns, (int)NP);
    PARODE_CUDA(cudaGetLastError());
    if (levels > 1) launch_blocked_tables(sh, P, 1, levels, nullptr, nullptr, 0, s);
    launch_blocked_carry(sh, items, count, 0, P, X0, work, sms, s);
    k_unpad_rows<<<grid_for(count * ns, sms), kPadThreads, 0, s>>>(dX, items, count, ns, (int)NP);
    PARODE_CUDA(cudaGetLastError());
}

}  // namespace

void noalloc_setup_device(int dev)
{
    if (dev < 0 || dev >= kMaxDevices) throw Error(kInvalidDeviceId, "device id out of range");
    int prev = -1;
    PARODE_CUDA(cudaGetDevice(&prev));
    PARODE_CUDA(cudaSetDevice(dev));
    try {
        std::lock_guard<std::mutex> g(g_mu);
        setup_device_locked(dev);
    } catch (...) {
        cudaSetDevice(prev);
        throw;
    }
    PARODE_CUDA(cudaSetDevice(prev));
}

}  // namespace parode

extern "C" void ParODE_AffineScanDevice(const double* dPhi, const double* dGamma, const double* dX0, int ns,
                                        long long count, double* dX, void* stream, int nErr[])
{
    int rc = parode::kOK;
    try {
        parode::affine_scan_device(dPhi, dGamma, dX0, ns, (long)count, dX, static_cast<cudaStream_t>(stream));
    } catch (const parode::Error& e) {
        std::fprintf(stderr, "ParODE_AffineScanDevice: %s\n", e.what());
        rc = e.code;
    } catch (...) {
        rc = parode::kDeviceError;
    }
    if (nErr) nErr[0] = rc;
}
