// api.cpp -- the exported C ABI of libParODEShared.so and its library state.
//
// Mirrors the reference's extern "C" layer and ParODE singleton
// (Sources/ParODE.cpp:23-174 and :244-572): initialisation states
// NOT / PARTIAL / FULL, the input registry, error codes in nErr[0], no
// exception crossing the ABI.  Differences, all additive: a mutex serialises
// calls; invalid device ids and input indices are reported instead of being
// undefined behaviour; GetErrorDescription knows every code.
#include "common.h"
#include "host_math.h"
#include "inputs.h"
#include "solver.h"
#include "batch.h"
#include "blocked.h"
#include "general.h"
#include "tuner.h"
#include "server.h"

#include "FTypeDef.h"
#include "ParODECInterface.h"
#include "parode_ext.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

using namespace parode;

namespace {
// PARODE_OPT_FAULT_ALLOC: allocations left before the injected failure (-1: none)
std::atomic<long long> g_fault_alloc{-1};
}  // namespace

bool parode::fault_alloc_now()
{
    long long v = g_fault_alloc.load();
    while (v >= 0) {
        if (g_fault_alloc.compare_exchange_weak(v, v - 1)) return v == 0;
    }
    return false;
}

namespace {

enum InitState { kNot = 0, kPartial = 1, kFull = 2 };

struct Library {
    std::recursive_mutex mu;
    InitState state = kNot;
    std::vector<int> available;  // device ordinals of compute capability 10.x
    std::vector<int> selected;
    InputRegistry inputs;
    int precision = kFP64;
    int path = kPathAuto;
    int log = 0;
    long long executions = 1;  // PARODE_OPT_EXECUTIONS: plans and batches
    int fault_withhold = 0;    // PARODE_OPT_FAULT_WITHHOLD (test hook)
    long long pool_keep = 0;   // PARODE_OPT_POOL_KEEP: last value set (the driver's default pool keeps 0)
    int discretise = 0;        // PARODE_OPT_DISCRETISE (batches and servers)
    std::vector<int> tune_inputs;  // sinusoid inputs of the tuner's synthetic systems, by input count
    cudaEvent_t t_start = nullptr, t_stop = nullptr;
    bool timer_running = false;

    void clean()
    {
        if (!selected.empty()) {
            cudaSetDevice(selected[0]);
            cudaDeviceSynchronize();
        }
        inputs.clear();
        if (t_start) cudaEventDestroy(t_start);
        if (t_stop) cudaEventDestroy(t_stop);
        t_start = t_stop = nullptr;
        timer_running = false;
        selected.clear();
        available.clear();
        state = kNot;
    }

    void enumerate()
    {
        available.clear();
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess) {
            cudaGetLastError();
            count = 0;
        }
        for (int d = 0; d < count; ++d) {
            cudaDeviceProp prop;
            if (cudaGetDeviceProperties(&prop, d) != cudaSuccess) continue;
            if (prop.major == 10) available.push_back(d);  // kernels are built for sm_100a only
        }
    }

    int init_devices(const std::vector<int>& ids)
    {
        for (int d : ids) {
            if (cudaSetDevice(d) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) {
                cudaGetLastError();
                return kCouldNotCreateGPUKernels;
            }
            // the allocation-free entry point's scratch and kernels are
            // loaded now, while the device still has memory to map them
            try {
                noalloc_setup_device(d);
            } catch (const Error&) {
                return kCouldNotCreateGPUKernels;
            }
        }
        selected = ids;
        cudaSetDevice(selected[0]);
        // measured block lengths of an earlier tuning run on this kind of GPU
        if (const char* tf = std::getenv("PARODE_TUNE_FILE")) {
            int e = 0;
            ParODE_TuneLoad(tf, nullptr, &e);
        }
        if (cudaEventCreate(&t_start) != cudaSuccess || cudaEventCreate(&t_stop) != cudaSuccess) {
            cudaGetLastError();
            return kNotEnoughResources;
        }
        state = kFull;
        return kOK;
    }
};

Library& lib()
{
    static Library* L = new Library();  // never destroyed: CUDA may be torn down first at exit
    return *L;
}

const char* describe(int code)
{
    switch (code) {
    case kOK: return "No Error";
    case kNoGPU: return "Sorry, no GPU available. Please make sure that a CUDA device of compute capability 10.x (B200) and its driver are installed.";
    case kNotInitialized: return "ParODE not initialized. Please call InitializeAllGPUs or InitializeSelectedGPUs.";
    case kCouldNotCreateGPUKernels: return "Could not create GPU kernels; the device could not be initialised or the input function does not compile.";
    case kNotEnoughResources: return "Not enough resources: a device allocation or transfer failed.";
    case kInvalidDeviceId: return "Invalid device id.";
    case kInvalidSystem: return "Invalid system: empty state, inconsistent matrix sizes or an empty time horizon.";
    case kInvalidSolverType: return "Invalid solver type (0 = Runge-Kutta 4, 1 = Adams-Bashforth-Moulton).";
    case kInvalidInput: return "Invalid input index: register the input function first.";
    case kInvalidArgument: return "Invalid argument.";
    case kDeviceError: return "A CUDA call failed.";
    default: return "Unknown Error";
    }
}

// Builds a SystemDesc from caller arrays.  `T` is float (C ABI) or double.
template <class T>
SystemDesc make_system(const T* A, const T* B, const T* C, const T* D, int nInputs, int nStates, int nOutputs,
                       int ZeroB, int ZeroC, int ZeroD, const T* x0)
{
    SystemDesc s;
    if (nStates <= 0 || !A || !x0) throw Error(kInvalidSystem, "the system has no states");
    s.n = nStates;
    s.m = nInputs > 0 ? nInputs : 0;
    s.p = nOutputs > 0 ? nOutputs : 0;
    s.zeroB = ZeroB == 1 || s.m == 0;
    s.zeroC = ZeroC == 1;
    s.zeroD = ZeroD == 1 || s.m == 0;
    if ((!s.zeroB && !B) || (!s.zeroC && (!C || s.p == 0)) || (!s.zeroD && (!D || s.p == 0)))
        throw Error(kInvalidSystem, "a matrix flagged present is missing");
    s.A.assign(A, A + (size_t)s.n * s.n);
    if (!s.zeroB) s.B.assign(B, B + (size_t)s.n * s.m);
    if (!s.zeroC) s.C.assign(C, C + (size_t)s.p * s.n);
    if (!s.zeroD) s.D.assign(D, D + (size_t)s.p * s.m);
    s.x0.assign(x0, x0 + s.n);
    return s;
}

int current_device_locked(Library& L)
{
    if (L.state != kFull || L.selected.empty()) throw Error(kNotInitialized, "ParODE not initialized");
    return L.selected[0];
}

template <class F>
int guarded(F&& f)
{
    try {
        f();
        return kOK;
    } catch (const Error& e) {
        if (lib().log) std::fprintf(stderr, "ParODE: %s\n", e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        return kNotEnoughResources;
    } catch (...) {
        return kDeviceError;
    }
}

// A host thread that is joined on every exit path (including exceptions).
class HelperThread {
public:
    template <class F>
    void run(F&& f) { t_ = std::thread(std::forward<F>(f)); }
    void join()
    {
        if (t_.joinable()) t_.join();
    }
    ~HelperThread() { join(); }

private:
    std::thread t_;
};

}  // namespace

extern "C" {

void GetErrorDescription(int* ErrNo, char strErrDescription[])
{
    if (!strErrDescription) return;
    const char* d = describe(ErrNo ? *ErrNo : 1);
    std::snprintf(strErrDescription, 256, "%s", d);
}

void InitializeAllGPUs(char* pszKernelFolder, char* pszIncludeFolder, int nErr[])
{
    (void)pszKernelFolder;
    (void)pszIncludeFolder;
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    int rc = guarded([&] {
        L.clean();
        L.enumerate();
        if (L.available.empty()) throw Error(kNoGPU, "no compute capability 10.x device");
        int r = L.init_devices(L.available);
        if (r != kOK) {
            L.clean();
            throw Error(r, "device initialisation failed");
        }
    });
    if (nErr) nErr[0] = rc;
}

void GetAvailableGPUs(int nGPUs[], int GPUIds[], int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    int rc = guarded([&] {
        L.clean();
        L.enumerate();
        L.state = kPartial;
    });
    int n = rc == kOK ? (int)L.available.size() : 0;
    if (nGPUs) nGPUs[0] = n;
    if (GPUIds)
        for (int i = 0; i < n; ++i) GPUIds[i] = L.available[i];
    if (nErr) nErr[0] = rc;
}

void GetDeviceName(int* DeviceId, char strDeviceName[], int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    int rc = kOK;
    if (strDeviceName) strDeviceName[0] = 0;
    if (L.state == kNot) {
        rc = kNotInitialized;
    } else {
        int id = DeviceId ? *DeviceId : -1;
        bool known = false;
        for (int d : L.available) known = known || d == id;
        cudaDeviceProp prop;
        if (!known || cudaGetDeviceProperties(&prop, id) != cudaSuccess) {
            cudaGetLastError();
            rc = kInvalidDeviceId;
        } else if (strDeviceName) {
            std::snprintf(strDeviceName, 256, "%s", prop.name);
        }
    }
    if (nErr) nErr[0] = rc;
}

void InitializeSelectedGPUs(int* nGPUs, int GPUIds[], char* pszKernelFolder, char* pszIncludeFolder, int nErr[])
{
    (void)pszKernelFolder;
    (void)pszIncludeFolder;
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    int rc = guarded([&] {
        if (L.state != kPartial) throw Error(kNotInitialized, "call GetAvailableGPUs first");
        int n = nGPUs ? *nGPUs : 0;
        if (n <= 0 || !GPUIds) throw Error(kNoGPU, "no device selected");
        std::vector<int> ids;
        for (int i = 0; i < n; ++i) {
            bool known = false;
            for (int d : L.available) known = known || d == GPUIds[i];
            if (!known) throw Error(kInvalidDeviceId, "device id not in GetAvailableGPUs");
            ids.push_back(GPUIds[i]);
        }
        int r = L.init_devices(ids);
        if (r != kOK) {
            L.clean();
            throw Error(r, "device initialisation failed");
        }
    });
    if (nErr) nErr[0] = rc;
}

void SimulateODE(fType A[], fType B[], fType C[], fType D[], int* nInputs, int* nStates, int* nOutputs, int* ZeroB,
                 int* ZeroC, int* ZeroD, int* uIndex, double* tStart, double* tEnd, double* tStep, fType x0[],
                 int* solver, fType tVect[], fType xVect[], int* nSteps, int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    if (nSteps) nSteps[0] = 0;
    int rc = guarded([&] {
        int dev = current_device_locked(L);
        if (!nInputs || !nStates || !nOutputs || !ZeroB || !ZeroC || !ZeroD || !uIndex || !tStart || !tEnd ||
            !tStep || !solver)
            throw Error(kInvalidArgument, "null argument");
        if (*solver != kRK4 && *solver != kABM) throw Error(kInvalidSolverType, "unknown solver");
        SystemDesc s = make_system<fType>(A, B, C, D, *nInputs, *nStates, *nOutputs, *ZeroB, *ZeroC, *ZeroD, x0);
        PlanOptions opt;
        opt.precision = L.precision;
        opt.path = L.path;
        opt.input_double = false;  // UFunc(fType t, ...) with fType = float, as the reference ABI
        opt.one_shot = true;
        Plan plan(dev, s, &L.inputs, *uIndex, *solver, *tStart, *tEnd, *tStep, opt);
        long T = plan.num_outputs();
        // fType is float: y is rounded on the device and copied straight into
        // xVect range by range while the later ranges are formed, and the time
        // vector is written as float on a helper thread
        static_assert(sizeof(fType) == sizeof(float), "the reference ABI's fType is float");
        HelperThread tv;
        const int sv = *solver;
        const double t0 = *tStart, t1 = *tEnd, h = *tStep;
        float* tOut = reinterpret_cast<float*>(tVect);
        if (tVect) tv.run([tOut, sv, t0, t1, h] { time_vector_f(sv, t0, t1, h, tOut); });
        try {
            plan.solve_to_host(nullptr, reinterpret_cast<float*>(xVect));
        } catch (...) {
            tv.join();
            throw;
        }
        tv.join();
        if (nSteps) nSteps[0] = (int)T;
        if (L.log)
            std::fprintf(stderr, "ParODE: SimulateODE solver=%d n=%d T=%ld path=%d launches=%d\n", *solver, s.n, T,
                         plan.path(), plan.launch_count());
    });
    if (nErr) nErr[0] = rc;
}

void RegisterInput(char uFunc[], int uIndex[], int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    int idx = -1;
    int rc = guarded([&] {
        if (L.state != kFull) throw Error(kNotInitialized, "ParODE not initialized");
        if (!uFunc) throw Error(kCouldNotCreateGPUKernels, "no source");
        cudaSetDevice(L.selected[0]);
        idx = L.inputs.add_user(std::string(uFunc));
    });
    if (uIndex) uIndex[0] = rc == kOK ? idx : rc;
    if (nErr) nErr[0] = rc;
}

void CloseGPUC()
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    L.clean();
}

void StartTimer(int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    int rc = guarded([&] {
        current_device_locked(L);
        cudaSetDevice(L.selected[0]);
        PARODE_CUDA(cudaDeviceSynchronize());
        PARODE_CUDA(cudaEventRecord(L.t_start, 0));
        PARODE_CUDA(cudaEventSynchronize(L.t_start));
        L.timer_running = true;
    });
    if (nErr) nErr[0] = rc;
}

void StopTimer(float fTime[], int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    int rc = guarded([&] {
        current_device_locked(L);
        cudaSetDevice(L.selected[0]);
        PARODE_CUDA(cudaDeviceSynchronize());
        PARODE_CUDA(cudaEventRecord(L.t_stop, 0));
        PARODE_CUDA(cudaEventSynchronize(L.t_stop));
        float ms = 0.f;
        if (L.timer_running) PARODE_CUDA(cudaEventElapsedTime(&ms, L.t_start, L.t_stop));
        if (fTime) fTime[0] = ms;
    });
    if (nErr) nErr[0] = rc;
}

// ---------------------------------------------------------------------------
// extensions (parode_ext.h)
// ---------------------------------------------------------------------------

void ParODE_SetOption(int option, long long value, int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    int rc = kOK;
    switch (option) {
    case PARODE_OPT_PRECISION:
        if (value != PARODE_PRECISION_FP64 && value != PARODE_PRECISION_MIXED && value != PARODE_PRECISION_TF32)
            rc = kInvalidArgument;
        else L.precision = (int)value;
        break;
    case PARODE_OPT_PATH:
        if (value < 0 || value > 5) rc = kInvalidArgument;
        else L.path = (int)value;
        break;
    case PARODE_OPT_LOG: L.log = (int)value; break;
    case PARODE_OPT_EXECUTIONS:
        if (value < 1) rc = kInvalidArgument;
        else L.executions = value;
        break;
    case PARODE_OPT_FAULT_ALLOC:
        if (value < -1) rc = kInvalidArgument;
        else g_fault_alloc.store(value);
        break;
    case PARODE_OPT_FAULT_WITHHOLD: L.fault_withhold = value != 0; break;
    case PARODE_OPT_POOL_KEEP:
        if (value < 0) {
            rc = kInvalidArgument;
        } else if (L.state != kFull || L.selected.empty()) {
            rc = kNotInitialized;
        } else {
            // the release threshold of each selected device's stream-ordered
            // pool, from which plans and batches take their device memory
            uint64_t keep = (uint64_t)value;
            for (int d : L.selected) {
                cudaMemPool_t pool = nullptr;
                if (cudaDeviceGetDefaultMemPool(&pool, d) != cudaSuccess ||
                    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
                    cudaGetLastError();
                    rc = kDeviceError;
                }
            }
            if (rc == kOK) L.pool_keep = value;
        }
        break;
    case PARODE_OPT_DISCRETISE:
        if (value != PARODE_DISCRETISE_AUTO && value != PARODE_DISCRETISE_HOST && value != PARODE_DISCRETISE_DEVICE)
            rc = kInvalidArgument;
        else L.discretise = (int)value;
        break;
    default: rc = kInvalidArgument;
    }
    if (nErr) nErr[0] = rc;
}

long long ParODE_GetOption(int option, int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    if (nErr) nErr[0] = kOK;
    switch (option) {
    case PARODE_OPT_PRECISION: return L.precision;
    case PARODE_OPT_PATH: return L.path;
    case PARODE_OPT_LOG: return L.log;
    case PARODE_OPT_EXECUTIONS: return L.executions;
    case PARODE_OPT_FAULT_ALLOC: return g_fault_alloc.load();
    case PARODE_OPT_FAULT_WITHHOLD: return L.fault_withhold;
    case PARODE_OPT_POOL_KEEP: return L.pool_keep;
    case PARODE_OPT_DISCRETISE: return L.discretise;
    default:
        if (nErr) nErr[0] = kInvalidArgument;
        return -1;
    }
}

long long ParODE_NumOutputs(int solver, double tStart, double tEnd, double tStep)
{
    long ns = 0;
    return num_outputs(solver, tStart, tEnd, tStep, &ns);
}

void ParODE_RegisterSinusoidInput(int nInputs, int nTerms, const double* amp, const double* freq,
                                  const double* phase, int uIndex[], int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    int idx = -1;
    int rc = guarded([&] {
        if (L.state != kFull) throw Error(kNotInitialized, "ParODE not initialized");
        idx = L.inputs.add_sinusoid(nInputs, nTerms, amp, freq, phase);
    });
    if (uIndex) uIndex[0] = rc == kOK ? idx : rc;
    if (nErr) nErr[0] = rc;
}

void ParODE_SimulateODE_d(const double* A, const double* B, const double* C, const double* D, int nInputs,
                          int nStates, int nOutputs, int ZeroB, int ZeroC, int ZeroD, int uIndex, double tStart,
                          double tEnd, double tStep, const double* x0, int solver, int precision, double* tVect,
                          double* yVect, long long nSteps[], int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    if (nSteps) nSteps[0] = 0;
    int rc = guarded([&] {
        int dev = current_device_locked(L);
        if (precision != PARODE_PRECISION_FP64 && precision != PARODE_PRECISION_MIXED &&
            precision != PARODE_PRECISION_TF32)
            throw Error(kInvalidArgument, "unknown precision");
        SystemDesc s = make_system<double>(A, B, C, D, nInputs, nStates, nOutputs, ZeroB, ZeroC, ZeroD, x0);
        PlanOptions opt;
        opt.precision = precision;
        opt.path = L.path;
        opt.input_double = true;
        opt.fault_withhold = L.fault_withhold;
        opt.log = L.log != 0;
        opt.one_shot = true;
        Plan plan(dev, s, &L.inputs, uIndex, solver, tStart, tEnd, tStep, opt);
        // the host time vector is built on a helper thread while the plan
        // is set up, solved and its outputs copied
        HelperThread tv;
        if (tVect) tv.run([=] { time_vector(solver, tStart, tEnd, tStep, tVect); });
        try {
            plan.solve_to_host(yVect, nullptr);
        } catch (...) {
            tv.join();
            throw;
        }
        tv.join();
        if (nSteps) nSteps[0] = plan.num_outputs();
    });
    if (nErr) nErr[0] = rc;
}

struct ParODE_Plan {
    std::unique_ptr<Plan> plan;
};

ParODE_Plan* ParODE_PlanCreate(const double* A, const double* B, const double* C, const double* D, int nInputs,
                               int nStates, int nOutputs, int ZeroB, int ZeroC, int ZeroD, int uIndex,
                               double tStart, double tEnd, double tStep, const double* x0, int solver, int precision,
                               int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    ParODE_Plan* out = nullptr;
    int rc = guarded([&] {
        int dev = current_device_locked(L);
        if (precision != PARODE_PRECISION_FP64 && precision != PARODE_PRECISION_MIXED &&
            precision != PARODE_PRECISION_TF32)
            throw Error(kInvalidArgument, "unknown precision");
        SystemDesc s = make_system<double>(A, B, C, D, nInputs, nStates, nOutputs, ZeroB, ZeroC, ZeroD, x0);
        PlanOptions opt;
        opt.precision = precision;
        opt.path = L.path;
        opt.input_double = true;
        opt.executions = (double)L.executions;
        opt.fault_withhold = L.fault_withhold;
        opt.log = L.log != 0;
        auto h = std::make_unique<ParODE_Plan>();
        h->plan = std::make_unique<Plan>(dev, s, &L.inputs, uIndex, solver, tStart, tEnd, tStep, opt);
        out = h.release();
    });
    if (nErr) nErr[0] = rc;
    return out;
}

ParODE_Plan* ParODE_PlanCreateShard(const double* A, const double* B, const double* C, const double* D, int nInputs,
                                    int nStates, int nOutputs, int ZeroB, int ZeroC, int ZeroD, int uIndex,
                                    double tStart, double tEnd, double tStep, const double* x0, int solver,
                                    int precision, int shard, int shards, int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    ParODE_Plan* out = nullptr;
    int rc = guarded([&] {
        int dev = current_device_locked(L);
        if (precision != PARODE_PRECISION_FP64 && precision != PARODE_PRECISION_MIXED &&
            precision != PARODE_PRECISION_TF32)
            throw Error(kInvalidArgument, "unknown precision");
        if (shards < 1 || shard < 0 || shard >= shards) throw Error(kInvalidArgument, "shard index out of range");
        SystemDesc s = make_system<double>(A, B, C, D, nInputs, nStates, nOutputs, ZeroB, ZeroC, ZeroD, x0);
        PlanOptions opt;
        opt.precision = precision;
        opt.path = kPathBlockedResponse;  // the partition runs on the block-response leaf
        opt.input_double = true;
        opt.executions = (double)L.executions;
        opt.shard = shard;
        opt.shards = shards;
        auto h = std::make_unique<ParODE_Plan>();
        h->plan = std::make_unique<Plan>(dev, s, &L.inputs, uIndex, solver, tStart, tEnd, tStep, opt);
        out = h.release();
    });
    if (nErr) nErr[0] = rc;
    return out;
}

void ParODE_PlanShardInfo(const ParODE_Plan* plan, long long info[5])
{
    for (int k = 0; k < 5; ++k) info[k] = 0;
    if (plan && plan->plan) plan->plan->shard_info(info);
}

void ParODE_PlanShardUp(ParODE_Plan* plan, double* dTop, void* stream, int nErr[])
{
    int rc = guarded([&] {
        if (!plan || !plan->plan || !dTop) throw Error(kInvalidArgument, "null plan or buffer");
        plan->plan->shard_up(dTop, (cudaStream_t)stream);
    });
    if (nErr) nErr[0] = rc;
}

void ParODE_PlanShardDown(ParODE_Plan* plan, const double* dGathered, double* yDev, void* stream, int nErr[])
{
    int rc = guarded([&] {
        if (!plan || !plan->plan || !dGathered) throw Error(kInvalidArgument, "null plan or buffer");
        plan->plan->shard_down(dGathered, yDev, (cudaStream_t)stream);
    });
    if (nErr) nErr[0] = rc;
}

void ParODE_PlanExecute(ParODE_Plan* plan, double* yDev, void* stream, int nErr[])
{
    int rc = guarded([&] {
        if (!plan || !plan->plan) throw Error(kInvalidArgument, "null plan");
        plan->plan->execute(yDev, (cudaStream_t)stream);
    });
    if (nErr) nErr[0] = rc;
}

void ParODE_PlanGetOutput(ParODE_Plan* plan, double* tVect, double* yVect, int nErr[])
{
    int rc = guarded([&] {
        if (!plan || !plan->plan) throw Error(kInvalidArgument, "null plan");
        plan->plan->get_output(tVect, yVect);
    });
    if (nErr) nErr[0] = rc;
}

long long ParODE_PlanNumOutputs(const ParODE_Plan* plan) { return plan && plan->plan ? plan->plan->num_outputs() : -1; }

int ParODE_PlanNumOutputChannels(const ParODE_Plan* plan) { return plan && plan->plan ? plan->plan->channels() : -1; }

int ParODE_PlanLaunchCount(const ParODE_Plan* plan) { return plan && plan->plan ? plan->plan->launch_count() : 0; }

int ParODE_PlanPrecision(const ParODE_Plan* plan) { return plan && plan->plan ? plan->plan->precision_used() : -1; }

int ParODE_PlanPath(const ParODE_Plan* plan) { return plan && plan->plan ? plan->plan->path() : -1; }

void ParODE_PlanResponseShape(const ParODE_Plan* plan, long long info[4])
{
    if (!info) return;
    info[0] = info[1] = info[2] = info[3] = 0;
    if (!plan || !plan->plan) return;
    plan->plan->response_shape(info);
}

void ParODE_PlanDestroy(ParODE_Plan* plan) { delete plan; }

void ParODE_PlanSetProfiling(ParODE_Plan* plan, int enable, int nErr[])
{
    int rc = guarded([&] {
        if (!plan || !plan->plan) throw Error(kInvalidArgument, "null plan");
        plan->plan->set_profiling(enable != 0);
    });
    if (nErr) nErr[0] = rc;
}

int ParODE_PlanStageTimes(ParODE_Plan* plan, float* ms, int cap, char* names, int names_cap, int nErr[])
{
    int count = 0;
    int rc = guarded([&] {
        if (!plan || !plan->plan) throw Error(kInvalidArgument, "null plan");
        auto st = plan->plan->stage_times();
        std::string joined;
        for (auto& kv : st) {
            if (count < cap && ms) ms[count] = kv.second;
            joined += kv.first;
            joined += '\n';
            ++count;
        }
        if (names && names_cap > 0) std::snprintf(names, (size_t)names_cap, "%s", joined.c_str());
    });
    if (nErr) nErr[0] = rc;
    return count;
}

// ---- batches ---------------------------------------------------------------

struct ParODE_Batch {
    std::unique_ptr<BatchPlan> batch;
};

ParODE_Batch* ParODE_BatchCreate(int nSystems, const double* const A[], const double* const B[],
                                 const double* const C[], const double* const D[], const int nInputs[],
                                 const int nStates[], const int nOutputs[], const int ZeroB[], const int ZeroC[],
                                 const int ZeroD[], const int uIndex[], const double tStart[], const double tEnd[],
                                 const double tStep[], const double* const x0[], const int solver[], int precision,
                                 int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    ParODE_Batch* out = nullptr;
    int rc = guarded([&] {
        int dev = current_device_locked(L);
        if (precision != PARODE_PRECISION_FP64 && precision != PARODE_PRECISION_MIXED &&
            precision != PARODE_PRECISION_TF32)
            throw Error(kInvalidArgument, "unknown precision");
        if (nSystems <= 0 || !A || !x0 || !nInputs || !nStates || !nOutputs || !ZeroB || !ZeroC || !ZeroD ||
            !uIndex || !tStart || !tEnd || !tStep || !solver)
            throw Error(kInvalidArgument, "batch arrays missing");
        std::vector<BatchSpec> specs((size_t)nSystems);
        for (int i = 0; i < nSystems; ++i) {
            specs[i].sys = make_system<double>(A[i], B ? B[i] : nullptr, C ? C[i] : nullptr, D ? D[i] : nullptr,
                                               nInputs[i], nStates[i], nOutputs[i], ZeroB[i], ZeroC[i], ZeroD[i],
                                               x0[i]);
            specs[i].uIndex = uIndex[i];
            specs[i].solver = solver[i];
            specs[i].t0 = tStart[i];
            specs[i].tEnd = tEnd[i];
            specs[i].h = tStep[i];
        }
        PlanOptions opt;
        // a batch runs the single-pass TF32 form as the mixed form
        opt.precision = precision == PARODE_PRECISION_TF32 ? (int)kMixed : precision;
        opt.path = L.path;
        opt.input_double = true;
        opt.log = L.log != 0;
        opt.executions = (double)L.executions;
        opt.discretise = L.discretise;
        auto h = std::make_unique<ParODE_Batch>();
        h->batch = std::make_unique<BatchPlan>(dev, std::move(specs), &L.inputs, opt);
        out = h.release();
    });
    if (nErr) nErr[0] = rc;
    return out;
}

void ParODE_BatchExecute(ParODE_Batch* batch, void* stream, int nErr[])
{
    int rc = guarded([&] {
        if (!batch || !batch->batch) throw Error(kInvalidArgument, "null batch");
        batch->batch->execute((cudaStream_t)stream);
    });
    if (nErr) nErr[0] = rc;
}

long long ParODE_BatchNumOutputs(const ParODE_Batch* batch, int i)
{
    if (!batch || !batch->batch || i < 0 || i >= batch->batch->size()) return -1;
    return batch->batch->num_outputs(i);
}

int ParODE_BatchNumOutputChannels(const ParODE_Batch* batch, int i)
{
    if (!batch || !batch->batch || i < 0 || i >= batch->batch->size()) return -1;
    return batch->batch->channels(i);
}

const double* ParODE_BatchDeviceOutput(const ParODE_Batch* batch, int i)
{
    if (!batch || !batch->batch || i < 0 || i >= batch->batch->size()) return nullptr;
    return batch->batch->device_output(i);
}

void ParODE_BatchGetOutput(ParODE_Batch* batch, int i, double* tVect, double* yVect, int nErr[])
{
    int rc = guarded([&] {
        if (!batch || !batch->batch) throw Error(kInvalidArgument, "null batch");
        batch->batch->get_output(i, tVect, yVect);
    });
    if (nErr) nErr[0] = rc;
}

int ParODE_BatchLaunchCount(const ParODE_Batch* batch)
{
    return (batch && batch->batch) ? batch->batch->launch_count() : 0;
}

int ParODE_BatchPath(const ParODE_Batch* batch, int i)
{
    if (!batch || !batch->batch || i < 0 || i >= batch->batch->size()) return -1;
    return batch->batch->path(i);
}

int ParODE_BatchPrecision(const ParODE_Batch* batch, int i)
{
    if (!batch || !batch->batch || i < 0 || i >= batch->batch->size()) return -1;
    return batch->batch->precision_used(i);
}

double ParODE_BatchStateSteps(const ParODE_Batch* batch)
{
    return (batch && batch->batch) ? batch->batch->state_steps() : 0.0;
}

void ParODE_BatchDestroy(ParODE_Batch* batch) { delete batch; }

// ---- serving loop -------------------------------------------------------------

struct ParODE_Server {
    std::unique_ptr<Server> server;
};

ParODE_Server* ParODE_ServerCreate(int precision, double hbmBudgetBytes, int maxBatch, int maxInflight, int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    ParODE_Server* out = nullptr;
    int rc = guarded([&] {
        int dev = current_device_locked(L);
        if (precision != PARODE_PRECISION_FP64 && precision != PARODE_PRECISION_MIXED &&
            precision != PARODE_PRECISION_TF32)
            throw Error(kInvalidArgument, "unknown precision");
        ServerOptions o;
        o.precision = precision == PARODE_PRECISION_TF32 ? (int)kMixed : precision;
        if (hbmBudgetBytes > 0) o.hbm_budget = hbmBudgetBytes;
        if (maxBatch > 0) o.max_batch = maxBatch;
        if (maxInflight > 0) o.max_inflight = maxInflight;
        o.log = L.log;
        o.discretise = L.discretise;
        auto h = std::make_unique<ParODE_Server>();
        h->server = std::make_unique<Server>(dev, &L.inputs, &L.mu, o);
        out = h.release();
    });
    if (nErr) nErr[0] = rc;
    return out;
}

long long ParODE_ServerSubmit(ParODE_Server* srv, const double* A, const double* B, const double* C, const double* D,
                              int nInputs, int nStates, int nOutputs, int ZeroB, int ZeroC, int ZeroD, int uIndex,
                              double tStart, double tEnd, double tStep, const double* x0, int solver, int nErr[])
{
    long long id = 0;
    int rc = guarded([&] {
        if (!srv || !srv->server) throw Error(kInvalidArgument, "null server");
        BatchSpec s;
        s.sys = make_system<double>(A, B, C, D, nInputs, nStates, nOutputs, ZeroB, ZeroC, ZeroD, x0);
        if (solver != kRK4 && solver != kABM) throw Error(kInvalidSolverType, "unknown solver type");
        s.uIndex = uIndex;
        s.solver = solver;
        s.t0 = tStart;
        s.tEnd = tEnd;
        s.h = tStep;
        if (!s.sys.zeroB || !s.sys.zeroD) {
            // resolve the input now, under the library lock: the server's
            // set-up threads then never touch the shared registry
            Library& L = lib();
            std::lock_guard<std::recursive_mutex> g(L.mu);
            s.input = L.inputs.get(uIndex);
            if (!s.input) throw Error(kInvalidInput, "uIndex does not name a registered input");
        }
        id = srv->server->submit(std::move(s));
    });
    if (nErr) nErr[0] = rc;
    return rc == kOK ? id : rc;
}

int ParODE_ServerPoll(ParODE_Server* srv, long long id, long long nSteps[], int nChannels[], int nErr[])
{
    int done = 0;
    int rc = guarded([&] {
        if (!srv || !srv->server) throw Error(kInvalidArgument, "null server");
        int err = 0;
        long long n = 0;
        int c = 0;
        done = srv->server->poll(id, &n, &c, &err);
        if (nSteps) nSteps[0] = n;
        if (nChannels) nChannels[0] = c;
        if (done && err) throw Error(err, "the request failed");
    });
    if (nErr) nErr[0] = rc;
    return done;
}

void ParODE_ServerResult(ParODE_Server* srv, long long id, double* tVect, double* yVect, double latencyMs[],
                         int nErr[])
{
    int rc = guarded([&] {
        if (!srv || !srv->server) throw Error(kInvalidArgument, "null server");
        srv->server->result(id, tVect, yVect, latencyMs);
    });
    if (nErr) nErr[0] = rc;
}

void ParODE_ServerStats(ParODE_Server* srv, double stats[], int nErr[])
{
    int rc = guarded([&] {
        if (!srv || !srv->server) throw Error(kInvalidArgument, "null server");
        if (!stats) return;
        ServerStats s = srv->server->stats();
        const double v[12] = {(double)s.submitted, (double)s.completed, (double)s.failed, s.p50_ms, s.p99_ms,
                              s.mean_ms, s.max_ms, s.state_steps, s.span_s, s.peak_bytes, (double)s.batches, 0.0};
        for (int k = 0; k < 12; ++k) stats[k] = v[k];
    });
    if (nErr) nErr[0] = rc;
}

void ParODE_ServerDestroy(ParODE_Server* srv) { delete srv; }

void ParODE_SimulateODEBatch(int nSystems, const double* const A[], const double* const B[], const double* const C[],
                             const double* const D[], const int nInputs[], const int nStates[], const int nOutputs[],
                             const int ZeroB[], const int ZeroC[], const int ZeroD[], const int uIndex[],
                             const double tStart[], const double tEnd[], const double tStep[],
                             const double* const x0[], const int solver[], int precision, double* const tVect[],
                             double* const yVect[], long long nSteps[], int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    int err = 0;
    ParODE_Batch* b = ParODE_BatchCreate(nSystems, A, B, C, D, nInputs, nStates, nOutputs, ZeroB, ZeroC, ZeroD,
                                         uIndex, tStart, tEnd, tStep, x0, solver, precision, &err);
    if (err == 0) {
        ParODE_BatchExecute(b, nullptr, &err);
        for (int i = 0; err == 0 && i < nSystems; ++i) {
            ParODE_BatchGetOutput(b, i, tVect ? tVect[i] : nullptr, yVect ? yVect[i] : nullptr, &err);
            if (nSteps) nSteps[i] = ParODE_BatchNumOutputs(b, i);
        }
    }
    ParODE_BatchDestroy(b);
    if (nErr) nErr[0] = err;
}


void ParODE_AffineScanGeneral(const double* dM, const double* dV, const double* dX0, int ns, long long count,
                              int precision, double* dX, void* stream, int nErr[])
{
    int rc = guarded([&] {
        if (precision != PARODE_PRECISION_FP64 && precision != PARODE_PRECISION_MIXED)
            throw Error(kInvalidArgument, "unknown precision");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        int* status = nullptr;
        if (fault_alloc_now()) throw Error(kNotEnoughResources, "device allocation failed (injected)");
        if (cudaMallocAsync(reinterpret_cast<void**>(&status), sizeof(int), s) != cudaSuccess) {
            cudaGetLastError();
            throw Error(kNotEnoughResources, "device allocation failed");
        }
        int host_status = 0;
        try {
            PARODE_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
            general_scan(dM, dV, dX0, ns, (long)count, precision, dX, status, s);
            PARODE_CUDA(cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, s));
            PARODE_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaFreeAsync(status, s);
            throw;
        }
        PARODE_CUDA(cudaFreeAsync(status, s));
        if (host_status != 0) throw Error(kDeviceError, "a device-side wait gave up (tensor-core completion not observed)");
    });
    if (nErr) nErr[0] = rc;
}


// ---------------------------------------------------------------------------
// measured block length of the response leaf (tuner.h)
// ---------------------------------------------------------------------------

}  // extern "C"

namespace {

// The GPU's name as the tuning file keys it (spaces replaced).
std::string gpu_key(const char* given)
{
    std::string name;
    if (given && *given) {
        name = given;
    } else {
        int dev = 0;
        cudaDeviceProp prop;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
            cudaGetLastError();
            throw Error(kNoGPU, "no device to key the tuning table");
        }
        name = prop.name;
    }
    for (char& c : name)
        if (c == ' ' || c == '\t') c = '_';
    return name;
}

// A stable system of the class with seeded entries: A = -1.5 I + 0.5 G / sqrt(n),
// B, C, D, x0 of unit scale (a counter-based generator, the same every call).
SystemDesc tune_system(int n, int m, int p)
{
    uint64_t st = 0x9E3779B97F4A7C15ull * (uint64_t)(n * 131 + m * 7 + p);
    auto unif = [&st]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto normal = [&unif]() { return std::sqrt(-2.0 * std::log(1.0 - unif())) * std::cos(6.283185307179586 * unif()); };
    SystemDesc s;
    s.n = n;
    s.m = m;
    s.p = p;
    s.zeroB = s.zeroC = s.zeroD = false;
    s.A.resize((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) s.A[(size_t)i * n + j] = (i == j ? -1.5 : 0.0) + 0.5 * normal() / std::sqrt((double)n);
    s.B.resize((size_t)n * m);
    for (double& v : s.B) v = normal();
    s.C.resize((size_t)p * n);
    for (double& v : s.C) v = normal();
    s.D.resize((size_t)p * m);
    for (double& v : s.D) v = normal();
    s.x0.resize(n);
    for (double& v : s.x0) v = normal();
    return s;
}

}  // namespace

extern "C" {

void ParODE_TuneResponseBlock(int solver, int nStates, int nInputs, int nOutputs, long long nSteps, int precision,
                              int log2B[], float msBest[], float msModel[], int nErr[])
{
    Library& L = lib();
    std::lock_guard<std::recursive_mutex> g(L.mu);
    int rc = guarded([&] {
        const int dev = current_device_locked(L);
        if (solver != kRK4 && solver != kABM) throw Error(kInvalidSolverType, "unknown solver");
        if (nStates < 1 || nInputs < 1 || nOutputs < 1 || nSteps < 2) throw Error(kInvalidSystem, "empty class");
        if (precision != PARODE_PRECISION_FP64 && precision != PARODE_PRECISION_MIXED &&
            precision != PARODE_PRECISION_TF32)
            throw Error(kInvalidArgument, "unknown precision");
        const int Ns = solver == kRK4 ? nStates : 4 * nStates;
        if (Ns > 1024) throw Error(kInvalidSystem, "scan dimension above 1024 is not supported");
        SystemDesc s = tune_system(nStates, nInputs, nOutputs);
        // a three-term sinusoid input per input count, registered once
        if ((int)L.tune_inputs.size() <= nInputs) L.tune_inputs.resize(nInputs + 1, -1);
        if (L.tune_inputs[nInputs] < 0) {
            std::vector<double> a((size_t)nInputs * 3), f(a.size()), ph(a.size());
            for (size_t q = 0; q < a.size(); ++q) {
                a[q] = 0.5 + 0.1 * (double)(q % 5);
                f[q] = 0.3 + 1.7 * (double)(q % 7);
                ph[q] = 0.4 * (double)q;
            }
            L.tune_inputs[nInputs] = L.inputs.add_sinusoid(nInputs, 3, a.data(), f.data(), ph.data());
        }
        const int uIndex = L.tune_inputs[nInputs];
        const double h = 1e-3, tEnd = ((double)nSteps - 0.5) * h;
        long nScan = 0;
        num_outputs(solver, 0.0, tEnd, h, &nScan);
        // the untuned choice: the blocked shape's block for scan dimensions up
        // to 64 (single solves), else the cost model's
        const int np = (int)round_up(Ns, 8);
        int Rdefault = 0;
        BlockedShape sh;
        if (Ns <= 64 && blocked_shape(Ns, nInputs, solver, &sh)) {
            Rdefault = sh.R;
        } else {
            double cost = 0.0;
            Rdefault = response_log2_block(solver, np, nStates, nInputs, nOutputs, nScan,
                                           precision != PARODE_PRECISION_FP64 ? 0.25 : 1.0, (double)L.executions,
                                           &cost);
        }
        while (Rdefault > 2 && (1L << Rdefault) / 2 >= nScan) --Rdefault;
        auto time_R = [&](int R) -> float {
            PlanOptions opt;
            opt.precision = precision;
            opt.path = kPathBlockedResponse;
            opt.input_double = true;
            opt.force_log2_block = R;
            Plan plan(dev, s, &L.inputs, uIndex, solver, 0.0, tEnd, h, opt);
            cudaStream_t st = plan.stream();
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            PARODE_CUDA(cudaEventCreate(&e0));
            PARODE_CUDA(cudaEventCreate(&e1));
            std::vector<float> ts;
            try {
                for (int it = 0; it < 2; ++it) plan.execute(nullptr, st);
                for (int it = 0; it < 5; ++it) {
                    PARODE_CUDA(cudaEventRecord(e0, st));
                    plan.execute(nullptr, st);
                    PARODE_CUDA(cudaEventRecord(e1, st));
                    PARODE_CUDA(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    PARODE_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                    ts.push_back(ms);
                }
                plan.get_output(nullptr, nullptr);  // reports a device wait that gave up
            } catch (...) {
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                throw;
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            std::sort(ts.begin(), ts.end());
            return ts[ts.size() / 2];
        };
        int best = -1;
        float best_ms = 0.f, model_ms = 0.f;
        for (int R = 2; R <= 7; ++R) {
            const long B = 1L << R;
            if (R > 2 && B / 2 >= nScan) break;
            const long K = response_window(solver, (int)B, nInputs);
            if (8.0 * ((double)B * nOutputs + np) * ((double)K + np) > 256e6) break;
            float ms = 0.f;
            try {
                ms = time_R(R);
            } catch (const Error& e) {
                // a block length the engine cannot build for this class (a
                // resource limit) is not a candidate; anything else is an error
                if (e.code != kNotEnoughResources && e.code != kInvalidArgument) throw;
                continue;
            }
            if (R == Rdefault) model_ms = ms;
            if (best < 0 || ms < best_ms) {
                best = R;
                best_ms = ms;
            }
        }
        if (best < 0) throw Error(kInvalidSystem, "no block length fits the class");
        if (model_ms == 0.f) model_ms = time_R(Rdefault);
        tune_store(tune_class(solver, Ns, nInputs, nOutputs, nScan, precision), best, best_ms);
        if (log2B) log2B[0] = best;
        if (msBest) msBest[0] = best_ms;
        if (msModel) msModel[0] = model_ms;
    });
    if (nErr) nErr[0] = rc;
}

int ParODE_TuneSave(const char* path, const char* gpuName, int nErr[])
{
    int n = 0;
    int rc = guarded([&] {
        if (!path) throw Error(kInvalidArgument, "no path");
        const std::string text = tune_dump(gpu_key(gpuName));
        std::ofstream f(path, std::ios::out | std::ios::trunc);
        if (!f) throw Error(kInvalidArgument, "cannot write the tuning file");
        f << text;
        for (char c : text) n += c == '\n';
    });
    if (nErr) nErr[0] = rc;
    return n;
}

int ParODE_TuneLoad(const char* path, const char* gpuName, int nErr[])
{
    int n = 0;
    int rc = guarded([&] {
        if (!path) throw Error(kInvalidArgument, "no path");
        std::ifstream f(path);
        if (!f) throw Error(kInvalidArgument, "cannot read the tuning file");
        std::stringstream ss;
        ss << f.rdbuf();
        n = tune_load_text(ss.str(), gpu_key(gpuName));
    });
    if (nErr) nErr[0] = rc;
    return n;
}

void ParODE_TuneClear() { tune_clear(); }

}  // extern "C"
