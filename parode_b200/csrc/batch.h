// batch.h -- many independent LTI solves in one set of launches.
//
// The reference solves one system per SimulateODE call, creating its solver
// and buffers each time (Sources/ParODE.cpp:281-337).  A batch keeps every
// system's matrices, power tables, scan buffers and outputs resident in one
// device arena and runs all systems together:
//  - scan dimension <= 64: the blocked path per padded dimension NP, batched
//    (one tables launch, one persistent leaf launch over work items of all
//    systems, one chain launch, one fix-up launch per NP);
//  - larger scan dimensions: the level-synchronous path with one grouped
//    contraction launch per level and tiling configuration over all systems;
//  - systems with inputs where it costs less: the block-response leaf (one
//    GEMM of W x [sample windows] per system for the block aggregates, the
//    level-synchronous scan over the blocks, one GEMM for the outputs), the
//    GEMMs of all such systems grouped into one launch each.
// Inputs: sum-of-sinusoid inputs are sampled by one batched launch; user
// (NVRTC) inputs by one launch per system.
#pragma once

#include "blocked.h"
#include "host_math.h"
#include "inputs.h"
#include "kernels.h"
#include "solver.h"

#include <cuda_runtime.h>

#include <memory>
#include <vector>

namespace parode {

struct BatchSpec {
    SystemDesc sys;
    int uIndex = 0;
    int solver = 0;
    double t0 = 0, tEnd = 0, h = 0;
    // the registered input, resolved by the caller under the library lock
    // (nullptr: looked up from uIndex during set-up)
    InputEntry* input = nullptr;
};

// Host staging of a batch's uploads: a pooled pinned block (kept for the next
// batch when this one is done), or pageable memory when pinning fails.
class HostStage {
public:
    explicit HostStage(size_t bytes);
    ~HostStage();
    // pins `blocks` free blocks of every class up to 2^max_log2 bytes ahead
    // of use (a server's start)
    static void prewarm(int blocks, int max_log2);
    HostStage(const HostStage&) = delete;
    HostStage& operator=(const HostStage&) = delete;
    char* data() { return p_; }

private:
    char* p_ = nullptr;
    size_t cap_ = 0;
    bool pinned_ = false;
    std::unique_ptr<char[]> owned_;
};

class BatchPlan {
public:
    BatchPlan(int device, std::vector<BatchSpec> specs, InputRegistry* inputs, const PlanOptions& opt);
    ~BatchPlan();
    BatchPlan(const BatchPlan&) = delete;
    BatchPlan& operator=(const BatchPlan&) = delete;

    // Enqueue all solves on `s` (nullptr: the batch's stream).
    void execute(cudaStream_t s);
    int size() const { return (int)sys_.size(); }
    long num_outputs(int i) const { return sys_[i].nOut; }
    int channels(int i) const { return sys_[i].p; }
    // Synchronises and copies system i's time vector and outputs to the host.
    void get_output(int i, double* t, double* y);
    const double* device_output(int i) const { return sys_[i].Y; }
    int launch_count() const { return launches_; }
    int precision_used(int i) const { return sys_[i].precision; }
    int path(int i) const
    {
        return sys_[i].resp ? kPathBlockedResponse : sys_[i].blocked ? kPathBlocked : kPathLevel;
    }
    // Response leaf geometry of system i: block length, window columns,
    // padded scan dimension, blocks (zeros on other paths).
    void response_shape(int i, long long info[4]) const
    {
        const Sys& q = sys_[i];
        info[0] = q.resp ? q.Bk : 0;
        info[1] = q.resp ? q.Kw : 0;
        info[2] = q.resp ? q.Np : 0;
        info[3] = q.resp ? q.nblocks : 0;
    }
    // Sum over systems of n * outputs (state*steps of one execute).
    double state_steps() const;
    size_t device_bytes() const { return arena_bytes_; }
    cudaStream_t stream() const { return stream_; }

private:
    struct Sys {
        int solver = 0, n = 0, m = 0, mu = 0, p = 0, Ns = 0, Np = 0, W = 3;
        long nOut = 0, nScan = 0, nU = 0, Tp = 1;
        int levels = 0;           // levels of the level-synchronous scan (over steps, or over blocks)
        int lev0 = 0;             // power-table level of scan level 0 (log2 of the block length)
        int pow_levels = 0;       // power-table levels P_0 .. P_{pow_levels - 1}
        bool blocked = false;
        bool resp = false;        // block-response leaf
        int Bk = 0, Kw = 0, Kpad = 0;  // response: block length, window columns (padded to even)
        long nblocks = 0;
        double* Wm = nullptr;     // response matrix: Bk p + Np rows of Kpad + Np
        bool resp_tc = false;     // mixed: response GEMMs on the tensor cores
        float* Psa = nullptr;     // W's aggregate rows, TF32-split
        float* Psw = nullptr;     // W's output rows (window columns), TF32-split
        int bucket = -1;          // blocked: index into buckets_
        double delta = 0;         // |Phi - R|_inf, R the exact 0/1 part (I or the ABM shift)
        int tc_levels = 0;        // mixed: lowest levels run on the tensor cores
        float* Ps = nullptr;      // mixed: pre-split P_l - R_l per tensor-core level
        int precision = 0;
        InputEntry* input = nullptr;
        double u_base = 0, u_dt = 0;
        double t0 = 0, tEnd = 0, h = 0;
        // device pointers inside the arena
        double *P = nullptr, *Bbar = nullptr, *C = nullptr, *D = nullptr, *X0 = nullptr, *U = nullptr;
        double *Y = nullptr, *V = nullptr, *G = nullptr, *CP = nullptr, *Cext = nullptr, *sin = nullptr;
        int K = 0;
        bool zeroB = true, zeroC = true, zeroD = true;
        long ntiles = 0;
    };
    struct Bucket {
        BlockedShape sh;
        std::vector<int> systems;
        int ms = 0, pmax = 1;
        long max_blocks = 0;
        bool stage = false;
        size_t leaf_smem = 0;
        BatchLaunch launch;  // device arrays filled at set-up
    };
    struct GroupedLaunch {
        LevelConfig cfg;
        LevelArgs* args = nullptr;  // device
        long* start = nullptr;      // device
        int nent = 0;
        long tiles = 0;
        size_t smem = 0;
        LevelArgs* swaps = nullptr;  // device: down-sweep entries of the tiled form, swapped first
        int nswap = 0;
        long swap_elems = 0;
        long* cta = nullptr;         // tensor-core launch: per-CTA tile ranges (ctas + 1)
        int ctas = 0;
    };

    void launch_grouped(const GroupedLaunch& g, cudaStream_t s);
    void build(std::vector<BatchSpec> specs, InputRegistry* inputs, const PlanOptions& opt);
    void release();  // idempotent: what the plan holds on the device goes back
    void build_responses();

    int device_ = 0;
    int sms_ = 148;
    int* dStatus_ = nullptr;  // set by a device wait that gave up
    cudaStream_t last_stream_ = nullptr;
    // the launch list as a CUDA graph (execute): 0 no execute yet, 1 one eager
    // execute, 2 graph instantiated, -1 capture failed (eager from then on)
    int graph_state_ = 0;
    void* disc_ = nullptr;  // A, B, the compact Phi, Bbar (and transposes) of every system
    cudaGraphExec_t graph_exec_ = nullptr;
    void enqueue(cudaStream_t s);
    bool capture_graph();
    cudaStream_t stream_ = nullptr;
    std::vector<cudaStream_t> forks_;
    std::vector<cudaEvent_t> events_;
    // set-up finished on stream_ (an execute on another stream waits for it)
    cudaEvent_t ready_ = nullptr;
    // host images of the set-up copies, kept until the plan is destroyed so
    // that the constructor returns without waiting for the device
    std::vector<std::unique_ptr<HostStage>> host_keep_;
    std::unique_ptr<HostStage> host_disc_;   // the host discretisation's results (small batches)
    std::unique_ptr<HostStage> host_stage_;  // the staged constant region
    std::unique_ptr<HostStage> host_jobs_;   // the staged job arrays
    InputRegistry* inputs_ = nullptr;
    PlanOptions opt_;
    std::vector<Sys> sys_;
    std::vector<Bucket> buckets_;
    std::vector<int> ls_;  // level-synchronous systems
    std::vector<int> rs_;  // block-response systems (their block scan joins the level launches)
    std::vector<GroupedLaunch> ls_power_, ls_up_, ls_down_;
    std::vector<GroupedLaunch> rs_agg_, rs_out_;  // response GEMMs: block aggregates, outputs
    std::vector<GroupedLaunch> rs_tc_, rs_state_;  // mixed: tensor-core aggregates + windows; FP64 state part
    CopyJob* dZero_ = nullptr;                     // mixed: the block scans' padding slots
    int nZero_ = 0;
    long maxZero_ = 0;
    SampleJob* dSampleJobs_ = nullptr;
    int nSampleJobs_ = 0;
    long maxSample_ = 0;
    int maxTerms_ = 1;  // the largest sinusoid term count of the sample jobs
    std::vector<int> user_inputs_;  // systems sampled by their own launch
    ForcingJob* dForcing_ = nullptr;
    OutputJob* dOutput_ = nullptr;
    CopyJob* dSeed_ = nullptr;
    int nSeed_ = 0;
    LevelArgs* dSplit_ = nullptr;  // mixed: P_l - R_l splits (one per system and tensor-core level)
    int nSplit_ = 0;
    long maxSplitElems_ = 0;
    long maxForcing_ = 0, maxOutput_ = 0, maxSeed_ = 0;
    void* arena_ = nullptr;
    size_t arena_bytes_ = 0;
    int launches_ = 0;
};

}  // namespace parode
