// solver.h -- a device-resident solve of one LTI system (a "plan").
//
// Replaces the reference's solver objects (GPUODESolverFixedStepIterative and
// its RungeKutta4thOrder / AdamsMoulton subclasses,
// Sources/GPUFixedStepIterative.cpp:131-466): set-up on the host in FP64,
// every per-step stage on the device, no host round trip inside a solve.
#pragma once

#include "blocked.h"
#include "host_math.h"
#include "inputs.h"
#include "kernels.h"

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace parode {

class BatchPlan;

// kPathBlocked chooses the leaf by cost; kPathBlockedResponse / kPathBlockedSweep
// force the block-response GEMM leaf / the in-block sweep leaf.
// kPathGeneral runs the reference's pipeline step for step: T copies of Phi,
// the forcing vectors, the general scan composing every pair (general.h).
enum Path : int {
    kPathAuto = 0,
    kPathLevel = 1,
    kPathBlocked = 2,
    kPathBlockedResponse = 3,
    kPathBlockedSweep = 4,
    kPathGeneral = 5
};

struct PlanOptions {
    int precision = 0;  // Precision
    int path = kPathAuto;
    bool input_double = true;  // fType of a user input function: double (true) or float
    bool log = false;          // set-up phase times on stderr
    // solves the plan is expected to run: the response leaf's block size
    // weighs the FP64 build of its tables against the work of that many
    // solves (1: one-shot, as SimulateODE and the server)
    double executions = 1.0;
    // test hook (PARODE_OPT_FAULT_WITHHOLD): the mixed response kernel's
    // first CTA withholds one pipeline arrive, so its bounded waits give up
    bool fault_withhold = false;
    // block-response leaf: log2 of the block length (0: the tuned value of
    // the system's class, else the cost model's / the shape's default)
    int force_log2_block = 0;
    // time partition of the solve across devices (setup_shard): this plan is
    // shard `shard` of `shards` (shards > 1)
    int shard = 0, shards = 1;
    // where a batch discretises its systems (DiscretiseAt)
    int discretise = 0;
    // solved once, right after creation, on the plan's own stream (the
    // one-shot SimulateODE calls): creation returns without waiting for its
    // device work, which the solve queues behind and whose synchronise ends both
    bool one_shot = false;
};

// Batch discretisation: by its cost (small batches on the host threads,
// large ones on the device), or forced to one side.  Both give the same bits.
enum DiscretiseAt { kDiscAuto = 0, kDiscHost = 1, kDiscDevice = 2 };

class Plan {
public:
    Plan(int device, const SystemDesc& sys, InputRegistry* inputs, int uIndex, int solver, double t0, double tEnd,
         double h, const PlanOptions& opt);
    ~Plan();
    Plan(const Plan&) = delete;
    Plan& operator=(const Plan&) = delete;

    // Enqueue one solve on `s` (nullptr = the plan's stream); y (device,
    // num_outputs() x channels() doubles) or nullptr for the plan's buffer.
    void execute(double* y, cudaStream_t s);
    // Synchronise and copy the last result (and the time vector) to the host.
    void get_output(double* t, double* y);
    void get_output_f32(float* t, float* y);  // the same values rounded to float (y on the device)
    // One-shot execute with y copied to the host (yd as double, or yf rounded
    // to float on the device; at most one non-null): on the block-response
    // path the output stage runs over four block ranges and each range's rows
    // are copied out on the side stream while the later ranges are formed.
    // The same bits as execute followed by get_output / get_output_f32.
    void solve_to_host(double* yd, float* yf);

    long num_outputs() const { return nOut_; }
    long scan_steps() const { return nScan_; }
    int padded_dim() const { return Np_; }
    // Scan dimensions above 64 run as a one-system BatchPlan (batch.h): the
    // response leaf with a level-synchronous scan over blocks, or the
    // level-synchronous scan over steps, with the batch's tensor-core levels.
    bool delegated() const { return (bool)batch_; }
    int channels() const { return p_; }
    int launch_count() const { return launches_; }
    int device() const { return device_; }
    cudaStream_t stream() const { return stream_; }
    const double* device_output() const;
    // kPathLevel, kPathBlocked (in-block sweep leaf) or kPathBlockedResponse
    int path() const { return br_ ? (int)kPathBlockedResponse : path_; }
    // Response leaf: block length, window columns, padded scan dimension,
    // blocks (zeros when not that path)
    void response_shape(long long info[4]) const;
    int precision_used() const { return precision_used_; }

    // Time shard (PlanOptions::shards > 1; block-response path only).  The
    // plan covers the scan steps [info[0], info[0] + info[1]) of the horizon;
    // its outputs are num_outputs() rows whose first ybase (3 for ABM, else
    // 0) are the start-up rows on shard 0 only, the rest the shard's steps.
    // shard_up writes info[2] items of info[3] doubles (the shard's chunk
    // aggregates) to dTop; once every shard's items are gathered in shard
    // order (info[4] x info[2] items), shard_down finishes the solve into y.
    void shard_info(long long info[5]) const;
    void shard_up(double* dTop, cudaStream_t s);
    void shard_down(const double* dGathered, double* y, cudaStream_t s);

    // Optional stage timing with CUDA events on the execution stream.
    void set_profiling(bool on);
    // Stage names and milliseconds of the last profiled execute (synchronises).
    std::vector<std::pair<std::string, float>> stage_times();

private:
    void build(int device, const SystemDesc& sys, InputRegistry* inputs, int uIndex, int solver, double t0,
               double tEnd, double h, const PlanOptions& opt);
    void release() noexcept;
    void alloc(double** p, long n);
    void carve(const std::vector<std::pair<double**, long>>& want);  // one allocation, parts assigned
    void h2d(void* dst, const void* src, size_t bytes);
    void mark(const char* stage, cudaStream_t s);
    void execute_body(double* y, cudaStream_t s);
    void execute_blocked(double* Y, cudaStream_t s);
    void execute_response(double* Y, cudaStream_t s);
    void execute_general(double* Y, cudaStream_t s);
    int carry(cudaStream_t s);
    LevelArgs response_agg_args() const;
    LevelArgs response_out_args(double* Y) const;
    int response_head(cudaStream_t s);  // inputs, aggregates, carry; returns the launches
    void response_outputs(double* Y, long c0, long c1, cudaStream_t s);  // blocks [c0, c1)
    void state_part(double* Y, long c0, long c1, cudaStream_t s);
    void setup_shard(const PlanOptions& opt);
    void fill_inputs(cudaStream_t s);

    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    SystemDesc sys_;
    InputRegistry* inputs_ = nullptr;
    InputEntry* input_ = nullptr;
    PlanOptions opt_;
    int solver_ = 0;
    double t0_ = 0, tEnd_ = 0, h_ = 0;
    long nOut_ = 0, nScan_ = 0, Tp_ = 1, nU_ = 0;
    int Ns_ = 0, Np_ = 0, p_ = 0, mu_ = 0, levels_ = 0;
    int path_ = kPathLevel;
    int launches_ = 0;
    double u_base_ = 0, u_dt_ = 0;
    std::vector<double> ypre_;  // ABM: outputs 0..2 computed on the host
    std::vector<double*> bufs_;
    double *dPow_ = nullptr, *dBbar_ = nullptr, *dC_ = nullptr, *dD_ = nullptr, *dX0_ = nullptr;
    double *dU_ = nullptr, *dV_ = nullptr, *dY_ = nullptr, *dYpre_ = nullptr;
    double* last_y_ = nullptr;
    BlockedShape shape_;
    long ntiles_ = 0, nblocks_ = 0;
    bool gen_ = false;
    int sms_ = 148;
    double *dG_ = nullptr, *dWork_ = nullptr, *dCP_ = nullptr, *dCext_ = nullptr;
    size_t stage_bytes_ = 0;
    int precision_used_ = 0;
    bool br_ = false;           // leaf = block response GEMM (kernels_br.cu)
    int brK_ = 0, brKpad_ = 0;  // window columns (padded to even)
    double* dW_ = nullptr;      // response matrix, (B p + NP) x (brKpad_ + NP)
    double* dMs_ = nullptr;     // general path: T copies of Phi (Ns x Ns each)
    double* dXs_ = nullptr;     // general path: the states x_k (T x Ns)
    // mixed form of the response leaf: aggregates and output windows on the
    // tensor cores (one grouped launch of two GEMMs), state part in FP64
    bool br_tc_ = false;
    LevelArgs* dTc_ = nullptr;  // device: the two GEMMs as k_split reads them
    RespArgs* dResp_ = nullptr; // device: the two GEMMs as the tensor-core kernel reads them
    float* dUh_ = nullptr;      // input samples as TF32 hi / lo planes
    float* dUl_ = nullptr;
    long* dTcStart_ = nullptr;  // device: their first tiles
    long* dTcCta_ = nullptr;    // device: tile ranges of the persistent CTAs
    int tcCtas_ = 0;
    int* dStatus_ = nullptr;
    bool one_pass_ = false;  // single-pass TF32 response GEMMs (hi*hi only)
    cudaStream_t side_ = nullptr;
    cudaEvent_t fork_[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t done_ = nullptr;  // recorded after each execute on its stream
    size_t bytes_ = 0;            // device bytes the plan holds
    std::unique_ptr<BatchPlan> batch_;
    bool profiling_ = false;
    std::vector<cudaEvent_t> events_;
    std::vector<std::string> marks_;
    // time shard (setup_shard)
    int shard_ = 0, shards_ = 1, shard_k_ = 0, shard_c_ = 0;
    long shard_begin_ = 0, nScanGlobal_ = 0;
    long u_joff_ = 0;           // index of the first input sample on the whole horizon
    double* dTop_ = nullptr;    // gathered top items + their scan's scratch
    ChunkLevels shard_levels_;  // the up-sweep's levels, reused by the down-sweep
    bool shard_up_done_ = false;
    bool tables_pending_ = false;  // one-shot response plan: the power table's stream joins before the carry
    char* pin_ = nullptr;  // pinned staging of the set-up copies (h2d)
    size_t pin_used_ = 0;
    bool pin_tried_ = false;
    // the launch list as a CUDA graph (execute): 0 none, 1 executed once into
    // graph_y_, 2 graph ready for graph_y_, -1 capture failed
    int graph_state_ = 0;
    double* graph_y_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    bool capture_graph(double* y);
};

}  // namespace parode
