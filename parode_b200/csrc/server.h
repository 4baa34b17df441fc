// server.h -- continuous-batching request loop over the batched engine.
//
// The reference serves nothing: one blocking SimulateODE call per system
// (Sources/ParODE.cpp:281-337).  The server accepts solves asynchronously
// (submit / poll / result), and a scheduler thread
//  - admits pending requests against an HBM budget (device bytes of the
//    batch each request would join, estimated before any allocation),
//  - forms a batch from what is pending as soon as capacity frees up, sets it
//    up (host FP64 discretisation, one stream-ordered arena) and enqueues it on
//    its own stream, so batches that arrive while others run overlap on the
//    device,
//  - hands finished batches (event query) to copy-out threads, which move
//    each request's outputs device-to-device into a pooled buffer of its own
//    (counted against the budget until the caller collects it with result())
//    and release the batch's arena.
// Latency of a request = completion - submission (host clock).
#pragma once

#include "batch.h"

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace parode {

struct ServerOptions {
    int precision = 0;
    double hbm_budget = 150e9;  // bytes of device memory for in-flight batches
    int max_batch = 256;        // systems per batch
    int max_inflight = 8;       // batches on the device (or being set up) at once
    int setup_threads = 4;      // host threads building batches concurrently
    int log = 0;                // 1: each batch's timeline on stderr; 2: also its set-up phases (which wait on the device)
    int discretise = 0;         // where batches discretise (PlanOptions::discretise)
    // device memory mapped into the stream-ordered pool at creation (at most
    // the budget and half the free memory)
    size_t prewarm_bytes = (size_t)32 << 30;
};

struct ServerStats {
    long submitted = 0, completed = 0, failed = 0;
    double p50_ms = 0, p99_ms = 0, mean_ms = 0, max_ms = 0;
    double state_steps = 0;     // sum of n x outputs of completed requests
    double span_s = 0;          // first submission -> last completion
    double peak_bytes = 0;      // largest device bytes in flight
    long batches = 0;
};

// Device bytes a request needs inside a batch (upper estimate, before any
// allocation): power table, scan buffers, inputs, outputs, constants.
size_t estimate_request_bytes(const BatchSpec& s, int precision);

class Server {
public:
    Server(int device, InputRegistry* inputs, std::recursive_mutex* inputs_mu, const ServerOptions& opt);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // Queues a solve; returns its id (> 0).  Throws Error when the request
    // alone exceeds the HBM budget or is invalid.
    long long submit(BatchSpec spec);
    // 1 when finished (result ready or failed), 0 while pending; fills the
    // output count and channels when finished.  Throws for an unknown id.
    int poll(long long id, long long* n_out, int* channels, int* err);
    // Copies the outputs (and time vector) of a finished request, releases it.
    void result(long long id, double* t, double* y, double* latency_ms);
    ServerStats stats();

private:
    struct Request {
        long long id = 0;
        BatchSpec spec;
        size_t bytes = 0;
        double t_submit = 0, t_done = 0;
        bool done = false;
        int err = 0;
        long n_out = 0;
        int channels = 0;
        double* dy = nullptr;  // n_out x channels on the device until collected
        size_t ny = 0;
        double state_steps = 0;
    };
    struct Inflight {
        std::unique_ptr<BatchPlan> plan;
        std::vector<std::shared_ptr<Request>> reqs;
        cudaEvent_t done = nullptr;
        size_t bytes = 0;
        // host times (log): admitted, enqueued on the device, seen finished
        double t_admit = 0, t_start = 0, t_ready = 0, t_seen = 0;
    };

    struct Job {
        std::vector<std::shared_ptr<Request>> reqs;
        size_t bytes = 0;
        double t_admit = 0;
    };

    void loop();
    void worker();
    void retirer();
    void admit_locked();
    // What retire() found for one request; published under mu_ by retirer().
    struct Outcome {
        int err = 0;
        double* dy = nullptr;
        size_t ny = 0;
        double t_done = 0;
    };
    void retire(Inflight& f, cudaStream_t st, std::vector<Outcome>& out);

    int device_;
    InputRegistry* inputs_;
    std::recursive_mutex* inputs_mu_;
    ServerOptions opt_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::shared_ptr<Request>> pending_;
    std::unordered_map<long long, std::shared_ptr<Request>> all_;
    std::vector<Inflight> inflight_;
    size_t inflight_bytes_ = 0;
    size_t held_bytes_ = 0;  // finished results not yet collected (device memory)
    cudaStream_t copy_stream_ = nullptr;  // result(): device -> caller copies
    long long next_id_ = 1;
    bool stop_ = false;
    std::vector<double> latencies_;
    ServerStats st_;
    double t_first_ = -1, t_last_ = 0;
    std::deque<Job> jobs_;      // admitted batches waiting for a set-up worker
    int setting_up_ = 0;        // batches admitted and not yet on the device
    bool workers_stop_ = false;
    std::condition_variable jobs_cv_;
    std::vector<std::thread> workers_;
    // finished batches wait here for a copy-out thread, off the scheduler
    std::deque<Inflight> retire_q_;
    int retiring_ = 0;
    std::condition_variable retire_cv_;
    std::vector<std::thread> retirers_;
    std::thread thread_;
};

}  // namespace parode
