// server.cpp -- continuous-batching request loop (see server.h).
#include "server.h"

#include "blocked.h"
#include "common.h"
#include "kernels.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>

namespace parode {

namespace {

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

}  // namespace

size_t estimate_request_bytes(const BatchSpec& b, int precision)
{
    const SystemDesc& s = b.sys;
    long nScan = 0;
    const long nOut = num_outputs(b.solver, b.t0, b.tEnd, b.h, &nScan);
    if (nOut <= 0 || nScan <= 0 || s.n <= 0) return 0;
    const int Ns = b.solver == kRK4 ? s.n : 4 * s.n;
    const int p = s.out_size();
    const int mu = (!s.zeroB || !s.zeroD) ? s.m : 0;
    const int W = b.solver == kRK4 ? 3 : 5;
    const long nU = b.solver == kRK4 ? 2 * nScan + 1 : nScan + 4;
    double bytes = 8.0 * ((double)nU * mu + (double)nOut * p);              // inputs, outputs
    bytes += 8.0 * ((double)s.n * W * std::max(mu, 1) + 2.0 * p * (s.n + s.m) + 4.0 * Ns);  // constants
    BlockedShape sh;
    if (blocked_shape(Ns, std::max(mu, 1), 0, &sh)) {
        const double NP = sh.NP;
        bytes += 8.0 * NP * NP * (sh.R + 2);                                  // power table + Phi
        bytes += 8.0 * ((double)(nScan + sh.S) / sh.B + 1) * NP;              // block aggregates
        bytes += 8.0 * sh.B * p * NP + 8.0 * p * NP;                          // output tables
    } else {
        const double Np = (double)round_up(Ns, 8);
        const long Tp = next_pow2(nScan);
        const int levels = std::max(ilog2(Tp), 1);
        bytes += 8.0 * (double)(Tp + 1) * Np;                                 // scan vectors
        bytes += 8.0 * Np * Np * (levels + 1);                                // power table + Phi
        if (precision == kMixed) bytes += (double)level_split_bytes((int)Np) * levels;
        bytes += 8.0 * (double)levels * 1024;                                 // launch descriptors
    }
    return (size_t)(bytes * 1.05) + (1u << 20);
}

Server::Server(int device, InputRegistry* inputs, std::recursive_mutex* inputs_mu, const ServerOptions& opt)
    : device_(device), inputs_(inputs), inputs_mu_(inputs_mu), opt_(opt)
{
    if (opt_.max_batch < 1 || opt_.max_inflight < 1 || !(opt_.hbm_budget > 0))
        throw Error(kInvalidArgument, "server options");
    // batches allocate from the device's stream-ordered pool; keep freed
    // memory in the pool (up to the budget) so that later batches reuse it
    // instead of mapping fresh memory on the request path
    {
        cudaMemPool_t pool = nullptr;
        PARODE_CUDA(cudaDeviceGetDefaultMemPool(&pool, device_));
        uint64_t keep = (uint64_t)opt_.hbm_budget;
        PARODE_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        // map part of the budget now (the pool keeps it once freed), so the
        // first batches do not pay for growing the pool on the request path
        size_t free_b = 0, total_b = 0;
        PARODE_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const size_t warm = std::min<size_t>({(size_t)opt_.hbm_budget, free_b / 2, opt_.prewarm_bytes});
        if (warm > 0) {
            cudaStream_t st = nullptr;
            PARODE_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            void* p = nullptr;
            if (cudaMallocAsync(&p, warm, st) == cudaSuccess) {
                cudaFreeAsync(p, st);
            } else {
                cudaGetLastError();  // a smaller pool just grows later
            }
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    }
    // pinned staging blocks for the batches' uploads (64 KiB .. 4 MiB, eight
    // of each), so that small batches do not pin memory on the request path
    HostStage::prewarm(8, 22);
    for (int k = 0; k < std::max(1, opt_.setup_threads); ++k) workers_.emplace_back([this] { worker(); });
    PARODE_CUDA(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) retirers_.emplace_back([this] { retirer(); });
    thread_ = std::thread([this] { loop(); });
}

Server::~Server()
{
    {
        std::lock_guard<std::mutex> g(mu_);
        stop_ = true;
        // requests not yet admitted are dropped
        for (auto& r : pending_) {
            r->done = true;
            r->err = kInvalidArgument;
        }
        pending_.clear();
    }
    cv_.notify_all();
    if (thread_.joinable()) thread_.join();  // returns once every admitted batch is retired
    {
        std::lock_guard<std::mutex> g(mu_);
        workers_stop_ = true;
    }
    jobs_cv_.notify_all();
    retire_cv_.notify_all();
    for (auto& w : workers_)
        if (w.joinable()) w.join();
    for (auto& w : retirers_)
        if (w.joinable()) w.join();
    // results nobody collected
    cudaSetDevice(device_);
    for (auto& kv : all_)
        if (kv.second->dy) cudaFreeAsync(kv.second->dy, copy_stream_);
    if (copy_stream_) {
        cudaStreamSynchronize(copy_stream_);
        cudaStreamDestroy(copy_stream_);
    }
}

long long Server::submit(BatchSpec spec)
{
    auto r = std::make_shared<Request>();
    r->bytes = estimate_request_bytes(spec, opt_.precision);
    if (r->bytes == 0) throw Error(kInvalidSystem, "empty time horizon or no states");
    if ((double)r->bytes > opt_.hbm_budget) throw Error(kNotEnoughResources, "request larger than the HBM budget");
    long nScan = 0;
    r->n_out = num_outputs(spec.solver, spec.t0, spec.tEnd, spec.h, &nScan);
    r->channels = spec.sys.out_size();
    r->state_steps = (double)spec.sys.n * (double)r->n_out;
    r->spec = std::move(spec);
    r->t_submit = now_s();
    {
        std::lock_guard<std::mutex> g(mu_);
        if (stop_) throw Error(kInvalidArgument, "server stopped");
        r->id = next_id_++;
        all_[r->id] = r;
        pending_.push_back(r);
        ++st_.submitted;
        if (t_first_ < 0) t_first_ = r->t_submit;
    }
    cv_.notify_all();
    return r->id;
}

int Server::poll(long long id, long long* n_out, int* channels, int* err)
{
    std::lock_guard<std::mutex> g(mu_);
    auto it = all_.find(id);
    if (it == all_.end()) throw Error(kInvalidArgument, "unknown request id");
    const Request& r = *it->second;
    if (n_out) *n_out = r.n_out;
    if (channels) *channels = r.channels;
    if (err) *err = r.err;
    return r.done ? 1 : 0;
}

void Server::result(long long id, double* t, double* y, double* latency_ms)
{
    std::shared_ptr<Request> r;
    {
        std::lock_guard<std::mutex> g(mu_);
        auto it = all_.find(id);
        if (it == all_.end()) throw Error(kInvalidArgument, "unknown request id");
        r = it->second;
        if (!r->done) throw Error(kInvalidArgument, "request not finished");
        all_.erase(it);
    }
    if (r->err != 0) throw Error(r->err, "the request failed");
    if (r->dy) {
        // the outputs wait on the device until collected: one copy into the
        // caller's buffer (pinned memory makes it fastest), then the device
        // memory returns to the pool and to the budget
        PARODE_CUDA(cudaSetDevice(device_));
        if (y) PARODE_CUDA(cudaMemcpyAsync(y, r->dy, sizeof(double) * r->ny, cudaMemcpyDeviceToHost, copy_stream_));
        PARODE_CUDA(cudaFreeAsync(r->dy, copy_stream_));
        r->dy = nullptr;
        PARODE_CUDA(cudaStreamSynchronize(copy_stream_));
        std::lock_guard<std::mutex> g(mu_);
        held_bytes_ -= sizeof(double) * r->ny;
        cv_.notify_all();
    }
    if (t) time_vector(r->spec.solver, r->spec.t0, r->spec.tEnd, r->spec.h, t);
    if (latency_ms) *latency_ms = (r->t_done - r->t_submit) * 1e3;
}

ServerStats Server::stats()
{
    std::lock_guard<std::mutex> g(mu_);
    ServerStats s = st_;
    s.p50_ms = percentile(latencies_, 0.50);
    s.p99_ms = percentile(latencies_, 0.99);
    s.max_ms = latencies_.empty() ? 0.0 : *std::max_element(latencies_.begin(), latencies_.end());
    double sum = 0;
    for (double v : latencies_) sum += v;
    s.mean_ms = latencies_.empty() ? 0.0 : sum / (double)latencies_.size();
    s.span_s = t_first_ >= 0 ? t_last_ - t_first_ : 0.0;
    return s;
}

// Scheduler thread: retire, admit, wait for news.
void Server::loop()
{
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
        for (size_t k = 0; k < inflight_.size();) {
            if (cudaEventQuery(inflight_[k].done) == cudaErrorNotReady) {
                ++k;
                continue;
            }
            // to a copy-out thread; its memory stays counted until it is retired
            inflight_[k].t_seen = now_s();
            retire_q_.push_back(std::move(inflight_[k]));
            inflight_.erase(inflight_.begin() + (long)k);
            retire_cv_.notify_one();
        }
        if (stop_ && pending_.empty() && jobs_.empty() && setting_up_ == 0 && inflight_.empty() &&
            retire_q_.empty() && retiring_ == 0)
            break;
        admit_locked();
        cv_.wait_for(lk, std::chrono::microseconds(inflight_.empty() && setting_up_ == 0 ? 2000 : 50));
    }
}

// Forms batches from the pending requests while the budget and the in-flight
// limit allow (first come, first served; a request that does not fit waits)
// and hands them to the set-up workers.
void Server::admit_locked()
{
    while (!pending_.empty() && (int)inflight_.size() + setting_up_ < opt_.max_inflight) {
        Job j;
        while (!pending_.empty() && (int)j.reqs.size() < opt_.max_batch) {
            const auto& r = pending_.front();
            if ((double)(inflight_bytes_ + held_bytes_ + j.bytes + r->bytes) > opt_.hbm_budget) break;
            j.bytes += r->bytes;
            j.reqs.push_back(r);
            pending_.pop_front();
        }
        if (j.reqs.empty()) break;  // waits for memory to free up
        j.t_admit = now_s();
        inflight_bytes_ += j.bytes;
        st_.peak_bytes = std::max(st_.peak_bytes, (double)(inflight_bytes_ + held_bytes_));
        ++st_.batches;
        ++setting_up_;
        jobs_.push_back(std::move(j));
        jobs_cv_.notify_one();
    }
}

// Set-up worker: builds an admitted batch (host discretisation, arena,
// staged copy) and enqueues its solve on its own stream, concurrently with
// the other workers and with batches already on the device.
void Server::worker()
{
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
        jobs_cv_.wait(lk, [&] { return workers_stop_ || !jobs_.empty(); });
        if (jobs_.empty()) {
            if (workers_stop_) break;
            continue;
        }
        Job j = std::move(jobs_.front());
        jobs_.pop_front();
        lk.unlock();
        Inflight f;
        f.reqs = j.reqs;
        f.bytes = j.bytes;
        f.t_admit = j.t_admit;
        f.t_start = now_s();
        int setup_err = 0;
        try {
            std::vector<BatchSpec> specs;
            specs.reserve(j.reqs.size());
            bool resolved = true;
            for (auto& r : j.reqs) {
                specs.push_back(r->spec);
                const SystemDesc& s = r->spec.sys;
                if ((!s.zeroB || !s.zeroD) && !r->spec.input) resolved = false;
            }
            PlanOptions po;
            po.precision = opt_.precision;
            po.input_double = true;
            po.log = opt_.log >= 2;
            po.discretise = opt_.discretise;
            if (resolved) {
                f.plan = std::make_unique<BatchPlan>(device_, std::move(specs), inputs_, po);
            } else {
                std::lock_guard<std::recursive_mutex> g(*inputs_mu_);  // the input registry is shared
                f.plan = std::make_unique<BatchPlan>(device_, std::move(specs), inputs_, po);
            }
            f.plan->execute(nullptr);
            PARODE_CUDA(cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming));
            PARODE_CUDA(cudaEventRecord(f.done, f.plan->stream()));
            f.t_ready = now_s();
        } catch (const Error& e) {
            setup_err = e.code;
            f.plan.reset();
        } catch (...) {
            setup_err = kDeviceError;
            f.plan.reset();
        }
        lk.lock();
        --setting_up_;
        if (!f.plan) {
            // failed set-up: finish the requests right away (the error is
            // published under the lock, as poll() reads it)
            inflight_bytes_ -= f.bytes;
            const double t = now_s();
            for (auto& r : f.reqs) {
                r->err = setup_err != 0 ? setup_err : kDeviceError;
                r->done = true;
                r->t_done = t;
                ++st_.failed;
            }
        } else {
            inflight_.push_back(std::move(f));
        }
        cv_.notify_all();
    }
}

// Copy-out thread: retires finished batches (several copies in flight at
// once, none on the scheduler thread).
void Server::retirer()
{
    cudaSetDevice(device_);
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) st = nullptr;
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
        retire_cv_.wait(lk, [this] { return !retire_q_.empty() || (workers_stop_ && retire_q_.empty()); });
        if (retire_q_.empty()) {
            if (workers_stop_) {
                lk.unlock();
                if (st) cudaStreamDestroy(st);
                return;
            }
            continue;
        }
        Inflight f = std::move(retire_q_.front());
        retire_q_.pop_front();
        ++retiring_;
        lk.unlock();
        std::vector<Outcome> out;
        retire(f, st, out);
        lk.lock();
        // publish under the lock: poll() and result() read these fields
        for (size_t i = 0; i < f.reqs.size(); ++i) {
            auto& r = f.reqs[i];
            r->err = out[i].err;
            r->dy = out[i].dy;
            r->ny = out[i].ny;
            r->t_done = out[i].t_done;
        }
        if (opt_.log) {
            const double t = now_s(), z = t_first_;
            std::fprintf(stderr,
                         "ParODE server batch (%zu requests): admitted %.1f ms, set-up from %.1f ms, on the device %.1f ms, "
                         "seen done %.1f ms, retired %.1f ms (after the first submission)\n",
                         f.reqs.size(), (f.t_admit - z) * 1e3, (f.t_start - z) * 1e3, (f.t_ready - z) * 1e3,
                         (f.t_seen - z) * 1e3, (t - z) * 1e3);
        }
        --retiring_;
        inflight_bytes_ -= f.bytes;
        for (auto& r : f.reqs)
            if (r->dy) held_bytes_ += sizeof(double) * r->ny;
        for (auto& r : f.reqs) {
            r->done = true;
            if (r->err == 0) {
                latencies_.push_back((r->t_done - r->t_submit) * 1e3);
                ++st_.completed;
                st_.state_steps += r->state_steps;
            } else {
                ++st_.failed;
            }
            t_last_ = std::max(t_last_, r->t_done);
        }
        cv_.notify_all();
    }
}

// Moves every request's outputs into a device buffer of its own (from the
// stream-ordered pool; device to device), checks the batch's device status,
// and frees the batch's arena.
void Server::retire(Inflight& f, cudaStream_t st, std::vector<Outcome>& out)
{
    int err = 0;
    try {
        f.plan->get_output(0, nullptr, nullptr);  // synchronises; throws if a device wait gave up
    } catch (const Error& e) {
        err = e.code;
    }
    out.assign(f.reqs.size(), Outcome());
    for (size_t i = 0; i < f.reqs.size(); ++i) {
        Outcome& o = out[i];
        o.err = err;
        if (err == 0) {
            o.ny = (size_t)f.plan->num_outputs((int)i) * f.plan->channels((int)i);
            if (cudaMallocAsync(reinterpret_cast<void**>(&o.dy), sizeof(double) * std::max<size_t>(o.ny, 1), st) !=
                cudaSuccess) {
                cudaGetLastError();
                o.dy = nullptr;
                o.err = kNotEnoughResources;
            } else if (cudaMemcpyAsync(o.dy, f.plan->device_output((int)i), sizeof(double) * o.ny,
                                       cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
                cudaGetLastError();
                o.err = kDeviceError;
            }
        }
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        for (auto& o : out) o.err = kDeviceError;
    }
    const double t = now_s();
    for (auto& o : out) {
        o.t_done = t;
        if (o.err != 0 && o.dy) {
            cudaFreeAsync(o.dy, st);
            o.dy = nullptr;
        }
    }
    if (f.done) cudaEventDestroy(f.done);
    f.plan.reset();
}

}  // namespace parode
