// batch.cpp -- BatchPlan: set-up on the host (FP64 discretisation, one arena,
// one staged copy), execution as a fixed sequence of batched launches.
#include "batch.h"
#include "tuner.h"

#include "common.h"

#include <algorithm>
#include <map>
#include <mutex>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>

namespace parode {

namespace {

constexpr size_t kAlign = 256;
constexpr size_t kSmemOptIn = 232448 - 1024;
constexpr int kTcConfig = 100;  // grouped launch of the tensor-core (3xTF32) level contraction

size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Byte layout of the arena, built before allocation.
struct Layout {
    size_t bytes = 0;
    size_t take(size_t n)
    {
        size_t off = bytes;
        bytes = align_up(bytes + std::max<size_t>(n, 1));
        return off;
    }
};

double sinusoid_host(const InputEntry* e, int i, double t)
{
    const double two_pi = 6.283185307179586476925286766559;
    double v = 0.0;
    for (int k = 0; k < e->K; ++k) {
        const int q = i * e->K + k;
        v += e->a[q] * std::sin(two_pi * e->f[q] * t + e->phi[q]);
    }
    return v;
}

// A batch discretises on the host threads when no system takes more than
// kHostDiscMaxSystem multiply-adds (RK4 n <= 69, ABM n <= 100: about a
// millisecond on one core) and the batch no more than kHostDiscMaxBatch.
constexpr double kHostDiscMaxSystem = 1e6;
constexpr double kHostDiscMaxBatch = 8e6;

template <class F>
void parallel_for(int n, F&& f)
{
    if (n <= 1) {  // one item: no thread to start (a server's small batches)
        if (n == 1) f(0);
        return;
    }
    int nt = (int)std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 32u);
    nt = std::min(nt, std::max(1, n));
    std::vector<std::thread> th;
    std::vector<std::exception_ptr> err(nt);
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            try {
                for (int i = t; i < n; i += nt) f(i);
            } catch (...) {
                err[t] = std::current_exception();
            }
        });
    for (auto& x : th) x.join();
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
}

// The discretisation of one system on the host, as the device kernel writes
// it (kernels_disc.cu): the compact Phi, Bbar zero-filled to n x W max(m, 1),
// its transpose when asked, and ||Phi - R||_inf over the stored rows (each
// row summed in order), every operation in the kernel's order.
double discretise_host(int solver, int n, int Ns, int W, double h, const SystemDesc& s, double* phi, double* bbar,
                       double* bbarT)
{
    const int mB = s.zeroB ? 0 : s.m, Wm = W * mB;
    std::fill(bbar, bbar + (size_t)n * W * std::max(mB, 1), 0.0);
    if (solver == kRK4) discretise_rk4(n, mB, s.A.data(), mB ? s.B.data() : nullptr, h, phi, bbar);
    else discretise_abm_last(n, mB, s.A.data(), mB ? s.B.data() : nullptr, h, phi, bbar);
    if (bbarT) {
        std::fill(bbarT, bbarT + (size_t)std::max(Wm, 1) * n, 0.0);
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < Wm; ++c) bbarT[(size_t)c * n + r] = bbar[(size_t)r * Wm + c];
    }
    const int d0 = solver == kRK4 ? 0 : 3 * n;
    double dmax = 0.0;
    for (int r = 0; r < n; ++r) {
        double sum = 0.0;
        for (int c = 0; c < Ns; ++c) sum += std::fabs(phi[(size_t)r * Ns + c] + -(c == d0 + r ? 1.0 : 0.0));
        dmax = std::max(dmax, sum);
    }
    return dmax;
}

}  // namespace

// Pinned host blocks for the batches' staged uploads (discretisation
// results or inputs, constants, job tables, response-table arguments), kept
// for the next batch.  From pinned memory an upload is an asynchronous DMA;
// from pageable memory the runtime first waits for the stream's earlier work,
// which would hold a batch's set-up behind its own (and, in a server, other
// batches') kernels.  Blocks come in power-of-two classes from 64 KiB and go
// back to their class; pinning new memory is slow (and serialises the
// driver), so a server pins a few blocks of the small classes when it starts.
// A failed pinning falls back to pageable memory.
namespace {

constexpr int kStageMinLog = 16;

struct PinnedBlocks {
    std::mutex mu;
    std::vector<std::vector<char*>> free = std::vector<std::vector<char*>>(48);
};

PinnedBlocks& pinned_blocks()
{
    static PinnedBlocks* p = new PinnedBlocks();
    return *p;
}

int stage_class(size_t bytes)
{
    int c = kStageMinLog;
    while (((size_t)1 << c) < bytes) ++c;
    return c;
}

}  // namespace

HostStage::HostStage(size_t bytes)
{
    const int c = stage_class(std::max<size_t>(bytes, 1));
    {
        PinnedBlocks& b = pinned_blocks();
        std::lock_guard<std::mutex> g(b.mu);
        if (!b.free[c].empty()) {
            p_ = b.free[c].back();
            b.free[c].pop_back();
            cap_ = (size_t)1 << c;
            pinned_ = true;
            return;
        }
    }
    void* q = nullptr;
    if (cudaHostAlloc(&q, (size_t)1 << c, cudaHostAllocPortable) == cudaSuccess) {
        p_ = static_cast<char*>(q);
        cap_ = (size_t)1 << c;
        pinned_ = true;
        return;
    }
    cudaGetLastError();
    owned_.reset(new char[std::max<size_t>(bytes, 1)]);
    p_ = owned_.get();
    cap_ = bytes;
}

HostStage::~HostStage()
{
    if (!pinned_ || !p_) return;
    PinnedBlocks& b = pinned_blocks();
    std::lock_guard<std::mutex> g(b.mu);
    b.free[stage_class(cap_)].push_back(p_);
}

void HostStage::prewarm(int blocks, int max_log2)
{
    for (int c = kStageMinLog; c <= max_log2; ++c) {
        int have = 0;
        {
            PinnedBlocks& b = pinned_blocks();
            std::lock_guard<std::mutex> g(b.mu);
            have = (int)b.free[c].size();
        }
        for (int k = have; k < blocks; ++k) {
            void* q = nullptr;
            if (cudaHostAlloc(&q, (size_t)1 << c, cudaHostAllocPortable) != cudaSuccess) {
                cudaGetLastError();
                return;
            }
            PinnedBlocks& b = pinned_blocks();
            std::lock_guard<std::mutex> g(b.mu);
            b.free[c].push_back(static_cast<char*>(q));
        }
    }
}

BatchPlan::BatchPlan(int device, std::vector<BatchSpec> specs, InputRegistry* inputs, const PlanOptions& opt)
    : device_(device), inputs_(inputs), opt_(opt)
{
    // a failed set-up gives back what it took (no destructor runs for it)
    try {
        build(std::move(specs), inputs, opt);
    } catch (...) {
        release();
        throw;
    }
}

void BatchPlan::build(std::vector<BatchSpec> specs, InputRegistry* inputs, const PlanOptions& opt)
{
    if (specs.empty()) throw Error(kInvalidArgument, "empty batch");
    if (specs.size() > 65535) throw Error(kInvalidArgument, "at most 65535 systems per batch");
    PARODE_CUDA(cudaSetDevice(device_));
    PARODE_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_));
    const int N = (int)specs.size();
    sys_.resize(N);
    // set-up phase times (PARODE_OPT_LOG)
    auto clock0 = std::chrono::steady_clock::now();
    std::string phases;
    auto phase = [&](const char* name, bool device) {
        if (!opt.log) return;
        if (device && stream_) PARODE_CUDA(cudaStreamSynchronize(stream_));
        const auto now = std::chrono::steady_clock::now();
        char b[64];
        std::snprintf(b, sizeof b, " %s %.1f ms", name, std::chrono::duration<double, std::milli>(now - clock0).count());
        phases += b;
        clock0 = now;
    };

    // ---- classification and sizes ----------------------------------------
    for (int i = 0; i < N; ++i) {
        const BatchSpec& b = specs[i];
        const SystemDesc& s = b.sys;
        Sys& q = sys_[i];
        if (b.solver != kRK4 && b.solver != kABM) throw Error(kInvalidSolverType, "unknown solver type");
        if (s.n <= 0) throw Error(kInvalidSystem, "the system has no states");
        if ((long)s.A.size() < (long)s.n * s.n || (long)s.x0.size() < s.n)
            throw Error(kInvalidSystem, "A or x0 too small");
        if (!s.zeroB && (s.m <= 0 || (long)s.B.size() < (long)s.n * s.m))
            throw Error(kInvalidSystem, "B has the wrong size");
        if (!s.zeroC && (s.p <= 0 || (long)s.C.size() < (long)s.p * s.n))
            throw Error(kInvalidSystem, "C has the wrong size");
        if (!s.zeroD && (s.p <= 0 || s.m <= 0 || (long)s.D.size() < (long)s.p * s.m))
            throw Error(kInvalidSystem, "D has the wrong size");
        q.solver = b.solver;
        q.n = s.n;
        q.m = s.m;
        q.t0 = b.t0;
        q.tEnd = b.tEnd;
        q.h = b.h;
        q.zeroB = s.zeroB;
        q.zeroC = s.zeroC;
        q.zeroD = s.zeroD;
        q.nOut = parode::num_outputs(b.solver, b.t0, b.tEnd, b.h, &q.nScan);
        if (q.nOut <= 0 || q.nScan <= 0) throw Error(kInvalidSystem, "empty time horizon");
        q.p = s.out_size();
        q.mu = (!s.zeroB || !s.zeroD) ? s.m : 0;
        if (q.mu > 0) {
            q.input = b.input ? b.input : (inputs ? inputs->get(b.uIndex) : nullptr);
            if (!q.input) throw Error(kInvalidInput, "uIndex does not name a registered input");
            if (q.input->kind == InputEntry::kSinusoid && q.input->m < q.mu)
                throw Error(kInvalidInput, "the sinusoid input has fewer channels than the system's inputs");
        }
        q.W = b.solver == kRK4 ? 3 : 5;
        q.Ns = b.solver == kRK4 ? s.n : 4 * s.n;
        if (q.solver == kRK4) {
            q.nU = 2 * q.nScan + 1;
            q.u_base = b.t0;
            q.u_dt = 0.5 * b.h;
        } else {
            q.nU = q.nScan + 4;
            q.u_base = (b.t0 + 3.0 * b.h) - 3.0 * b.h;
            q.u_dt = b.h;
        }
        BlockedShape sh;
        const bool can_block = blocked_shape(q.Ns, std::max(q.mu, 1), 0, &sh);
        // block-response leaf for systems with inputs when it costs less than
        // the level-synchronous sweeps (4 Np^2 per step) or, for scan
        // dimensions <= 64, half the in-block sweeps
        if (q.mu > 0 && opt.path != kPathLevel && opt.path != kPathBlockedSweep) {
            const int np = (int)round_up(q.Ns, 8);
            double cost = 0.0;
            // mixed: the window and aggregate products run on the tensor cores
            const double wweight = opt.precision == kMixed ? 0.25 : 1.0;
            int R = response_log2_block(q.solver, np, q.n, q.mu, q.p, q.nScan, wweight, opt.executions, &cost);
            // a block length forced by the caller or measured for this class of
            // systems (tuner.h) replaces the cost model's
            int Rt = opt.force_log2_block;
            if (Rt < 2) Rt = tuned_log2_block(tune_class(q.solver, q.Ns, q.mu, q.p, q.nScan, opt.precision));
            if (Rt >= 2 && Rt <= 7) {
                while (Rt > 2 && (1L << Rt) / 2 >= q.nScan) --Rt;
                R = Rt;
            }
            const double sweeps = 4.0 * np * np;
            // a blocked bucket chains its tiles one after another: long
            // horizons go to the response leaf's level-synchronous block scan
            const bool long_chain = can_block && q.nScan >= (1L << 15);
            if (opt.path == kPathBlockedResponse || long_chain || cost < (can_block ? 0.5 : 1.0) * sweeps) {
                if (np > 1024) throw Error(kInvalidSystem, "scan dimension above 1024 is not supported");
                q.resp = true;
                q.Np = np;
                q.lev0 = R;
                q.Bk = 1 << R;
                q.Kw = response_window(q.solver, q.Bk, q.mu);
                q.Kpad = (q.Kw + 1) & ~1;
                q.nblocks = (q.nScan + q.Bk - 1) / q.Bk;
                q.Tp = next_pow2(q.nblocks);
                q.levels = ilog2(q.Tp);
                q.pow_levels = R + q.levels;  // P_0 .. P_{R-1} also double W's tables
                rs_.push_back(i);
            }
        }
        q.blocked = !q.resp && opt.path != kPathLevel && can_block;
        if (q.resp) {
        } else if (q.blocked) {
            q.Np = sh.NP;
            int bi = -1;
            for (int k = 0; k < (int)buckets_.size(); ++k)
                if (buckets_[k].sh.NP == q.Np) bi = k;
            if (bi < 0) {
                buckets_.emplace_back();
                bi = (int)buckets_.size() - 1;
                buckets_[bi].sh.NP = q.Np;
            }
            q.bucket = bi;
            buckets_[bi].systems.push_back(i);
            buckets_[bi].ms = std::max(buckets_[bi].ms, q.mu);
            buckets_[bi].pmax = std::max(buckets_[bi].pmax, q.p);
        } else {
            q.Np = (int)round_up(q.Ns, 8);
            if (q.Np > 1024) throw Error(kInvalidSystem, "scan dimension above 1024 is not supported");
            q.Tp = next_pow2(q.nScan);
            q.levels = ilog2(q.Tp);
            q.pow_levels = q.levels;
            ls_.push_back(i);
        }
        // mixed form: level-synchronous scans (over steps or over response
        // blocks) run their lower levels on the tensor cores; the blocked
        // buckets stay FP64 here
        q.precision = (opt.precision == kMixed && !q.blocked) ? kMixed : kFP64;
    }
    // bucket shapes: the widest input of the bucket sizes the sample staging
    for (Bucket& bk : buckets_) {
        if (!blocked_shape(bk.sh.NP, std::max(bk.ms, 1), 0, &bk.sh))
            throw Error(kInvalidArgument, "blocked shape for the batch");
        long stage = 0;
        for (int i : bk.systems) {
            const Sys& q = sys_[i];
            stage = std::max<long>(stage, (long)q.n * q.W * q.m + (long)q.p * q.n + (long)q.p * q.m);
        }
        bk.stage = batch_leaf_smem(bk.sh, bk.ms, stage) <= kSmemOptIn;
        bk.leaf_smem = batch_leaf_smem(bk.sh, bk.ms, bk.stage ? stage : 0);
        for (int i : bk.systems) {
            Sys& q = sys_[i];
            q.ntiles = (q.nScan + bk.sh.S - 1) / bk.sh.S;
            bk.max_blocks = std::max(bk.max_blocks, q.ntiles * (bk.sh.S / bk.sh.B));
        }
    }

    phase("classify", false);
    // ---- discretisation: the compact Phi (RK4: n x n; ABM: its last block
    // row, n x 4n, the rows above being the exact shift; expanded into the
    // padded power table's level 0 later), Bbar (and its transpose for the
    // level-synchronous systems) into the batch's discretisation buffer, and
    // each system's distance ||Phi - R|| (it sizes the tensor-core levels of
    // the layout below).  Host and device take every operation in the same
    // order (host_math.cpp, kernels_disc.cu): the same bits either way.  A
    // batch of small systems runs it on the host threads, with no device round
    // trip (a server sets batches up while others run); a large one on the
    // device.
    PARODE_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    struct DiscOff {
        size_t A, B, phi, bbar, bbarT, work;
    };
    std::vector<DiscOff> doff(N);
    double disc_total = 0.0, disc_max = 0.0;  // multiply-adds of the discretisation GEMMs
    for (int i = 0; i < N; ++i) {
        const Sys& q = sys_[i];
        const double n = q.n, mB = specs[i].sys.zeroB ? 0 : q.m;
        const double c = q.solver == kRK4 ? 3.0 * n * n * (n + mB) : n * n * (n + mB);
        disc_total += c;
        disc_max = std::max(disc_max, c);
    }
    const bool disc_host = opt.discretise == kDiscHost || (opt.discretise == kDiscAuto &&
                                                            disc_max <= kHostDiscMaxSystem &&
                                                            disc_total <= kHostDiscMaxBatch);
    // the device discretisation runs while the host sets up the constants and
    // the ABM start-up; its distances are read just before the layout needs
    // them (its stream, staged inputs and pinned readback live until then; the
    // guard waits for the stream before they go, also when a step fails)
    cudaStream_t dstream = nullptr;
    std::unique_ptr<HostStage> dstage, ddelta;
    struct StreamGuard {
        cudaStream_t* s;
        ~StreamGuard()
        {
            if (*s) {
                cudaStreamSynchronize(*s);
                cudaStreamDestroy(*s);
            }
        }
    } dguard{&dstream};
    if (disc_host) {
        Layout D;
        for (int i = 0; i < N; ++i) {
            const Sys& q = sys_[i];
            const int mB = specs[i].sys.zeroB ? 0 : q.m;
            doff[i].phi = D.take(sizeof(double) * (size_t)q.n * q.Ns);
            doff[i].bbar = D.take(sizeof(double) * (size_t)q.n * q.W * std::max(mB, 1));
            doff[i].bbarT = (!q.blocked && !q.resp) ? D.take(sizeof(double) * (size_t)std::max(q.W * mB, 1) * q.n) : 0;
        }
        if (fault_alloc_now()) throw Error(kNotEnoughResources, "batch discretisation buffer (injected)");
        cudaError_t e = cudaMallocAsync(&disc_, std::max<size_t>(D.bytes, 8), stream_);
        if (e != cudaSuccess) {
            cudaGetLastError();
            disc_ = nullptr;
            throw Error(kNotEnoughResources, "batch discretisation buffer allocation failed");
        }
        host_disc_ = std::make_unique<HostStage>(D.bytes);  // kept with the plan: the copy is asynchronous
        char* hd = host_disc_->data();
        parallel_for(N, [&](int i) {
            const Sys& q = sys_[i];
            sys_[i].delta = discretise_host(q.solver, q.n, q.Ns, q.W, q.h, specs[i].sys,
                                            reinterpret_cast<double*>(hd + doff[i].phi),
                                            reinterpret_cast<double*>(hd + doff[i].bbar),
                                            doff[i].bbarT ? reinterpret_cast<double*>(hd + doff[i].bbarT) : nullptr);
        });
        PARODE_CUDA(cudaMemcpyAsync(disc_, hd, D.bytes, cudaMemcpyHostToDevice, stream_));
    } else {
        // A and B go up, the kernel fills the buffer and the distances come
        // back.  The set-up waits for it, so it runs on a stream of the
        // greatest priority: a batch set up while others execute is not
        // queued behind their kernels.
        {
            int least = 0, greatest = 0;
            PARODE_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
            PARODE_CUDA(cudaStreamCreateWithPriority(&dstream, cudaStreamNonBlocking, greatest));
        }
        Layout D;
        for (int i = 0; i < N; ++i) {  // staged inputs first
            const SystemDesc& s = specs[i].sys;
            const int mB = s.zeroB ? 0 : s.m;
            doff[i].A = D.take(sizeof(double) * (size_t)sys_[i].n * sys_[i].n);
            doff[i].B = mB ? D.take(sizeof(double) * (size_t)sys_[i].n * mB) : 0;
        }
        const size_t jobs_at = D.take(sizeof(DiscJob) * (size_t)N);
        // the product tiles of the three stages (32 x 32 outputs each)
        long ntiles[3] = {0, 0, 0};
        for (int i = 0; i < N; ++i) {
            const Sys& q = sys_[i];
            const int mB = specs[i].sys.zeroB ? 0 : q.m;
            const long tn = (q.n + 31) / 32, tm = mB > 0 ? (mB + 31) / 32 : 0;
            for (int st = 0; st < (q.solver == kRK4 ? 3 : 1); ++st) ntiles[st] += tn * tn + tn * tm;
        }
        size_t tiles_at[3];
        for (int st = 0; st < 3; ++st) tiles_at[st] = D.take(sizeof(DiscTile) * (size_t)std::max<long>(ntiles[st], 1));
        const size_t staged = D.bytes;
        const size_t delta_at = D.take(sizeof(double) * (size_t)N);
        for (int i = 0; i < N; ++i) {
            const SystemDesc& s = specs[i].sys;
            const Sys& q = sys_[i];
            const int mB = s.zeroB ? 0 : s.m;
            doff[i].phi = D.take(sizeof(double) * (size_t)q.n * q.Ns);
            doff[i].bbar = D.take(sizeof(double) * (size_t)q.n * q.W * std::max(mB, 1));
            doff[i].bbarT = (!q.blocked && !q.resp) ? D.take(sizeof(double) * (size_t)std::max(q.W * mB, 1) * q.n) : 0;
            doff[i].work = D.take(sizeof(double) * (size_t)discretise_work_doubles(q.n, mB));
        }
        if (fault_alloc_now()) throw Error(kNotEnoughResources, "batch discretisation buffer (injected)");
        cudaError_t e = cudaMallocAsync(&disc_, std::max<size_t>(D.bytes, 8), dstream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            disc_ = nullptr;
            throw Error(kNotEnoughResources, "batch discretisation buffer allocation failed");
        }
        char* db = static_cast<char*>(disc_);
        dstage = std::make_unique<HostStage>(staged);  // gaps are copied, never read
        char* hs_data = dstage->data();
        std::vector<DiscJob> jobs(N);
        parallel_for(N, [&](int i) {
            const SystemDesc& s = specs[i].sys;
            const Sys& q = sys_[i];
            const int mB = s.zeroB ? 0 : s.m;
            std::memcpy(hs_data + doff[i].A, s.A.data(), sizeof(double) * (size_t)q.n * q.n);
            if (mB) std::memcpy(hs_data + doff[i].B, s.B.data(), sizeof(double) * (size_t)q.n * mB);
            DiscJob& j = jobs[i];
            j.A = reinterpret_cast<const double*>(db + doff[i].A);
            j.B = mB ? reinterpret_cast<const double*>(db + doff[i].B) : nullptr;
            j.phi = reinterpret_cast<double*>(db + doff[i].phi);
            j.bbar = reinterpret_cast<double*>(db + doff[i].bbar);
            j.bbarT = doff[i].bbarT ? reinterpret_cast<double*>(db + doff[i].bbarT) : nullptr;
            j.work = reinterpret_cast<double*>(db + doff[i].work);
            j.delta = reinterpret_cast<double*>(db + delta_at) + i;
            j.n = q.n;
            j.m = mB;
            j.solver = q.solver;
            j.h = q.h;
        });
        std::memcpy(hs_data + jobs_at, jobs.data(), sizeof(DiscJob) * (size_t)N);
        const DiscTile* dtiles[3];
        for (int st = 0; st < 3; ++st) {
            std::vector<DiscTile> tl;
            tl.reserve((size_t)ntiles[st]);
            for (int i = 0; i < N; ++i) discretise_tiles(jobs[i], st, tl);
            if ((long)tl.size() != ntiles[st]) throw Error(kDeviceError, "discretisation tiles: count mismatch");
            std::memcpy(hs_data + tiles_at[st], tl.data(), sizeof(DiscTile) * tl.size());
            dtiles[st] = reinterpret_cast<const DiscTile*>(db + tiles_at[st]);
        }
        PARODE_CUDA(cudaMemcpyAsync(db, hs_data, staged, cudaMemcpyHostToDevice, dstream));
        launch_discretise_batch(reinterpret_cast<const DiscJob*>(db + jobs_at), N, dtiles, ntiles, sms_, dstream);
        ddelta = std::make_unique<HostStage>(sizeof(double) * (size_t)N);
        PARODE_CUDA(cudaMemcpyAsync(ddelta->data(), db + delta_at, sizeof(double) * (size_t)N, cudaMemcpyDeviceToHost,
                                    dstream));
        }
    phase(disc_host ? "discretise (host)" : "discretise (device)", false);
    // ---- constant region: layout first, then the host set-up (threads over
    // systems) writes straight into its staged slots
    Layout L;
    struct Off {
        size_t c, d, cext, x0, sin, ypre;
        size_t cT, dT;  // level-synchronous systems: transposed copies (coalesced per-row kernels)
        size_t P, U, Y, V, G, CP, Ps, W, Psa, Psw;
    };
    std::vector<Off> off(N);
    for (int i = 0; i < N; ++i) {
        const SystemDesc& s = specs[i].sys;
        Sys& q = sys_[i];
        Off& o = off[i];
        o.c = L.take(sizeof(double) * (s.zeroC ? 1 : (size_t)q.p * q.n));
        o.d = L.take(sizeof(double) * (s.zeroD ? 1 : (size_t)q.p * s.m));
        o.x0 = L.take(sizeof(double) * (size_t)q.Np);
        o.cext = (q.blocked || q.resp) ? L.take(sizeof(double) * (size_t)q.p * q.Np) : 0;
        o.sin = 0;
        if (q.mu > 0 && q.input->kind == InputEntry::kSinusoid) {
            q.K = q.input->K;
            o.sin = L.take(sizeof(double) * 3 * q.input->a.size());
        }
        o.ypre = q.solver == kABM ? L.take(sizeof(double) * 3 * (size_t)q.p) : 0;
        o.cT = o.dT = 0;
        if (!q.blocked && !q.resp) {
            o.cT = L.take(sizeof(double) * (size_t)q.n * q.p);
            o.dT = L.take(sizeof(double) * (size_t)std::max(s.m, 1) * q.p);
        }
    }
    // uninitialised: every slot is written below (the alignment gaps are
    // copied but never read)
    auto stage = std::make_unique<HostStage>(L.bytes);
    auto slot = [&](size_t o) { return reinterpret_cast<double*>(stage->data() + o); };
    parallel_for(N, [&](int i) {
        const SystemDesc& s = specs[i].sys;
        Sys& q = sys_[i];
        const Off& o = off[i];
        if (s.zeroC) slot(o.c)[0] = 0.0;
        else std::memcpy(slot(o.c), s.C.data(), sizeof(double) * (size_t)q.p * q.n);
        if (s.zeroD) slot(o.d)[0] = 0.0;
        else std::memcpy(slot(o.d), s.D.data(), sizeof(double) * (size_t)q.p * s.m);
        double* x0 = slot(o.x0);
        std::fill(x0, x0 + q.Np, 0.0);
        if (q.solver == kRK4)
            for (int r = 0; r < q.n; ++r) x0[r] = s.x0[r];  // ABM: the start-up below
        if (q.blocked || q.resp) {
            double* cext = slot(o.cext);
            std::fill(cext, cext + (size_t)q.p * q.Np, 0.0);
            const int xoff = q.solver == kRK4 ? 0 : 3 * q.n;
            for (int r = 0; r < q.p; ++r)
                for (int c = 0; c < q.n; ++c) {
                    double v = 0.0;
                    if (!s.zeroC) v = s.C[(size_t)r * q.n + c];
                    else if (s.zeroD) v = (r == c) ? 1.0 : 0.0;
                    cext[(size_t)r * q.Np + xoff + c] = v;
                }
        }
        if (o.sin) {
            const InputEntry* e = q.input;
            double* prm = slot(o.sin);
            const size_t na = e->a.size();
            std::memcpy(prm, e->a.data(), sizeof(double) * na);
            std::memcpy(prm + na, e->f.data(), sizeof(double) * na);
            std::memcpy(prm + 2 * na, e->phi.data(), sizeof(double) * na);
        }
        if (!q.blocked && !q.resp) {
            double* ct = slot(o.cT);
            double* dt = slot(o.dT);
            std::fill(ct, ct + (size_t)q.n * q.p, 0.0);
            std::fill(dt, dt + (size_t)std::max(s.m, 1) * q.p, 0.0);
            if (!s.zeroC)
                for (int r = 0; r < q.p; ++r)
                    for (int c = 0; c < q.n; ++c) ct[(size_t)c * q.p + r] = s.C[(size_t)r * q.n + c];
            if (!s.zeroD)
                for (int r = 0; r < q.p; ++r)
                    for (int c = 0; c < s.m; ++c) dt[(size_t)c * q.p + r] = s.D[(size_t)r * s.m + c];
        }
    });
    phase("host constants", false);
    // ABM start-up: nine inputs at t0 + j h/2 (sinusoids on the host; user
    // functions through their compiled kernel, sampled first on this thread);
    // the four states into x0, the outputs 0..2 into their slot (threads over
    // systems)
    std::vector<std::vector<double>> U9s(N);
    for (int i = 0; i < N; ++i) {
        Sys& q = sys_[i];
        if (q.solver != kABM) continue;
        const SystemDesc& s = specs[i].sys;
        std::vector<double>& U9 = U9s[i];
        U9.assign((size_t)9 * std::max(s.m, 1), 0.0);
        if (q.mu > 0 && q.input->kind != InputEntry::kSinusoid) {
            double* dU9 = nullptr;
            PARODE_CUDA(cudaMalloc(&dU9, sizeof(double) * 9 * q.mu));
            std::unique_ptr<double, decltype(&cudaFree)> keep(dU9, &cudaFree);
            inputs_->fill(q.input, device_, dU9, q.mu, q.t0, 0.5 * q.h, 9, opt_.input_double, nullptr);
            PARODE_CUDA(cudaMemcpy(U9.data(), dU9, sizeof(double) * 9 * q.mu, cudaMemcpyDeviceToHost));
        }
    }
    parallel_for(N, [&](int i) {
        Sys& q = sys_[i];
        if (q.solver != kABM) return;
        const SystemDesc& s = specs[i].sys;
        std::vector<double>& U9 = U9s[i];
        if (q.mu > 0 && q.input->kind == InputEntry::kSinusoid)
            for (int j = 0; j < 9; ++j)
                for (int c = 0; c < q.mu; ++c) U9[(size_t)j * q.mu + c] = sinusoid_host(q.input, c, q.t0 + j * 0.5 * q.h);
        SystemDesc s0 = s;
        if (s0.zeroB) s0.m = 0;
        double* x0 = slot(off[i].x0);
        abm_startup(s0, U9.data(), q.h, x0);  // the first 4 n of the Np slots
        double* ypre = slot(off[i].ypre);
        for (int k = 0; k < 3; ++k) {
            const double* x = x0 + (size_t)k * q.n;
            const double* u = &U9[(size_t)(2 * k) * std::max(s.m, 1)];
            for (int o = 0; o < q.p; ++o) {
                double v = 0.0;
                if (s.zeroC && s.zeroD) {
                    v = x[o];
                } else {
                    if (!s.zeroC)
                        for (int c = 0; c < q.n; ++c) v += s.C[(size_t)o * q.n + c] * x[c];
                    if (!s.zeroD)
                        for (int c = 0; c < s.m; ++c) v += s.D[(size_t)o * s.m + c] * u[c];
                }
                ypre[(size_t)k * q.p + o] = v;
            }
        }
    });
    phase("abm-start-up", false);
    if (dstream) {
        PARODE_CUDA(cudaStreamSynchronize(dstream));
        const double* dl = reinterpret_cast<const double*>(ddelta->data());
        for (int i = 0; i < N; ++i) sys_[i].delta = dl[i];
        phase("distances", false);
    }
    const size_t const_end = L.bytes;
    // work buffers (offsets only; not staged); per-kind totals for the log
    size_t kind_bytes[5] = {0, 0, 0, 0, 0};  // power tables + scan vectors, W, W split, samples, outputs
    for (int i = 0; i < N; ++i) {
        const size_t at0 = L.bytes;
        Sys& q = sys_[i];
        Off& o = off[i];
        if (q.blocked) {
            const Bucket& bk = buckets_[q.bucket];
            o.P = L.take(sizeof(double) * (size_t)(bk.sh.R + 1) * q.Np * q.Np);
            o.G = L.take(sizeof(double) * (size_t)q.ntiles * (bk.sh.S / bk.sh.B) * q.Np);
            o.CP = L.take(sizeof(double) * (size_t)bk.sh.B * q.p * q.Np);
        } else {
            o.P = L.take(sizeof(double) * (size_t)std::max(q.pow_levels, 1) * q.Np * q.Np);
            o.V = L.take(sizeof(double) * (size_t)(q.Tp + 1) * q.Np);  // slot -1 holds the initial state
            // mixed: tensor cores for the scan levels below the top four whose
            // P - R stays small (|P_l - R_l| <~ 2^l |Phi - R|: at most 1/4);
            // the rest, and the power table, stay FP64
            if (q.precision == kMixed) {
                int lv = 0;
                while (lv < q.levels - 4 && std::ldexp(q.delta, q.lev0 + lv) <= 0.25) ++lv;
                q.tc_levels = lv;
            }
            o.Ps = q.tc_levels > 0 ? L.take(level_split_bytes(q.Np) * (size_t)q.tc_levels) : 0;
            const size_t at1 = L.bytes;
            if (q.resp) o.W = L.take(sizeof(double) * ((size_t)q.Bk * q.p + q.Np) * ((size_t)q.Kpad + q.Np));
            const size_t at2 = L.bytes;
            if (q.resp && q.precision == kMixed) {
                q.resp_tc = true;
                o.Psa = L.take(gemm_split_bytes(q.Np, q.Kw));
                o.Psw = L.take(gemm_split_bytes(q.Bk * q.p, q.Kw));
            }
            kind_bytes[1] += at2 - at1;
            kind_bytes[2] += L.bytes - at2;
            kind_bytes[0] -= L.bytes - at1;
        }
        // the response GEMMs read whole sample windows: the last block's
        // window runs past the samples into a zero padding
        const size_t upad = q.resp ? (size_t)(2 * q.Bk + 8) * q.mu + 2 : 0;
        const size_t at3 = L.bytes;
        o.U = q.mu > 0 ? L.take(sizeof(double) * ((size_t)q.nU * q.mu + upad)) : 0;
        const size_t at4 = L.bytes;
        o.Y = L.take(sizeof(double) * (size_t)q.nOut * q.p);
        kind_bytes[0] += at3 - at0;
        kind_bytes[3] += at4 - at3;
        kind_bytes[4] += L.bytes - at4;
    }
    const size_t work_end = L.bytes;

    // job arrays go after the work region, staged; their pointers are
    // computed from the arena base, so allocate first
    arena_bytes_ = work_end;  // grows below
    // pre-compute the job array sizes to reserve space
    size_t job_bytes = 0;
    {
        size_t nb = 0;
        for (Bucket& bk : buckets_) {
            long tiles = 0;
            for (int i : bk.systems) tiles += sys_[i].ntiles;
            (void)tiles;
            nb += bk.systems.size();
        }
        // upper bounds: LeafArgs + 3 pointer arrays per blocked system, items
        // (<= tiles), jobs and level args per LS system and level
        long items_ub = 0;
        for (Bucket& bk : buckets_)
            for (int i : bk.systems) items_ub += sys_[i].ntiles;
        long lev_entries = 0;
        for (int i : ls_) lev_entries += 4L * std::max(sys_[i].levels, 1);
        for (int i : rs_) lev_entries += 4L * std::max(sys_[i].pow_levels, 1) + 8;
        job_bytes = nb * (sizeof(LeafArgs) + 3 * sizeof(double*) + 4 * kAlign) +
                    (size_t)items_ub * sizeof(BatchItem) + buckets_.size() * 8 * kAlign +
                    (size_t)N * (sizeof(SampleJob) + sizeof(ForcingJob) + sizeof(OutputJob) + 2 * sizeof(CopyJob) + sizeof(PhiJob)) +
                    8 * kAlign + (size_t)lev_entries * (2 * sizeof(LevelArgs) + sizeof(long) + 128) +
                    (size_t)(3 * 64 * 8) * 2 * kAlign + (size_t)2 * 64 * (2 * sms_ + 1) * sizeof(long) +
                    ((size_t)1 << 20);
    }
    arena_bytes_ = align_up(work_end + job_bytes);
    phase("layout", false);
    // keep the arena and the response tables' workspace (at most 1 GiB per
    // group) in the pool once freed: the workspace groups then reuse one
    // mapping, and the next batch of this size maps nothing new
    {
        cudaMemPool_t pool = nullptr;
        PARODE_CUDA(cudaDeviceGetDefaultMemPool(&pool, device_));
        uint64_t keep = 0;
        PARODE_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        uint64_t want = (uint64_t)arena_bytes_ + (rs_.empty() ? 0 : ((uint64_t)5 << 29));
        if (keep < want) PARODE_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &want));
    }
    {
        // stream-ordered: creating or destroying a batch does not synchronise
        // the device, so batches can come and go while others run
        if (fault_alloc_now()) throw Error(kNotEnoughResources, "batch arena allocation failed (injected)");
        cudaError_t e = cudaMallocAsync(&arena_, arena_bytes_, stream_);
        if (e != cudaSuccess) {
            cudaGetLastError();
            arena_ = nullptr;
            throw Error(kNotEnoughResources, "batch arena allocation failed");
        }
    }
    char* base = static_cast<char*>(arena_);
    auto dp = [&](size_t o) { return reinterpret_cast<double*>(base + o); };
    for (int i = 0; i < N; ++i) {
        Sys& q = sys_[i];
        const Off& o = off[i];
        q.P = dp(o.P);
        q.Bbar = reinterpret_cast<double*>(static_cast<char*>(disc_) + doff[i].bbar);
        q.C = dp(o.c);
        q.D = dp(o.d);
        q.X0 = dp(o.x0);
        q.Y = dp(o.Y);
        q.U = q.mu > 0 ? dp(o.U) : nullptr;
        if (q.blocked) {
            q.G = dp(o.G);
            q.CP = dp(o.CP);
            q.Cext = dp(o.cext);
        } else {
            q.V = dp(o.V);
            if (q.tc_levels > 0) q.Ps = reinterpret_cast<float*>(base + o.Ps);
            if (q.resp) {
                q.Cext = dp(o.cext);
                q.Wm = dp(o.W);
            }
            if (q.resp_tc) {
                q.Psa = reinterpret_cast<float*>(base + o.Psa);
                q.Psw = reinterpret_cast<float*>(base + o.Psw);
            }
        }
        if (q.mu > 0 && q.input->kind == InputEntry::kSinusoid) q.sin = dp(o.sin);
    }

    phase("arena", true);
    // ---- job arrays (staged after the work region) ----------------------------
    Layout J;
    J.bytes = work_end;
    // sized by the reservation (uninitialised: the alignment gaps are copied,
    // never read); a job array past it is an error below
    auto jstage = std::make_unique<HostStage>(arena_bytes_ - work_end);
    auto jput = [&](const void* src, size_t n) {
        size_t at = J.take(n);
        if (J.bytes > arena_bytes_) throw Error(kDeviceError, "batch job arrays overflow the arena reservation");
        std::memcpy(jstage->data() + (at - work_end), src, n);
        return at;
    };
    std::vector<CopyJob> setup_copies;
    for (Bucket& bk : buckets_) {
        std::vector<LeafArgs> la;
        std::vector<double*> cps;
        std::vector<const double*> cexts, x0s;
        std::vector<BatchItem> items;
        long total_tiles = 0;
        for (int i : bk.systems) total_tiles += sys_[i].ntiles;
        const long target_items = 4L * sms_;
        const long chunk = std::max<long>(1, (total_tiles + target_items - 1) / target_items);
        for (int k = 0; k < (int)bk.systems.size(); ++k) {
            const Sys& q = sys_[bk.systems[k]];
            LeafArgs a;
            a.solver = q.solver;
            a.n = q.n;
            a.m = q.mu;
            a.p = q.p;
            a.zeroB = q.zeroB;
            a.zeroC = q.zeroC;
            a.zeroD = q.zeroD;
            a.nScan = q.nScan;
            a.ntiles = q.ntiles;
            a.ybase = q.solver == kRK4 ? 0 : 3;
            a.P = q.P;
            a.Bbar = q.Bbar;
            a.C = q.C;
            a.D = q.D;
            a.U = q.U;
            a.gen = 0;
            a.stage = bk.stage ? 1 : 0;
            a.Y = q.Y;
            a.G = q.G;
            la.push_back(a);
            cps.push_back(q.CP);
            cexts.push_back(q.Cext);
            x0s.push_back(q.X0);
            for (long t = 0; t < q.ntiles; t += chunk) {
                BatchItem it;
                it.sys = k;
                it.t0 = t;
                it.t1 = std::min(q.ntiles, t + chunk);
                items.push_back(it);
            }
        }
        std::stable_sort(items.begin(), items.end(),
                         [](const BatchItem& x, const BatchItem& y) { return (x.t1 - x.t0) > (y.t1 - y.t0); });
        BatchLaunch& b = bk.launch;
        b.nsys = (int)la.size();
        b.nitems = (int)items.size();
        b.grid = (int)std::min<long>(b.nitems, sms_);
        b.ms = bk.ms;
        b.leaf_smem = bk.leaf_smem;
        b.max_blocks = bk.max_blocks;
        b.pmax = bk.pmax;
        b.sys = reinterpret_cast<const LeafArgs*>(base + jput(la.data(), sizeof(LeafArgs) * la.size()));
        b.items = reinterpret_cast<const BatchItem*>(base + jput(items.data(), sizeof(BatchItem) * items.size()));
        b.CPs = reinterpret_cast<double* const*>(base + jput(cps.data(), sizeof(double*) * cps.size()));
        b.Cexts = reinterpret_cast<const double* const*>(base + jput(cexts.data(), sizeof(double*) * cexts.size()));
        b.X0s = reinterpret_cast<const double* const*>(base + jput(x0s.data(), sizeof(double*) * x0s.size()));
    }
    phase("jobs/buckets", false);
    // input samples
    {
        std::vector<SampleJob> sj;
        for (int i = 0; i < N; ++i) {
            const Sys& q = sys_[i];
            if (q.mu <= 0) continue;
            if (q.input->kind != InputEntry::kSinusoid) {
                user_inputs_.push_back(i);
                continue;
            }
            SampleJob j;
            j.U = q.U;
            j.m = q.mu;
            j.K = q.K;
            const int mi = q.input->m;
            j.a = q.sin;
            j.f = q.sin + (long)mi * q.K;
            j.phi = q.sin + 2L * mi * q.K;
            j.base = q.u_base;
            j.dt = q.u_dt;
            j.count = q.nU;
            maxSample_ = std::max(maxSample_, (q.nU + kSampleRun - 1) / kSampleRun * q.mu);  // threads: runs x channels
            maxTerms_ = std::max(maxTerms_, q.K);
            sj.push_back(j);
        }
        nSampleJobs_ = (int)sj.size();
        if (nSampleJobs_)
            dSampleJobs_ = reinterpret_cast<SampleJob*>(base + jput(sj.data(), sizeof(SampleJob) * sj.size()));
    }
    // level-synchronous systems: forcing, seed, output jobs and the grouped
    // levels; response systems: their GEMMs, seed and block-scan levels
    std::vector<int> lv = ls_;
    lv.insert(lv.end(), rs_.begin(), rs_.end());
    if (!lv.empty()) {
        std::vector<ForcingJob> fj;
        std::vector<OutputJob> oj;
        std::vector<CopyJob> cj;
        int Lmax = 0, Pmax = 0;
        for (int i : rs_) {
            const Sys& q = sys_[i];
            CopyJob c;
            c.dst = q.V;
            c.src = q.X0;
            c.N = q.Np;
            cj.push_back(c);
            maxSeed_ = std::max<long>(maxSeed_, q.Np);
            Lmax = std::max(Lmax, q.levels);
            Pmax = std::max(Pmax, q.pow_levels);
        }
        for (int i : ls_) {
            const Sys& q = sys_[i];
            ForcingJob f;
            f.V = q.V + q.Np;
            f.Np = q.Np;
            f.n = q.n;
            f.m = q.zeroB ? 0 : q.m;
            f.solver = q.solver;
            f.BbarT = reinterpret_cast<double*>(static_cast<char*>(disc_) + doff[i].bbarT);
            f.U = q.U;
            f.T = q.nScan;
            f.Tp = q.Tp;
            fj.push_back(f);
            maxForcing_ = std::max(maxForcing_, q.Tp * (long)q.Np);
            OutputJob o;
            o.Y = q.Y;
            o.V = q.V;
            o.Np = q.Np;
            o.xoff = q.solver == kRK4 ? 0 : 3 * q.n;
            o.n = q.n;
            o.m = q.mu;
            o.p = q.p;
            o.CT = dp(off[i].cT);
            o.DT = dp(off[i].dT);
            o.zeroC = q.zeroC;
            o.zeroD = q.zeroD;
            o.U = q.U;
            o.ustride = q.solver == kRK4 ? 2 : 1;
            o.uoff = q.solver == kRK4 ? 0 : 3;
            o.count = q.nScan;
            o.ybase = q.solver == kRK4 ? 0 : 3;
            oj.push_back(o);
            maxOutput_ = std::max(maxOutput_, q.nScan * (long)q.p);
            CopyJob c;
            c.dst = q.V;
            c.src = q.X0;
            c.N = q.Np;
            cj.push_back(c);
            maxSeed_ = std::max<long>(maxSeed_, q.Np);
            Lmax = std::max(Lmax, q.levels);
            Pmax = std::max(Pmax, q.pow_levels);
        }
        if (!fj.empty()) {
            dForcing_ = reinterpret_cast<ForcingJob*>(base + jput(fj.data(), sizeof(ForcingJob) * fj.size()));
            dOutput_ = reinterpret_cast<OutputJob*>(base + jput(oj.data(), sizeof(OutputJob) * oj.size()));
        }
        dSeed_ = reinterpret_cast<CopyJob*>(base + jput(cj.data(), sizeof(CopyJob) * cj.size()));
        nSeed_ = (int)cj.size();
        // grouped level launches: for each level, entries grouped by tiling config
        // one persistent tensor-core launch over the entries' tiles
        // A level's launches in two steps: prepare (grouping by tiling
        // configuration, tile prefix sums, tensor maps; no shared state, so
        // the levels are prepared on all host threads) and emit (their arrays
        // appended to the staged job tables, in launch order)
        struct PreparedGroup {
            LevelConfig cfg;
            std::vector<LevelArgs> stored, swaps;
            std::vector<long> start;
            long tiles = 0, swap_elems = 0;
            size_t smem = 0;
        };
        struct PreparedLevel {
            std::vector<PreparedGroup> groups;
            std::vector<LevelArgs> tc;
            std::vector<unsigned char> maps;
            std::vector<long> tc_start, tc_ranges;
            long tc_tiles = 0;
            int tc_ctas = 0;
        };
        auto prepare_tc = [&](PreparedLevel& P, bool threads) {
            // TMA tensor maps of the entries' source columns (128 bytes each)
            P.maps.resize(P.tc.size() * 128);
            if (threads && P.tc.size() >= 1024) {
                const int chunks = 32;
                const size_t per = (P.tc.size() + chunks - 1) / chunks;
                parallel_for(chunks, [&](int ck) {
                    PARODE_CUDA(cudaSetDevice(device_));  // the encoder needs the device's context
                    for (size_t k = ck * per; k < std::min(P.tc.size(), (size_t)(ck + 1) * per); ++k)
                        level_encode_src_map(P.tc[k], &P.maps[k * 128]);
                });
            } else {
                for (size_t k = 0; k < P.tc.size(); ++k) level_encode_src_map(P.tc[k], &P.maps[k * 128]);
            }
            for (const LevelArgs& a : P.tc) {
                P.tc_start.push_back(P.tc_tiles);
                P.tc_tiles += level_tc_tiles(a);
            }
            // one persistent CTA per SM, tile ranges balanced by work
            P.tc_ctas = (int)std::min<long>(sms_, P.tc_tiles);
            P.tc_ranges = level_tc_ranges(P.tc, P.tc_ctas);
        };
        auto prepare = [&](const std::vector<std::pair<int, LevelArgs>>& ents, int l) {
            // group by (config id, CW); entries keep the original form for the
            // swap of a tiled down-sweep and the stored form for the contraction
            PreparedLevel P;
            std::vector<std::pair<int, int>> keys;
            // mixed form: levels below the top four of a system run on the
            // tensor cores (3xTF32); the top four, where high powers of Phi
            // amplify rounding, stay FP64
            for (const auto& e : ents) {
                if (e.second.ncols <= 0) continue;
                const Sys& q = sys_[e.first];
                if (l >= 0 && l < q.tc_levels && level_tc_supported(e.second)) {
                    // exact part of P = Phi^(2^k), k = lev0 + l: I for RK4; for
                    // ABM the companion shift S^(2^k) (block b reads block
                    // min(b + 2^k, 3))
                    const int k = q.lev0 + l;
                    LevelArgs t = e.second;
                    t.rn = q.solver == kRK4 ? 0 : q.n;
                    t.rsh = std::min(1 << std::min(k, 2), 3);
                    t.Ps = q.Ps + (size_t)l * (level_split_bytes(q.Np) / sizeof(float));
                    P.tc.push_back(t);
                    continue;
                }
                LevelConfig c = level_config(e.second);
                std::pair<int, int> key(c.id, c.CW);
                size_t g = 0;
                while (g < keys.size() && keys[g] != key) ++g;
                if (g == keys.size()) {
                    keys.push_back(key);
                    P.groups.emplace_back();
                    P.groups.back().cfg = c;
                }
                PreparedGroup& G = P.groups[g];
                G.stored.push_back(level_grouped_args(e.second));
                if (c.id >= 5 && e.second.cpy) G.swaps.push_back(e.second);
            }
            for (PreparedGroup& G : P.groups) {
                for (const LevelArgs& a : G.stored) {
                    LevelConfig c = level_config(a);
                    G.start.push_back(G.tiles);
                    G.tiles += level_tiles(c, a);
                    G.smem = std::max(G.smem, c.smem);
                }
                for (const LevelArgs& a : G.swaps) G.swap_elems = std::max(G.swap_elems, a.ncols * (long)a.Np);
            }
            if (!P.tc.empty()) prepare_tc(P, false);  // the levels already run on all threads
            return P;
        };
        auto emit_tc = [&](PreparedLevel& P) {
            const size_t moff = jput(P.maps.data(), P.maps.size());
            for (size_t k = 0; k < P.tc.size(); ++k) P.tc[k].src_map = base + moff + k * 128;
            GroupedLaunch gl;
            gl.cfg.id = kTcConfig;
            gl.nent = (int)P.tc.size();
            gl.tiles = P.tc_tiles;
            gl.args = reinterpret_cast<LevelArgs*>(base + jput(P.tc.data(), sizeof(LevelArgs) * P.tc.size()));
            gl.start = reinterpret_cast<long*>(base + jput(P.tc_start.data(), sizeof(long) * P.tc_start.size()));
            gl.ctas = P.tc_ctas;
            gl.cta = reinterpret_cast<long*>(base + jput(P.tc_ranges.data(), sizeof(long) * P.tc_ranges.size()));
            return gl;
        };
        auto emit = [&](std::vector<GroupedLaunch>& out, PreparedLevel& P) {
            for (PreparedGroup& G : P.groups) {
                GroupedLaunch gl;
                gl.cfg = G.cfg;
                gl.nent = (int)G.stored.size();
                gl.tiles = G.tiles;
                gl.smem = G.smem;
                gl.args = reinterpret_cast<LevelArgs*>(base + jput(G.stored.data(), sizeof(LevelArgs) * G.stored.size()));
                gl.start = reinterpret_cast<long*>(base + jput(G.start.data(), sizeof(long) * G.start.size()));
                if (!G.swaps.empty()) {
                    gl.swap_elems = G.swap_elems;
                    gl.nswap = (int)G.swaps.size();
                    gl.swaps = reinterpret_cast<LevelArgs*>(base + jput(G.swaps.data(), sizeof(LevelArgs) * G.swaps.size()));
                }
                out.push_back(gl);
            }
            if (!P.tc.empty()) out.push_back(emit_tc(P));
        };
        auto add_level = [&](std::vector<GroupedLaunch>& out, const std::vector<std::pair<int, LevelArgs>>& ents,
                             int l) {
            PreparedLevel P = prepare(ents, l);
            emit(out, P);
        };
        auto make_tc = [&](std::vector<LevelArgs>& tc) {
            PreparedLevel P;
            P.tc = tc;
            prepare_tc(P, true);
            return emit_tc(P);
        };
        // the levels of every system: power table, up-sweep, down-sweep, in
        // launch order
        struct LevelTask {
            std::vector<GroupedLaunch>* out;
            int l, tc_level;
            int kind;  // 0 power table, 1 up-sweep, 2 down-sweep
            PreparedLevel P;
        };
        std::vector<LevelTask> tasks;
        for (int l = 1; l < Pmax; ++l) tasks.push_back(LevelTask{&ls_power_, l, -1, 0, {}});  // the power table stays FP64
        for (int l = 0; l < Lmax; ++l) tasks.push_back(LevelTask{&ls_up_, l, l, 1, {}});
        for (int l = Lmax - 1; l >= 0; --l) tasks.push_back(LevelTask{&ls_down_, l, l, 2, {}});
        // few systems: the levels are prepared inline (starting a thread per
        // level costs more than their work)
        auto over_tasks = [&](auto&& body) {
            if (lv.size() < 32)
                for (int t = 0; t < (int)tasks.size(); ++t) body(t);
            else
                parallel_for((int)tasks.size(), body);
        };
        over_tasks([&](int t) {
            // the tensor-map encoder needs the device's context current on this thread
            PARODE_CUDA(cudaSetDevice(device_));
            LevelTask& T = tasks[t];
            const int l = T.l;
            std::vector<std::pair<int, LevelArgs>> ents;
            for (int i : lv) {
                const Sys& q = sys_[i];
                const long Np = q.Np;
                LevelArgs a;
                if (T.kind == 0) {
                    if (l >= q.pow_levels) continue;
                    a.P = q.P + (long)(l - 1) * Np * Np;
                    a.ldp = Np;
                    a.Np = q.Np;
                    a.ncols = Np;
                    a.src = a.P;
                    a.src_gs = 1;
                    a.src_ks = Np;
                    a.dst = q.P + (long)l * Np * Np;
                    a.dst_gs = 1;
                    a.dst_is = Np;
                } else {
                    if (l >= q.levels) continue;
                    const long d = 1L << l;
                    const long items = q.resp ? q.nblocks : q.nScan;
                    a.P = q.P + (long)(q.lev0 + l) * Np * Np;
                    a.ldp = Np;
                    a.Np = q.Np;
                    a.ncols = sweep_columns(items, q.Tp, d);
                    if (T.kind == 1) {
                        a.src = q.V + d * Np;
                        a.src_gs = 2 * d * Np;
                        a.acc = q.V + 2 * d * Np;
                        a.acc_gs = 2 * d * Np;
                        a.dst = q.V + 2 * d * Np;
                        a.dst_gs = 2 * d * Np;
                    } else {
                        // in place: node prefix in slot g 2d - 1, right half's prefix
                        // replaces the left half's aggregate in slot g 2d + d - 1
                        a.src = q.V;
                        a.src_gs = 2 * d * Np;
                        a.acc = q.V + d * Np;
                        a.acc_gs = 2 * d * Np;
                        a.dst = q.V + d * Np;
                        a.dst_gs = 2 * d * Np;
                    }
                }
                ents.push_back({i, a});
            }
            T.P = prepare(ents, T.tc_level);
        });
        phase("jobs/levels prepared", false);
        for (LevelTask& T : tasks) emit(*T.out, T.P);
        phase("jobs/scan-levels", false);
        // response GEMMs (FP64 tiled DMMA): the block aggregates into scan
        // slots 0 .. Tp - 1 (zeros past the last block), then the outputs from
        // [sample window; X_b], X_b = the scanned state in slot b - 1
        std::vector<std::pair<int, LevelArgs>> agg, out, state;
        std::vector<LevelArgs> tcg;
        std::vector<CopyJob> zero;
        for (int i : rs_) {
            const Sys& q = sys_[i];
            const long ld = q.Kpad + q.Np;
            if (q.resp_tc) {
                // mixed: the aggregates and the window part of the outputs on
                // the tensor cores (3xTF32, W pre-split at set-up); the
                // initial-state part C Phi^j X_b of the outputs stays FP64
                LevelArgs a;
                a.P = q.Wm + (long)q.Bk * q.p * ld;
                a.ldp = ld;
                a.Np = q.Np;
                a.M = q.Np;
                a.K = q.Kw;
                a.ncols = q.nblocks;
                a.src = q.U;
                a.src_gs = (q.solver == kRK4 ? 2L : 1L) * q.Bk * q.mu;
                a.src_ks = 1;
                a.dst = q.V + q.Np;
                a.dst_gs = q.Np;
                a.Ps = q.Psa;
                LevelArgs w = a;
                w.P = q.Wm;
                w.M = q.Bk * q.p;
                w.dst = q.Y + (q.solver == kRK4 ? 0L : 3L * q.p);
                w.dst_gs = (long)q.Bk * q.p;
                w.dst_limit = q.nScan * (long)q.p;
                w.Ps = q.Psw;
                if (!level_tc_supported(a) || !level_tc_supported(w))
                    throw Error(kInvalidArgument, "response GEMM not supported by the tensor-core kernel");
                tcg.push_back(a);
                tcg.push_back(w);
                LevelArgs x;
                x.P = q.Wm + q.Kpad;
                x.ldp = ld;
                x.Np = q.Np;
                x.M = q.Bk * q.p;
                x.K = q.Np;
                x.ncols = q.nblocks;
                x.src = q.V;
                x.src_gs = q.Np;
                x.src_ks = 1;
                x.acc = w.dst;
                x.acc_gs = w.dst_gs;
                x.dst = w.dst;
                x.dst_gs = w.dst_gs;
                x.dst_limit = w.dst_limit;
                state.push_back({i, x});
                if (q.Tp > q.nblocks) {
                    CopyJob z;
                    z.dst = q.V + (1 + q.nblocks) * (long)q.Np;
                    z.N = (q.Tp - q.nblocks) * (long)q.Np;
                    zero.push_back(z);
                    maxZero_ = std::max(maxZero_, z.N);
                }
                continue;
            }
            LevelArgs a;
            a.P = q.Wm + (long)q.Bk * q.p * ld;
            a.ldp = ld;
            a.Np = q.Np;
            a.M = q.Np;
            a.K = q.Kpad;
            a.ncols = q.Tp;
            a.src_cols = q.nblocks;
            a.src = q.U;
            a.src_gs = (q.solver == kRK4 ? 2L : 1L) * q.Bk * q.mu;
            a.src_ks = 1;
            a.dst = q.V + q.Np;
            a.dst_gs = q.Np;
            a.dst_is = 1;
            agg.push_back({i, a});
            LevelArgs b = a;
            b.P = q.Wm;
            b.M = q.Bk * q.p;
            b.K = (int)ld;
            b.K1 = q.Kpad;
            b.src2 = q.V;
            b.src2_gs = q.Np;
            b.ncols = q.nblocks;
            b.src_cols = 0;
            b.dst = q.Y + (q.solver == kRK4 ? 0L : 3L * q.p);
            b.dst_gs = (long)q.Bk * q.p;
            b.dst_limit = q.nScan * (long)q.p;
            out.push_back({i, b});
            if ((a.K & 1) || (b.K & 1) || (ld & 1) || (a.src_gs & 1))
                throw Error(kInvalidArgument, "response GEMM shapes must be even");
        }
        if (!agg.empty()) {
            add_level(rs_agg_, agg, -1);
            add_level(rs_out_, out, -1);
        }
        if (!tcg.empty()) {
            rs_tc_.push_back(make_tc(tcg));
            add_level(rs_state_, state, -1);
        }
        nZero_ = (int)zero.size();
        if (nZero_ > 0) dZero_ = reinterpret_cast<CopyJob*>(base + jput(zero.data(), sizeof(CopyJob) * zero.size()));
    }
    // mixed: P_l - R_l of every tensor-core level, split once per execute
    // after the power table
    {
        std::vector<LevelArgs> sp;
        for (int i : lv) {
            const Sys& q = sys_[i];
            for (int l = 0; l < q.tc_levels; ++l) {
                const int k = q.lev0 + l;
                LevelArgs a;
                a.P = q.P + (long)k * q.Np * q.Np;
                a.ldp = q.Np;
                a.Np = q.Np;
                a.rn = q.solver == kRK4 ? 0 : q.n;
                a.rsh = std::min(1 << std::min(k, 2), 3);
                a.Ps = q.Ps + (size_t)l * (level_split_bytes(q.Np) / sizeof(float));
                sp.push_back(a);
                maxSplitElems_ = std::max<long>(maxSplitElems_, (long)level_split_bytes(q.Np) / 8);
            }
        }
        for (int i : rs_) {
            const Sys& q = sys_[i];
            if (!q.resp_tc) continue;
            const long ld = q.Kpad + q.Np;
            LevelArgs a;
            a.P = q.Wm + (long)q.Bk * q.p * ld;
            a.ldp = ld;
            a.Np = q.Np;
            a.M = q.Np;
            a.K = q.Kw;
            a.Ps = q.Psa;
            sp.push_back(a);
            maxSplitElems_ = std::max<long>(maxSplitElems_, (long)gemm_split_bytes(a.M, a.K) / 8);
            a.P = q.Wm;
            a.M = q.Bk * q.p;
            a.Ps = q.Psw;
            sp.push_back(a);
            maxSplitElems_ = std::max<long>(maxSplitElems_, (long)gemm_split_bytes(a.M, a.K) / 8);
        }
        nSplit_ = (int)sp.size();
        if (nSplit_ > 0) dSplit_ = reinterpret_cast<LevelArgs*>(base + jput(sp.data(), sizeof(LevelArgs) * sp.size()));
    }
    // set-up copies: compact Phi -> P level 0 (padded, the ABM shift rows
    // written exactly), ABM outputs 0..2 -> Y rows 0..2
    std::vector<PhiJob> phi_jobs;
    long max_phi = 0;
    for (int i = 0; i < N; ++i) {
        const Sys& q = sys_[i];
        PhiJob pj;
        pj.dst = q.P;
        pj.src = reinterpret_cast<double*>(static_cast<char*>(disc_) + doff[i].phi);
        pj.n = q.n;
        pj.Np = q.Np;
        pj.solver = q.solver;
        phi_jobs.push_back(pj);
        max_phi = std::max(max_phi, (long)q.Np * q.Np);
        if (q.solver == kABM) {
            CopyJob y;
            y.dst = q.Y;
            y.src = dp(off[i].ypre);
            y.N = 3L * q.p;
            setup_copies.push_back(y);
        }
    }
    {
        const int zero[4] = {0, 0, 0, 0};
        dStatus_ = reinterpret_cast<int*>(base + jput(zero, sizeof(zero)));
    }
    long max_copy = 0;
    for (const CopyJob& c : setup_copies) max_copy = std::max(max_copy, c.N);
    const CopyJob* dSetup =
        reinterpret_cast<const CopyJob*>(base + jput(setup_copies.data(), sizeof(CopyJob) * setup_copies.size()));
    const PhiJob* dPhi = reinterpret_cast<const PhiJob*>(base + jput(phi_jobs.data(), sizeof(PhiJob) * phi_jobs.size()));
    if (J.bytes > arena_bytes_) throw Error(kDeviceError, "batch job arrays overflow the arena reservation");

    phase("jobs", false);
    // ---- upload and set-up launches ------------------------------------------
    // from here on the device reads the staged blocks: a failure waits for the
    // stream before the blocks go back to the pool
    try {
    // work buffers start zeroed (the response windows' sample padding relies on it)
    if (!rs_.empty()) PARODE_CUDA(cudaMemsetAsync(base + const_end, 0, work_end - const_end, stream_));
    PARODE_CUDA(cudaMemcpyAsync(base, stage->data(), const_end, cudaMemcpyHostToDevice, stream_));
    PARODE_CUDA(cudaMemcpyAsync(base + work_end, jstage->data(), J.bytes - work_end, cudaMemcpyHostToDevice, stream_));
    for (size_t k = 0; k < setup_copies.size(); k += 65535)
        launch_copy_batch(dSetup + k, (int)std::min<size_t>(65535, setup_copies.size() - k), max_copy, stream_);
    for (size_t k = 0; k < phi_jobs.size(); k += 65535)
        launch_phi_batch(dPhi + k, (int)std::min<size_t>(65535, phi_jobs.size() - k), max_phi, stream_);
    phase("upload", true);
    // the power table P_l = Phi^(2^l), the response matrices and, in the
    // mixed form, the splits of the tensor-core operands depend on Phi alone:
    // formed here with Phi, once per batch, like the rest of the discretisation
    for (const Bucket& bk : buckets_) launch_batch_stage(0, bk.sh, bk.launch, stream_);
    for (const GroupedLaunch& g : ls_power_) launch_grouped(g, stream_);
    phase("power-tables", true);
    build_responses();
    phase("responses", true);
    for (int k = 0; k < nSplit_; k += 65535)
        launch_level_split(dSplit_ + k, std::min(65535, nSplit_ - k), maxSplitElems_, stream_);
    const int nforks = (int)buckets_.size() + (lv.empty() ? 0 : 1);
    forks_.resize(nforks, nullptr);
    for (auto& f : forks_) PARODE_CUDA(cudaStreamCreateWithFlags(&f, cudaStreamNonBlocking));
    events_.resize(nforks + 1, nullptr);
    for (auto& e : events_) PARODE_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    // no wait for the device here: executes are ordered after the set-up by
    // ready_, and the host images stay alive with the plan
    PARODE_CUDA(cudaEventCreateWithFlags(&ready_, cudaEventDisableTiming));
    PARODE_CUDA(cudaEventRecord(ready_, stream_));
    host_stage_ = std::move(stage);
    host_jobs_ = std::move(jstage);
    phase("splits", true);
    } catch (...) {
        if (stream_) cudaStreamSynchronize(stream_);
        throw;
    }
    if (opt.log)
        std::fprintf(stderr,
                     "ParODE batch set-up (%d systems, %zu response, %zu level, %zu buckets, %.2f GB: tables+scan %.2f, "
                     "W %.2f, W split %.2f, samples %.2f, outputs %.2f):%s\n",
                     N, rs_.size(), ls_.size(), buckets_.size(), arena_bytes_ / 1e9, kind_bytes[0] / 1e9,
                     kind_bytes[1] / 1e9, kind_bytes[2] / 1e9, kind_bytes[3] / 1e9, kind_bytes[4] / 1e9, phases.c_str());
}

void BatchPlan::build_responses()
{
    // W of every response system from Phi, its power table, Bbar, Cext and
    // D, in groups whose table workspace stays under 1 GiB
    const size_t cap = (size_t)1 << 30;
    size_t k = 0;
    while (k < rs_.size()) {
        std::vector<ResponseArgs> ra;
        std::vector<const double*> pow;
        size_t ws = 0;
        int maxR = 0;
        for (; k < rs_.size(); ++k) {
            const Sys& q = sys_[rs_[k]];
            ResponseArgs a;
            a.solver = q.solver;
            a.n = q.n;
            a.m = q.mu;
            a.p = q.p;
            a.NP = q.Np;
            a.B = q.Bk;
            a.zeroB = q.zeroB;
            a.zeroD = q.zeroD;
            a.Phi = q.P;
            a.Bbar = q.Bbar;
            a.Cext = q.Cext;
            a.D = q.D;
            a.Wm = q.Wm;
            a.K = q.Kw;
            a.Kpad = q.Kpad;
            a.NPstate = q.Np;
            const size_t need = sizeof(double) * response_workspace_doubles(a);
            if (!ra.empty() && ws + need > cap) break;
            a.CPt = reinterpret_cast<double*>(ws);  // offsets until the workspace exists
            ra.push_back(a);
            pow.push_back(q.P);
            ws += need;
            maxR = std::max(maxR, q.lev0);
        }
        const int nent = (int)ra.size();
        char* buf = nullptr;
        // meta: the entries, their CTA starts, and per doubling step (and the
        // product step) the GEMM arguments and tile starts
        const size_t meta = align_up(sizeof(ResponseArgs) * nent) + 2 * align_up(sizeof(long) * nent) +
                            (size_t)(maxR + 1) * (align_up(2 * sizeof(LevelArgs) * nent) + align_up(2 * sizeof(long) * nent));
        PARODE_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&buf), ws + meta, stream_));
        struct Workspace {  // freed after the stream's uses, also when a step below fails
            char* p;
            cudaStream_t s;
            ~Workspace() { cudaFreeAsync(p, s); }
        } wsguard{buf, stream_};
        for (ResponseArgs& a : ra) {
            const size_t off = reinterpret_cast<size_t>(a.CPt);
            response_workspace_carve(a, reinterpret_cast<double*>(buf + off));
        }
        std::vector<long> is(nent), fs(nent);
        long ictas = 0, fctas = 0;
        for (int e = 0; e < nent; ++e) {
            is[e] = ictas;
            fs[e] = fctas;
            ictas += response_init_ctas(ra[e]);
            fctas += response_fill_ctas(ra[e]);
        }
        // host image of the meta region (pinned: the copy does not wait for
        // the power tables launched before it); gaps are copied, never read
        auto img = std::make_unique<HostStage>(meta);
        size_t at = 0;
        auto put = [&](const void* src, size_t n) {
            const size_t o = at;
            std::memcpy(img->data() + o, src, n);
            at = align_up(at + std::max<size_t>(n, 1));
            return buf + ws + o;
        };
        const ResponseArgs* dArgs = reinterpret_cast<const ResponseArgs*>(put(ra.data(), sizeof(ResponseArgs) * nent));
        const long* dIs = reinterpret_cast<const long*>(put(is.data(), sizeof(long) * nent));
        const long* dFs = reinterpret_cast<const long*>(put(fs.data(), sizeof(long) * nent));
        struct Step {
            LevelConfig cfg;
            const LevelArgs* args;
            const long* start;
            int nent;
            long tiles;
        };
        std::vector<Step> steps;
        for (int l = 0; l <= maxR; ++l) {
            // l < maxR: doubling step l; l == maxR: the products with Bbar
            std::vector<LevelArgs> ents;
            for (int e = 0; e < nent; ++e) {
                LevelArgs two[2];
                int c = 2;
                if (l < maxR) c = response_doubling_args(ra[e], pow[e], l, two);
                else response_product_args(ra[e], two);
                for (int q = 0; q < c; ++q) ents.push_back(level_grouped_args(two[q]));
            }
            if (ents.empty()) continue;
            Step st;
            st.cfg = level_config(ents[0]);
            std::vector<long> start;
            long tiles = 0;
            for (const LevelArgs& a : ents) {
                if (level_config(a).id != st.cfg.id) throw Error(kDeviceError, "response tables: mixed tilings");
                start.push_back(tiles);
                tiles += level_tiles(st.cfg, a);
            }
            st.nent = (int)ents.size();
            st.tiles = tiles;
            st.args = reinterpret_cast<const LevelArgs*>(put(ents.data(), sizeof(LevelArgs) * ents.size()));
            st.start = reinterpret_cast<const long*>(put(start.data(), sizeof(long) * start.size()));
            steps.push_back(st);
        }
        PARODE_CUDA(cudaMemcpyAsync(buf + ws, img->data(), meta, cudaMemcpyHostToDevice, stream_));
        launch_response_init(dArgs, dIs, nent, ictas, stream_);
        for (const Step& st : steps)
            launch_affine_level_grouped(st.cfg, st.args, st.start, st.nent, st.tiles, st.cfg.smem, stream_);
        launch_response_fill(dArgs, dFs, nent, fctas, stream_);
        host_keep_.push_back(std::move(img));  // the copy may read it until it runs
    }
}

BatchPlan::~BatchPlan() { release(); }

void BatchPlan::release()
{
    cudaSetDevice(device_);
    if (last_stream_ && last_stream_ != stream_) cudaStreamSynchronize(last_stream_);
    if (stream_) cudaStreamSynchronize(stream_);
    last_stream_ = nullptr;
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
    cudaStream_t fs = stream_ ? stream_ : cudaStreamPerThread;
    if (disc_) cudaFreeAsync(disc_, fs);
    disc_ = nullptr;
    for (auto& f : forks_)
        if (f) {
            cudaStreamSynchronize(f);
            cudaStreamDestroy(f);
            f = nullptr;
        }
    for (auto& e : events_)
        if (e) {
            cudaEventDestroy(e);
            e = nullptr;
        }
    if (ready_) cudaEventDestroy(ready_);
    ready_ = nullptr;
    if (arena_) cudaFreeAsync(arena_, fs);
    arena_ = nullptr;
    if (stream_) {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }
    stream_ = nullptr;
}

double BatchPlan::state_steps() const
{
    double t = 0;
    for (const Sys& q : sys_) t += (double)q.n * (double)q.nOut;
    return t;
}

void BatchPlan::execute(cudaStream_t s)
{
    PARODE_CUDA(cudaSetDevice(device_));
    if (!s) s = stream_;
    if (s != stream_) PARODE_CUDA(cudaStreamWaitEvent(s, ready_, 0));
    last_stream_ = s;
    // a batch executed again replays its launch list as one CUDA graph
    // (captured at the second execute): one host launch per execute
    if (graph_state_ == 1) graph_state_ = capture_graph() ? 2 : -1;
    if (graph_state_ == 2) {
        PARODE_CUDA(cudaGraphLaunch(graph_exec_, s));
        return;
    }
    enqueue(s);
    if (graph_state_ == 0) graph_state_ = 1;
}

bool BatchPlan::capture_graph()
{
    // on the batch's own stream (never the legacy stream); a failure of any
    // step leaves the batch executing launch by launch
    if (cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    bool ok = true;
    try {
        enqueue(stream_);
    } catch (...) {
        ok = false;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(stream_, &g);
    if (!ok || e != cudaSuccess || !g) {
        cudaGetLastError();
        if (g) cudaGraphDestroy(g);
        return false;
    }
    const cudaError_t ei = cudaGraphInstantiate(&graph_exec_, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        cudaGetLastError();
        graph_exec_ = nullptr;
        return false;
    }
    return true;
}

void BatchPlan::enqueue(cudaStream_t s)
{
    int launches = 0;
    // inputs for everything first
    if (nSampleJobs_ > 0) {
        for (int k = 0; k < nSampleJobs_; k += 65535) {
            launch_samples_batch(dSampleJobs_ + k, std::min(65535, nSampleJobs_ - k), maxSample_, maxTerms_, s);
            ++launches;
        }
    }
    for (int i : user_inputs_) {
        const Sys& q = sys_[i];
        inputs_->fill(q.input, device_, q.U, q.mu, q.u_base, q.u_dt, q.nU, opt_.input_double, s);
        ++launches;
    }
    // fork: one stream per blocked bucket and one for the level-synchronous set
    PARODE_CUDA(cudaEventRecord(events_[0], s));
    int f = 0;
    for (Bucket& bk : buckets_) {
        cudaStream_t fs = forks_[f++];
        PARODE_CUDA(cudaStreamWaitEvent(fs, events_[0], 0));
        for (int stage = 1; stage < 4; ++stage) {
            launch_batch_stage(stage, bk.sh, bk.launch, fs);
            ++launches;
        }
    }
    if (!ls_.empty() || !rs_.empty()) {
        cudaStream_t fs = forks_[f++];
        PARODE_CUDA(cudaStreamWaitEvent(fs, events_[0], 0));
        const int nls = (int)ls_.size();
        if (nls > 0) {
            launch_forcing_batch(dForcing_, nls, maxForcing_, fs);
            ++launches;
        }
        for (const GroupedLaunch& g : rs_agg_) {
            launch_grouped(g, fs);
            ++launches;
        }
        for (const GroupedLaunch& g : rs_tc_) {
            launch_grouped(g, fs);
            ++launches;
        }
        if (nZero_ > 0) {
            for (int k = 0; k < nZero_; k += 65535) {
                launch_copy_batch(dZero_ + k, std::min(65535, nZero_ - k), maxZero_, fs);
                ++launches;
            }
        }
        for (const GroupedLaunch& g : ls_up_) {
            launch_grouped(g, fs);
            ++launches;
        }
        launch_copy_batch(dSeed_, nSeed_, maxSeed_, fs);
        ++launches;
        for (const GroupedLaunch& g : ls_down_) {
            if (g.nswap > 0) {
                launch_swap_grouped(g.swaps, g.nswap, g.swap_elems, fs);
                ++launches;
            }
            launch_grouped(g, fs);
            ++launches;
        }
        if (nls > 0) {
            launch_output_batch(dOutput_, nls, maxOutput_, fs);
            ++launches;
        }
        for (const GroupedLaunch& g : rs_out_) {
            launch_grouped(g, fs);
            ++launches;
        }
        for (const GroupedLaunch& g : rs_state_) {
            launch_grouped(g, fs);
            ++launches;
        }
    }
    // join
    for (int k = 0; k < f; ++k) {
        PARODE_CUDA(cudaEventRecord(events_[k + 1], forks_[k]));
        PARODE_CUDA(cudaStreamWaitEvent(s, events_[k + 1], 0));
    }
    launches_ = launches;
}

void BatchPlan::launch_grouped(const GroupedLaunch& g, cudaStream_t s)
{
    if (g.cfg.id == kTcConfig) launch_level_tc(g.args, g.start, g.nent, g.cta, g.ctas, dStatus_, s);
    else launch_affine_level_grouped(g.cfg, g.args, g.start, g.nent, g.tiles, g.smem, s);
}

void BatchPlan::get_output(int i, double* t, double* y)
{
    if (i < 0 || i >= size()) throw Error(kInvalidArgument, "system index out of range");
    const Sys& q = sys_[i];
    PARODE_CUDA(cudaSetDevice(device_));
    // the last execute's stream (joined from the batch's fork streams) and
    // the batch stream; no device-wide synchronisation, other batches run on
    PARODE_CUDA(cudaStreamSynchronize(last_stream_ ? last_stream_ : stream_));
    PARODE_CUDA(cudaStreamSynchronize(stream_));
    int st = 0;
    PARODE_CUDA(cudaMemcpyAsync(&st, dStatus_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    if (y)
        PARODE_CUDA(cudaMemcpyAsync(y, q.Y, sizeof(double) * (size_t)q.nOut * q.p, cudaMemcpyDeviceToHost, stream_));
    PARODE_CUDA(cudaStreamSynchronize(stream_));
    if (st != 0) throw Error(kDeviceError, "a tensor-core wait gave up (the result is incomplete)");
    if (t) time_vector(q.solver, q.t0, q.tEnd, q.h, t);
}

}  // namespace parode
