// solver.cpp -- plan set-up and execution (see solver.h).
#include "solver.h"

#include "batch.h"
#include "common.h"
#include "general.h"
#include "kernels.h"
#include "tuner.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

namespace parode {

namespace {

// Streams and events of finished plans, kept per device for the next plan
// (creating two streams and five events cost ~0.1 ms of every one-shot
// SimulateODE call).  Returned idle: the plan synchronises them first.
struct HandlePool {
    std::mutex mu;
    std::vector<std::pair<int, cudaStream_t>> streams;
    std::vector<std::pair<int, cudaEvent_t>> events;
    std::vector<char*> pinned;
};

HandlePool& handles()
{
    static HandlePool* p = new HandlePool();
    return *p;
}

cudaStream_t take_stream(int dev)
{
    {
        HandlePool& h = handles();
        std::lock_guard<std::mutex> g(h.mu);
        for (size_t k = 0; k < h.streams.size(); ++k)
            if (h.streams[k].first == dev) {
                cudaStream_t s = h.streams[k].second;
                h.streams[k] = h.streams.back();
                h.streams.pop_back();
                return s;
            }
    }
    cudaStream_t s = nullptr;
    PARODE_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return s;
}

cudaEvent_t take_event(int dev)
{
    {
        HandlePool& h = handles();
        std::lock_guard<std::mutex> g(h.mu);
        for (size_t k = 0; k < h.events.size(); ++k)
            if (h.events[k].first == dev) {
                cudaEvent_t e = h.events[k].second;
                h.events[k] = h.events.back();
                h.events.pop_back();
                return e;
            }
    }
    cudaEvent_t e = nullptr;
    PARODE_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return e;
}

void give_stream(int dev, cudaStream_t s)
{
    HandlePool& h = handles();
    std::lock_guard<std::mutex> g(h.mu);
    h.streams.emplace_back(dev, s);
}

void give_event(int dev, cudaEvent_t e)
{
    HandlePool& h = handles();
    std::lock_guard<std::mutex> g(h.mu);
    h.events.emplace_back(dev, e);
}

// Pinned host blocks for a plan's small set-up copies (W's arguments, Phi,
// B, C, D, the initial state, tensor maps): from pageable memory each copy
// waits for its staging, from pinned memory it is queued at once.  A plan
// holds one block until its set-up has synchronised.
constexpr size_t kPinBlock = (size_t)512 << 10;

char* take_pinned()
{
    {
        HandlePool& h = handles();
        std::lock_guard<std::mutex> g(h.mu);
        if (!h.pinned.empty()) {
            char* p = h.pinned.back();
            h.pinned.pop_back();
            return p;
        }
    }
    void* p = nullptr;
    if (cudaHostAlloc(&p, kPinBlock, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;  // the copies then go from pageable memory
    }
    return static_cast<char*>(p);
}

void give_pinned(char* p)
{
    HandlePool& h = handles();
    std::lock_guard<std::mutex> g(h.mu);
    h.pinned.push_back(p);
}

}  // namespace

Plan::Plan(int device, const SystemDesc& sys, InputRegistry* inputs, int uIndex, int solver, double t0,
           double tEnd, double h, const PlanOptions& opt)
    : device_(device), sys_(sys), inputs_(inputs), opt_(opt), solver_(solver), t0_(t0), tEnd_(tEnd), h_(h)
{
    // a failed set-up returns what it took (buffers, streams, events, the
    // pinned block) before the error leaves
    try {
        build(device, sys, inputs, uIndex, solver, t0, tEnd, h, opt);
    } catch (...) {
        release();
        throw;
    }
}

void Plan::build(int device, const SystemDesc& sys, InputRegistry* inputs, int uIndex, int solver, double t0,
                 double tEnd, double h, const PlanOptions& opt)
{
    if (solver != kRK4 && solver != kABM) throw Error(kInvalidSolverType, "unknown solver type");
    if (sys.n <= 0) throw Error(kInvalidSystem, "the system has no states");
    if ((long)sys.A.size() < (long)sys.n * sys.n || (long)sys.x0.size() < sys.n)
        throw Error(kInvalidSystem, "A or x0 too small");
    if (!sys.zeroB && (sys.m <= 0 || (long)sys.B.size() < (long)sys.n * sys.m))
        throw Error(kInvalidSystem, "B has the wrong size");
    if (!sys.zeroC && (sys.p <= 0 || (long)sys.C.size() < (long)sys.p * sys.n))
        throw Error(kInvalidSystem, "C has the wrong size");
    if (!sys.zeroD && (sys.p <= 0 || sys.m <= 0 || (long)sys.D.size() < (long)sys.p * sys.m))
        throw Error(kInvalidSystem, "D has the wrong size");
    nOut_ = parode::num_outputs(solver, t0, tEnd, h, &nScan_);
    if (nOut_ <= 0 || nScan_ <= 0) throw Error(kInvalidSystem, "empty time horizon");
    p_ = sys.out_size();
    // inputs are sampled whenever B or D is present (reference Kernels/u.cl)
    mu_ = (!sys.zeroB || !sys.zeroD) ? sys.m : 0;
    if (mu_ > 0) {
        input_ = inputs ? inputs->get(uIndex) : nullptr;
        if (!input_) throw Error(kInvalidInput, "uIndex does not name a registered input");
    }
    Ns_ = solver == kRK4 ? sys.n : 4 * sys.n;
    Np_ = (int)round_up(Ns_, 8);
    if (Np_ > 1024) throw Error(kInvalidSystem, "scan dimension above 1024 is not supported");
    if (opt.path == kPathGeneral && Ns_ > 64)
        throw Error(kInvalidArgument, "the general scan supports scan dimensions up to 64");
    if ((opt.shards > 1 || opt.shard != 0) && (Ns_ > 64 || opt.path == kPathGeneral || opt.path == kPathLevel))
        throw Error(kInvalidArgument, "a time shard runs on the block-response path (scan dimension <= 64, inputs)");
    if (Ns_ > 64 && opt.path != kPathBlocked && opt.path != kPathBlockedSweep) {
        // scan dimensions above 64: the batch engine's one-system form (the
        // response leaf or the level-synchronous scan, tensor-core levels in
        // the mixed form)
        PARODE_CUDA(cudaSetDevice(device_));
        PARODE_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        PARODE_CUDA(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming));
        BatchSpec b;
        b.sys = sys;
        b.uIndex = uIndex;
        b.solver = solver;
        b.t0 = t0;
        b.tEnd = tEnd;
        b.h = h;
        b.input = input_;
        std::vector<BatchSpec> specs;
        specs.push_back(std::move(b));
        PlanOptions bo = opt;
        if (bo.precision == kTF32) bo.precision = kMixed;  // the batch engine has no single-pass form
        batch_ = std::make_unique<BatchPlan>(device, std::move(specs), inputs, bo);
        precision_used_ = batch_->precision_used(0);
        path_ = batch_->path(0);
        return;
    }
    Tp_ = next_pow2(nScan_);
    levels_ = ilog2(Tp_);
    path_ = kPathLevel;
    if (opt.path == kPathGeneral) {
        path_ = kPathGeneral;
        Np_ = general_padded_dim(Ns_);
        precision_used_ = (opt.precision != kFP64 && compose_tc_supported(Np_)) ? kMixed : kFP64;
        const double bytes = (double)nScan_ * Np_ * Np_ * 8.0 + (double)general_scan_bytes(Np_, nScan_);
        if (bytes > 24e9) throw Error(kNotEnoughResources, "the general scan holds a copy of Phi per step");
    } else {
        const bool can_block = blocked_shape(Ns_, mu_, solver, &shape_);
        if (opt.path >= kPathBlocked && !can_block)
            throw Error(kInvalidArgument, "the blocked path supports scan dimensions up to 64");
        if (opt.path != kPathLevel && can_block) path_ = kPathBlocked;
    }
    if (path_ == kPathBlocked) {
        Np_ = shape_.NP;
        ntiles_ = (nScan_ + shape_.S - 1) / shape_.S;
        nblocks_ = ntiles_ * (shape_.S / shape_.B);
        long c = nblocks_;
        int lev = shape_.R;
        while (c > shape_.S_items) {
            c = (c + shape_.B - 1) / shape_.B;
            lev += shape_.R;
        }
        levels_ = std::max(lev + ilog2(next_pow2(c)), shape_.R);
        // input samples are produced by their own wide kernel, overlapped
        // with the power-table kernel, rather than inside the leaf (where the
        // FP64 sin evaluations would compete with the scan for issue slots)
        gen_ = false;
        stage_bytes_ = blocked_leaf_stage_bytes(shape_, sys.n, mu_, p_, solver);
        // the leaf as GEMMs with the block response matrix (kernels_br.cu)
        // when that costs fewer flops than the in-block sweeps: about
        // 2 (B p + NP) K / B per step against 4 NP^2.  The mixed form runs the
        // aggregate and output-window products on the tensor cores (3xTF32)
        // and keeps the initial-state part of the outputs in FP64.
        if (mu_ > 0 && opt.path != kPathBlockedSweep) {
            const int K = response_window(solver, shape_.B, mu_);
            const double resp = 2.0 * ((double)shape_.B * p_ + Np_) * K / shape_.B;
            const double sweeps = 4.0 * Np_ * Np_;
            if (opt.path == kPathBlockedResponse || resp < 0.5 * sweeps) {
                br_ = true;
                br_tc_ = opt.precision != kFP64;
                one_pass_ = opt.precision == kTF32;
                if (br_tc_) precision_used_ = one_pass_ ? kTF32 : kMixed;
                // a block length forced by the caller or measured for this
                // class of systems (tuner.h) replaces the shape's default
                int Rt = opt.force_log2_block;
                if (Rt < 2) Rt = tuned_log2_block(tune_class(solver, Ns_, mu_, p_, nScan_, opt.precision));
                if (Rt >= 2 && Rt <= 7) {
                    while (Rt > 2 && (1L << Rt) / 2 >= nScan_) --Rt;
                    shape_.R = Rt;
                    shape_.B = 1 << Rt;
                }
                const int Kb = response_window(solver, shape_.B, mu_);
                brK_ = Kb;
                brKpad_ = (Kb + 1) & ~1;
                nblocks_ = (nScan_ + shape_.B - 1) / shape_.B;
                // the chunked carry over blocks reads P_R .. P_{R + 4 h + 3}
                levels_ = shape_.R + chunk_carry_table_levels(nblocks_);
            }
        }
        // otherwise the mixed form runs the in-block sweeps on the tensor
        // cores (3xTF32) when the shape allows it, with the longest tile that
        // fits its shared-memory layout; otherwise the solve stays in FP64
        if (opt.precision != kFP64 && !br_) {
            // largest (levels per block, tile) that fits: the tensor-core
            // operands need bucket starts on 8-row boundaries (S >= 4B) and
            // M = 128 slices (S >= 128)
            BlockedShape tc = shape_;
            bool fits = false;
            for (int R = shape_.R; R >= 2 && !fits; --R) {
                tc = shape_;
                tc.R = R;
                tc.B = 1 << R;
                tc.items_smem = (size_t)R * tc.NP * tc.NP * sizeof(double) + (size_t)tc.S_items * tc.NP * sizeof(double);
                for (int S = shape_.S; S >= std::max(128, 4 * tc.B) && !fits; S >>= 1) {
                    tc.S = S;
                    fits = blocked_leaf_tc_bytes(tc, sys.n, mu_, p_, solver) > 0;
                }
            }
            if (fits) {
                shape_ = tc;
                precision_used_ = kMixed;
                ntiles_ = (nScan_ + shape_.S - 1) / shape_.S;
                nblocks_ = ntiles_ * (shape_.S / shape_.B);
                long c2 = nblocks_;
                int lev2 = shape_.R;
                while (c2 > shape_.S_items) {
                    c2 = (c2 + shape_.B - 1) / shape_.B;
                    lev2 += shape_.R;
                }
                levels_ = std::max(lev2 + ilog2(next_pow2(c2)), shape_.R);
            }
        }
        if (opt.path == kPathBlockedResponse && !br_)
            throw Error(kInvalidArgument, "the response leaf needs inputs");
    }
    if (opt.shards > 1 || opt.shard != 0) setup_shard(opt);
    PARODE_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_));
    // set-up phase times on stderr with PARODE_OPT_LOG (device phases then
    // wait for the device)
    auto clock0 = std::chrono::steady_clock::now();
    std::string phases;
    auto phase = [&](const char* name, bool device) {
        if (!opt.log) return;
        if (device && stream_) PARODE_CUDA(cudaStreamSynchronize(stream_));
        const auto now = std::chrono::steady_clock::now();
        char b[64];
        std::snprintf(b, sizeof b, " %s %.3f ms", name, std::chrono::duration<double, std::milli>(now - clock0).count());
        phases += b;
        clock0 = now;
    };

    PARODE_CUDA(cudaSetDevice(device_));
    stream_ = take_stream(device_);
    side_ = take_stream(device_);
    for (auto& e : fork_) e = take_event(device_);
    done_ = take_event(device_);

    phase("streams", false);
    const int n = sys.n, mB = sys.zeroB ? 0 : sys.m;
    const int W = solver == kRK4 ? 3 : 5;
    std::vector<double> X0((size_t)Np_, 0.0);
    bool tables_forked = false;  // the power table is built on side_ (joined before the final synchronise)
    // ---- device buffers: one block from the stream-ordered pool, carved
    // (each cudaMallocAsync costs a few microseconds even from a warm pool)
    std::vector<std::pair<double**, long>> want;
    double* st = nullptr;
    long npow = std::max(levels_, 1);
    want.emplace_back(&dPow_, npow * (long)Np_ * Np_);
    want.emplace_back(&dBbar_, (long)n * W * std::max(mB, 1));
    // the discretisation's inputs and work (kernels_disc.cu: the host
    // restatement's operation order, so the same bits as host_math.cpp)
    double *dDA = nullptr, *dDB = nullptr, *dPhiC = nullptr, *dDWork = nullptr;
    double *dDJob = nullptr, *dPhiJob = nullptr;
    double* dTiles[3] = {nullptr, nullptr, nullptr};
    long ntiles[3] = {0, 0, 0};
    {
        const long tn = (n + 31) / 32, tm = mB > 0 ? (mB + 31) / 32 : 0;
        for (int st = 0; st < (solver == kRK4 ? 3 : 1); ++st) ntiles[st] = tn * tn + tn * tm;
        const auto words = [](size_t bytes) { return (long)((bytes + 7) / 8); };
        want.emplace_back(&dDA, (long)n * n);
        if (mB) want.emplace_back(&dDB, (long)n * mB);
        want.emplace_back(&dPhiC, (long)n * Ns_);
        want.emplace_back(&dDWork, discretise_work_doubles(n, mB));
        want.emplace_back(&dDJob, words(sizeof(DiscJob)));
        want.emplace_back(&dPhiJob, words(sizeof(PhiJob)));
        for (int st = 0; st < 3; ++st)
            if (ntiles[st]) want.emplace_back(&dTiles[st], words(sizeof(DiscTile) * (size_t)ntiles[st]));
    }
    want.emplace_back(&dC_, std::max<long>(1, (long)p_ * n));
    want.emplace_back(&dD_, std::max<long>(1, (long)p_ * std::max(sys.m, 1)));
    want.emplace_back(&dX0_, Np_);
    want.emplace_back(&st, 1);
    if (path_ == kPathLevel || path_ == kPathGeneral) {
        want.emplace_back(&dV_, (Tp_ + 1) * (long)Np_);  // a leading slot holds the initial state
        if (path_ == kPathGeneral) {
            want.emplace_back(&dMs_, nScan_ * (long)Np_ * Np_);
            want.emplace_back(&dXs_, nScan_ * (long)Np_);
        }
    } else {
        want.emplace_back(&dG_, nblocks_ * (long)Np_);
        want.emplace_back(&dWork_, std::max(blocked_items_scratch(shape_, nblocks_),
                                            chunk_carry_scratch(nblocks_) + 1 + shard_k_) *
                                       (long)Np_);
        if (shards_ > 1) {
            // the gathered top items of every shard, then the scratch of their scan
            const long items = (long)shards_ * shard_c_;
            want.emplace_back(&dTop_, (items + chunk_carry_scratch(items) + 1) * (long)Np_);
        }
        want.emplace_back(&dCP_, (long)shape_.B * p_ * Np_);
        want.emplace_back(&dCext_, (long)p_ * Np_);
    }
    want.emplace_back(&dY_, nOut_ * (long)p_);
    if (solver == kRK4) {
        nU_ = 2 * nScan_ + 1;
        u_base_ = t0;
        u_dt_ = 0.5 * h;
        u_joff_ = 2 * shard_begin_;
    } else {
        // ABM scan inputs on the grid (t0 + 3h) - 3h + j h
        // (reference Sources/AdamsMoulton.cpp:426-432 with FP64 time)
        nU_ = nScan_ + 4;
        u_base_ = (t0 + 3.0 * h) - 3.0 * h;
        u_dt_ = h;
        u_joff_ = shard_begin_;
    }
    // the response leaf reads whole windows: the last block's window runs
    // past the samples into a zero padding
    const long pad = (mu_ > 0 && !gen_ && br_) ? (2L * shape_.B + 8) * mu_ + 2 : 0;
    // the mixed response GEMMs read the samples as TF32 planes (their TMA
    // boxes run up to 15 samples past a window); FP64 samples are then only
    // the scratch a user input function fills before the split
    const bool planes = mu_ > 0 && !gen_ && br_tc_;
    const long nf = nU_ * (long)mu_ + pad + 16;
    double* dh = nullptr;
    double* dl = nullptr;
    if (mu_ > 0 && !gen_) {
        if (!planes || input_->kind != InputEntry::kSinusoid) want.emplace_back(&dU_, nU_ * (long)mu_ + pad);
        if (planes) {
            want.emplace_back(&dh, (nf + 1) / 2);
            if (!one_pass_) want.emplace_back(&dl, (nf + 1) / 2);  // the single-pass form reads no lo plane
        }
    }
    carve(want);
    phase("allocate", false);
    dStatus_ = reinterpret_cast<int*>(st);
    PARODE_CUDA(cudaMemsetAsync(st, 0, sizeof(double), stream_));
    if (!(path_ == kPathLevel || path_ == kPathGeneral)) {
        // output rows of the scan state: C at the state block (the last n of
        // the ABM companion state), or the state itself when C and D are absent
        std::vector<double> Cext((size_t)p_ * Np_, 0.0);
        const int xoff = solver == kRK4 ? 0 : 3 * n;
        for (int o = 0; o < p_; ++o)
            for (int c = 0; c < n; ++c) {
                double v = 0.0;
                if (!sys.zeroC) v = sys.C[(size_t)o * n + c];
                else if (sys.zeroD) v = (o == c) ? 1.0 : 0.0;
                Cext[(size_t)o * Np_ + xoff + c] = v;
            }
        h2d(dCext_, Cext.data(), sizeof(double) * Cext.size());
    }
    phase("output rows", false);
    if (mu_ > 0 && !gen_) {
        // every execute writes all nU x mu samples: only the padding is zeroed
        if (dU_ && pad) PARODE_CUDA(cudaMemsetAsync(dU_ + nU_ * mu_, 0, sizeof(double) * (size_t)pad, stream_));
        const size_t used = (size_t)nU_ * mu_;  // rewritten by every execute
        if (dh) {
            dUh_ = reinterpret_cast<float*>(dh);
            PARODE_CUDA(cudaMemsetAsync(dUh_ + used, 0, sizeof(float) * ((size_t)nf - used), stream_));
        }
        if (dl) {
            dUl_ = reinterpret_cast<float*>(dl);
            PARODE_CUDA(cudaMemsetAsync(dUl_ + used, 0, sizeof(float) * ((size_t)nf - used), stream_));
        }
    }
    phase("padding", true);
    // ---- discretisation on the device: A and B up, Phi's compact form and
    // Bbar from the tiled products, Phi expanded into the power table's
    // level 0 (zero padded; ABM: the shift rows above the last block row)
    {
        DiscJob j;
        j.A = dDA;
        j.B = mB ? dDB : nullptr;
        j.phi = dPhiC;
        j.bbar = dBbar_;
        j.work = dDWork;
        j.delta = nullptr;  // the distance to the exact part sizes batch layouts only
        j.n = n;
        j.m = mB;
        j.solver = solver;
        j.h = h;
        h2d(dDA, sys.A.data(), sizeof(double) * (size_t)n * n);
        if (mB) h2d(dDB, sys.B.data(), sizeof(double) * (size_t)n * mB);
        h2d(dDJob, &j, sizeof j);
        const DiscTile* dt[3] = {nullptr, nullptr, nullptr};
        for (int st = 0; st < 3; ++st) {
            if (!ntiles[st]) continue;
            std::vector<DiscTile> tl;
            tl.reserve((size_t)ntiles[st]);
            discretise_tiles(j, st, tl);
            if ((long)tl.size() != ntiles[st]) throw Error(kDeviceError, "discretisation tiles: count mismatch");
            h2d(dTiles[st], tl.data(), sizeof(DiscTile) * tl.size());
            dt[st] = reinterpret_cast<const DiscTile*>(dTiles[st]);
        }
        // no transpose, no distance: the finish's elements spread over CTAs
        const int parts = std::max(1, std::min(32, (n * n + 255) / 256));
        launch_discretise_batch(reinterpret_cast<const DiscJob*>(dDJob), 1, dt, ntiles, sms_, stream_, parts);
        PhiJob pj;
        pj.dst = dPow_;
        pj.src = dPhiC;
        pj.n = n;
        pj.Np = Np_;
        pj.solver = solver;
        h2d(dPhiJob, &pj, sizeof pj);
        launch_phi_batch(reinterpret_cast<const PhiJob*>(dPhiJob), 1, (long)Np_ * Np_, stream_);
    }
    phase("discretise (device)", true);
    if (!sys.zeroC)
        h2d(dC_, sys.C.data(), sizeof(double) * (size_t)p_ * n);
    if (!sys.zeroD)
        h2d(dD_, sys.D.data(), sizeof(double) * (size_t)p_ * sys.m);

    // ---- initial scan state -------------------------------------------------
    if (solver == kRK4) {
        for (int r = 0; r < n; ++r) X0[r] = sys.x0[r];
    } else {
        // start-up inputs u(t0 + j h/2), j = 0..8, evaluated on the device
        // as the reference does (Sources/AdamsMoulton.cpp:51-88)
        std::vector<double> U9((size_t)9 * std::max(sys.m, 1), 0.0);
        if (mu_ > 0) {
            double* dU9 = nullptr;
            alloc(&dU9, 9L * mu_);
            inputs_->fill(input_, device_, dU9, mu_, t0, 0.5 * h, 9, opt_.input_double, stream_);
            PARODE_CUDA(cudaMemcpyAsync(U9.data(), dU9, sizeof(double) * 9 * mu_, cudaMemcpyDeviceToHost, stream_));
            PARODE_CUDA(cudaStreamSynchronize(stream_));
        }
        SystemDesc s0 = sys;
        if (s0.zeroB) s0.m = 0;
        std::vector<double> Xs((size_t)4 * n);
        abm_startup(s0, U9.data(), h, Xs.data());
        for (int r = 0; r < 4 * n; ++r) X0[r] = Xs[r];
        // outputs 0..2 from the start-up states (Sources/GPUFixedStepIterative.cpp:150-172)
        ypre_.assign((size_t)3 * p_, 0.0);
        for (int i = 0; i < 3; ++i) {
            const double* x = &Xs[(size_t)i * n];
            const double* u = &U9[(size_t)(2 * i) * std::max(sys.m, 1)];
            for (int o = 0; o < p_; ++o) {
                double v = 0.0;
                if (sys.zeroC && sys.zeroD) {
                    v = x[o];
                } else {
                    if (!sys.zeroC)
                        for (int c = 0; c < n; ++c) v += sys.C[(size_t)o * n + c] * x[c];
                    if (!sys.zeroD)
                        for (int c = 0; c < sys.m; ++c) v += sys.D[(size_t)o * sys.m + c] * u[c];
                }
                ypre_[(size_t)i * p_ + o] = v;
            }
        }
        alloc(&dYpre_, 3L * p_);
        h2d(dYpre_, ypre_.data(), sizeof(double) * ypre_.size());
    }
    h2d(dX0_, X0.data(), sizeof(double) * Np_);
    phase("copies+start-up", true);
    if (br_) {
        // the carry's powers P_1 .. P_levels (Phi^(2^l)) depend on Phi alone:
        // formed once here, on the side stream beside W (both only read level 0)
        PARODE_CUDA(cudaEventRecord(fork_[0], stream_));
        PARODE_CUDA(cudaStreamWaitEvent(side_, fork_[0], 0));
        launch_blocked_tables(shape_, dPow_, 1, levels_, nullptr, nullptr, p_, side_);
        PARODE_CUDA(cudaEventRecord(fork_[1], side_));
        tables_forked = true;
        // block response matrix from Phi (power-table level 0), Bbar, Cext, D
        alloc(&dW_, (long)(shape_.B * p_ + Np_) * (brKpad_ + Np_));
        ResponseArgs ra;
        ra.solver = solver;
        ra.n = n;
        ra.m = mu_;
        ra.p = p_;
        ra.NP = Np_;
        ra.B = shape_.B;
        ra.zeroB = sys.zeroB;
        ra.zeroD = sys.zeroD;
        ra.Phi = dPow_;
        ra.Bbar = dBbar_;
        ra.Cext = dCext_;
        ra.D = dD_;
        ra.Wm = dW_;
        ra.K = brK_;
        ra.Kpad = brKpad_;
        ra.NPstate = Np_;
        double* dra = nullptr;
        alloc(&dra, (long)((sizeof(ResponseArgs) + 7) / 8));
        h2d(dra, &ra, sizeof(ra));
        launch_block_response(reinterpret_cast<const ResponseArgs*>(dra), 1, Np_, p_, brKpad_, stream_);
        phase("W", true);
        if (br_tc_) {
            // the two tensor-core GEMMs over the sample windows: aggregates
            // into G, output windows into the plan's y buffer (the FP64 state
            // part then adds into the caller's y); W pre-split into TF32 hi/lo
            const long ld = brKpad_ + Np_;
            LevelArgs e[2];
            LevelArgs& a = e[0];
            a.P = dW_ + (long)shape_.B * p_ * ld;
            a.ldp = ld;
            a.Np = Np_;
            a.M = Np_;
            a.K = brK_;
            LevelArgs& w = e[1];
            w = a;
            w.P = dW_;
            w.M = shape_.B * p_;
            const size_t sa = gemm_split_bytes(a.M, a.K), sw = gemm_split_bytes(w.M, w.K);
            double* ps = nullptr;
            alloc(&ps, (long)((sa + sw) / 8));
            a.Ps = reinterpret_cast<const float*>(ps);
            w.Ps = reinterpret_cast<const float*>(reinterpret_cast<char*>(ps) + sa);
            // two 128-byte TMA maps (hi and lo planes) over the windows
            const long stride = (solver == kRK4 ? 2L : 1L) * shape_.B * mu_;
            double* maps = nullptr;
            alloc(&maps, 32);
            unsigned char host_maps[256];
            resp_encode_plane_maps(dUh_, dUl_, nblocks_, brK_, stride, host_maps);
            h2d(maps, host_maps, 256);
            RespArgs r[2];
            r[0].Ps = a.Ps;
            r[0].rows = Np_;
            r[0].K = brK_;
            r[0].ncols = nblocks_;
            r[0].maps = maps;
            r[0].dst = dG_;
            r[0].dst_gs = Np_;
            r[0].fault_withhold = opt.fault_withhold ? 1 : 0;
            r[1] = r[0];
            r[1].Ps = w.Ps;
            r[1].rows = shape_.B * p_;
            r[1].dst = dY_ + (solver == kRK4 ? 0L : 3L * p_);
            r[1].dst_gs = (long)shape_.B * p_;
            r[1].dst_limit = nScan_ * (long)p_;
            r[1].fault_withhold = 0;
            const long start[2] = {0, resp_tc_tiles(r[0])};
            const long tiles = start[1] + resp_tc_tiles(r[1]);
            // both GEMMs in one persistent launch (the output windows beside
            // the carry on a second stream slowed the latency-bound carry
            // launches more than they saved)
            tcCtas_ = (int)std::min<long>(sms_, tiles);
            const std::vector<long> ranges = resp_tc_ranges({r[0], r[1]}, tcCtas_);
            double* d = nullptr;
            alloc(&d, (long)((2 * sizeof(LevelArgs) + 7) / 8));
            dTc_ = reinterpret_cast<LevelArgs*>(d);
            alloc(&d, (long)((2 * sizeof(RespArgs) + 7) / 8));
            dResp_ = reinterpret_cast<RespArgs*>(d);
            alloc(&d, 2);
            dTcStart_ = reinterpret_cast<long*>(d);
            alloc(&d, (long)ranges.size());
            dTcCta_ = reinterpret_cast<long*>(d);
            h2d(dTc_, e, sizeof(e));
            h2d(dResp_, r, sizeof(r));
            h2d(dTcStart_, start, sizeof(start));
            h2d(dTcCta_, ranges.data(), sizeof(long) * ranges.size());
            launch_level_split(dTc_, 2, (long)std::max(sa, sw) / 8, stream_);
            phase("tensor-core set-up", true);
        }
    }
    // a one-shot response plan joins the power table's stream just before the
    // carry, its first user: the solve's samples and response GEMMs run
    // beside the table's squarings
    const bool one_shot = opt.one_shot && shards_ == 1;
    if (tables_forked && one_shot && br_) tables_pending_ = true;
    else if (tables_forked) PARODE_CUDA(cudaStreamWaitEvent(stream_, fork_[1], 0));
    if (!one_shot) {
        PARODE_CUDA(cudaStreamSynchronize(stream_));
        if (pin_) {  // the set-up copies are done: the block goes back to the pool
            give_pinned(pin_);
            pin_ = nullptr;
        }
    }  // else the pinned block stays with the plan until release() has synchronised
    phase("sync", false);
    if (opt.log) std::fprintf(stderr, "ParODE plan set-up (n=%d T=%ld path=%d):%s\n", sys.n, nScan_, path(), phases.c_str());
    // keep a plan's worth of freed memory in the pool, so that the next plan
    // of this size (the next SimulateODE call) maps nothing new.  The pool's
    // reserved memory runs above the plan's bytes (its mapping granularity,
    // the stream and handle pools' neighbours), and a threshold of exactly
    // the plan's bytes let it release the large block between calls (a 250 MB
    // block re-mapped per cfg2 call: 3 ms instead of 7 us): twice the plan
    // plus 256 MiB of slack
    {
        cudaMemPool_t pool = nullptr;
        PARODE_CUDA(cudaDeviceGetDefaultMemPool(&pool, device_));
        uint64_t keep = 0;
        PARODE_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        uint64_t want = 2 * (uint64_t)bytes_ + ((uint64_t)256 << 20);
        if (keep < want) PARODE_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &want));
    }
}

Plan::~Plan() { release(); }

void Plan::release() noexcept
{
    cudaSetDevice(device_);
    if (batch_) {
        // the batch's work joins into the caller's stream or this plan's
        if (stream_) {
            if (done_) cudaStreamWaitEvent(stream_, done_, 0);
            cudaStreamSynchronize(stream_);
        }
        batch_.reset();
    }
    // the buffers return to the device's stream-ordered pool once the last
    // execute (on whatever stream) and the plan's own work are done
    if (stream_ && done_) cudaStreamWaitEvent(stream_, done_, 0);
    if (stream_ && side_ && fork_[0]) {
        cudaEventRecord(fork_[0], side_);
        cudaStreamWaitEvent(stream_, fork_[0], 0);
    }
    for (double* p : bufs_) {
        if (stream_) cudaFreeAsync(p, stream_);
        else cudaFree(p);
    }
    const bool ok_s = !stream_ || cudaStreamSynchronize(stream_) == cudaSuccess;
    if (pin_ && ok_s) give_pinned(pin_);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    const bool ok_d = !side_ || cudaStreamSynchronize(side_) == cudaSuccess;
    for (cudaEvent_t e : events_) cudaEventDestroy(e);
    // idle streams and events go back to the pool for the next plan (handles
    // of a failed context are destroyed instead)
    const bool reuse = ok_s && ok_d;
    for (cudaEvent_t e : fork_)
        if (e) reuse ? give_event(device_, e) : (void)cudaEventDestroy(e);
    if (done_) reuse ? give_event(device_, done_) : (void)cudaEventDestroy(done_);
    if (side_) reuse ? give_stream(device_, side_) : (void)cudaStreamDestroy(side_);
    if (stream_) reuse ? give_stream(device_, stream_) : (void)cudaStreamDestroy(stream_);
    // idempotent
    bufs_.clear();
    events_.clear();
    for (auto& e : fork_) e = nullptr;
    done_ = nullptr;
    side_ = stream_ = nullptr;
    pin_ = nullptr;
    graph_exec_ = nullptr;
}

void Plan::h2d(void* dst, const void* src, size_t bytes)
{
    // through the plan's pinned block while it has room, else from pageable memory
    if (!pin_ && !pin_tried_) {
        pin_ = take_pinned();
        pin_tried_ = true;
    }
    const size_t at = (pin_used_ + 15) & ~(size_t)15;
    if (pin_ && at + bytes <= kPinBlock) {
        std::memcpy(pin_ + at, src, bytes);
        PARODE_CUDA(cudaMemcpyAsync(dst, pin_ + at, bytes, cudaMemcpyHostToDevice, stream_));
        pin_used_ = at + bytes;
        return;
    }
    PARODE_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_));
}

void Plan::alloc(double** p, long n)
{
    // stream-ordered: plans that come and go (every SimulateODE call makes
    // one) reuse the pool's memory instead of mapping and unmapping it
    *p = nullptr;
    const size_t bytes = sizeof(double) * (size_t)std::max<long>(n, 1);
    if (fault_alloc_now()) throw Error(kNotEnoughResources, "device allocation failed (injected)");
    cudaError_t e = cudaMallocAsync((void**)p, bytes, stream_);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        throw Error(kNotEnoughResources, "device allocation failed");
    }
    bufs_.push_back(*p);
    bytes_ += bytes;
}

void Plan::carve(const std::vector<std::pair<double**, long>>& want)
{
    // 256-byte aligned parts of one block (TMA and bulk copies need 16)
    size_t total = 0;
    for (const auto& w : want) total += (sizeof(double) * (size_t)std::max<long>(w.second, 1) + 255) & ~(size_t)255;
    double* base = nullptr;
    alloc(&base, (long)(total / sizeof(double)));
    char* at = reinterpret_cast<char*>(base);
    for (const auto& w : want) {
        *w.first = reinterpret_cast<double*>(at);
        at += (sizeof(double) * (size_t)std::max<long>(w.second, 1) + 255) & ~(size_t)255;
    }
}

void Plan::set_profiling(bool on) { profiling_ = on; }

void Plan::mark(const char* stage, cudaStream_t s)
{
    if (!profiling_) return;
    size_t k = marks_.size();
    if (events_.size() <= k) {
        cudaEvent_t e;
        PARODE_CUDA(cudaEventCreate(&e));
        events_.push_back(e);
    }
    marks_.push_back(stage);
    PARODE_CUDA(cudaEventRecord(events_[k], s));
}

std::vector<std::pair<std::string, float>> Plan::stage_times()
{
    std::vector<std::pair<std::string, float>> out;
    if (marks_.size() < 2) return out;
    PARODE_CUDA(cudaEventSynchronize(events_[marks_.size() - 1]));
    for (size_t k = 1; k < marks_.size(); ++k) {
        float ms = 0.f;
        PARODE_CUDA(cudaEventElapsedTime(&ms, events_[k - 1], events_[k]));
        out.emplace_back(marks_[k], ms);
    }
    return out;
}

void Plan::fill_inputs(cudaStream_t s)
{
    if (mu_ <= 0) return;
    if (dUh_)
        inputs_->fill_planes(input_, device_, dUh_, dUl_, dU_, mu_, u_base_, u_dt_, nU_, opt_.input_double, s, u_joff_);
    else inputs_->fill(input_, device_, dU_, mu_, u_base_, u_dt_, nU_, opt_.input_double, s, u_joff_);
}

void Plan::execute(double* y, cudaStream_t s)
{
    if (shards_ > 1) throw Error(kInvalidArgument, "a time-shard plan runs through its up and down phases");
    PARODE_CUDA(cudaSetDevice(device_));
    if (!s) s = stream_;
    // a plan executed again into the same output buffer replays its launch
    // list as one CUDA graph (captured at the second such execute; stage
    // profiling and the one-system batch form run launch by launch)
    if (!profiling_ && !batch_ && graph_state_ >= 0) {
        if (graph_state_ == 0 || y != graph_y_) {
            if (graph_exec_) {
                cudaGraphExecDestroy(graph_exec_);
                graph_exec_ = nullptr;
            }
            graph_state_ = 1;
            graph_y_ = y;
        } else if (graph_state_ == 1) {
            graph_state_ = capture_graph(y) ? 2 : -1;
        }
        if (graph_state_ == 2) {
            PARODE_CUDA(cudaGraphLaunch(graph_exec_, s));
            last_y_ = y ? y : dY_;
            PARODE_CUDA(cudaEventRecord(done_, s));
            return;
        }
    }
    execute_body(y, s);
    PARODE_CUDA(cudaEventRecord(done_, s));
}

bool Plan::capture_graph(double* y)
{
    if (cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    bool ok = true;
    try {
        execute_body(y, stream_);
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

const double* Plan::device_output() const { return batch_ ? batch_->device_output(0) : dY_; }

void Plan::response_shape(long long info[4]) const
{
    info[0] = info[1] = info[2] = info[3] = 0;
    if (batch_) {
        batch_->response_shape(0, info);
        return;
    }
    if (!br_) return;
    info[0] = shape_.B;
    info[1] = brK_;
    info[2] = Np_;
    info[3] = (nScan_ + shape_.B - 1) / shape_.B;
}

void Plan::execute_body(double* y, cudaStream_t s)
{
    if (batch_) {
        batch_->execute(s);
        if (y)
            PARODE_CUDA(cudaMemcpyAsync(y, batch_->device_output(0), sizeof(double) * (size_t)nOut_ * p_,
                                        cudaMemcpyDeviceToDevice, s));
        launches_ = batch_->launch_count() + (y ? 1 : 0);
        last_y_ = y;
        return;
    }
    if (path_ == kPathBlocked) {
        execute_blocked(y ? y : dY_, s);
        return;
    }
    if (path_ == kPathGeneral) {
        execute_general(y ? y : dY_, s);
        return;
    }
    double* Y = y ? y : dY_;
    const long Np = Np_;
    const int n = sys_.n;
    int launches = 0;
    marks_.clear();
    mark("start", s);

    fill_inputs(s);
    launches += mu_ > 0 ? 1 : 0;
    mark("inputs", s);
    // V slots: dV_ = slot -1 (the initial state), V1 = slots 0 .. Tp-1
    double* V1 = dV_ + Np;
    launch_forcing(V1, Np_, n, sys_.zeroB ? 0 : sys_.m, solver_, dBbar_, dU_, nScan_, Tp_, s);
    ++launches;
    mark("forcing", s);

    // power table P_l = Phi^(2^l): the up-sweep matrix of every node at level
    // l (reference Kernels/MMKernelScanUpsweep.cl:24-53 computes these per node)
    for (int l = 1; l < levels_; ++l) {
        LevelArgs a;
        a.P = dPow_ + (long)(l - 1) * Np * Np;
        a.ldp = Np;
        a.Np = Np_;
        a.ncols = Np;
        a.src = a.P;
        a.src_gs = 1;
        a.src_ks = Np;
        a.dst = dPow_ + (long)l * Np * Np;
        a.dst_gs = 1;
        a.dst_is = Np;
        launch_affine_level(a, s);
        ++launches;
    }
    mark("power_table", s);
    // up-sweep: v[k] = P_l v[k-d] + v[k] (reference Kernels/MVVKernelScanUpsweep.cl:25-48)
    for (int l = 0; l < levels_; ++l) {
        long d = 1L << l;
        LevelArgs a;
        a.P = dPow_ + (long)l * Np * Np;
        a.ldp = Np;
        a.Np = Np_;
        a.ncols = sweep_columns(nScan_, Tp_, d);
        a.src = V1 + (d - 1) * Np;
        a.src_gs = 2 * d * Np;
        a.acc = V1 + (2 * d - 1) * Np;
        a.acc_gs = 2 * d * Np;
        a.dst = V1 + (2 * d - 1) * Np;
        a.dst_gs = 2 * d * Np;
        launch_affine_level(a, s);
        ++launches;
    }
    // the scan is seeded with the initial state (the reference's carry
    // (I, x0), Sources/GPUFixedStepIterative.cpp:191-198,327-330), held in slot -1
    launch_copy(dV_, dX0_, Np, s);
    ++launches;
    // down-sweep, in place: the node over [g 2d, g 2d + 2d) has its prefix
    // (the state at its start) in slot g 2d - 1 and its left half's aggregate in
    // slot g 2d + d - 1; the right half's prefix P_l prefix + aggregate replaces
    // the aggregate, the left half keeps the node's slot.  This is the
    // reference's down-sweep (Kernels/MVVKernelScanDownsweep.cl:25-48 with
    // RootCopyKernelScanDownsweep.cl:11-19) without its copy: the state x_k
    // ends in slot k - 1, x_0 in slot -1.
    for (int l = levels_ - 1; l >= 0; --l) {
        long d = 1L << l;
        LevelArgs a;
        a.P = dPow_ + (long)l * Np * Np;
        a.ldp = Np;
        a.Np = Np_;
        a.ncols = sweep_columns(nScan_, Tp_, d);
        a.src = dV_;
        a.src_gs = 2 * d * Np;
        a.acc = V1 + (d - 1) * Np;
        a.acc_gs = 2 * d * Np;
        a.dst = V1 + (d - 1) * Np;
        a.dst_gs = 2 * d * Np;
        launch_affine_level(a, s);
        ++launches;
    }
    mark("sweeps", s);
    // outputs (reference Kernels/SystemOutput.cl with strides (1,0)/(2,0) for
    // RK4 and (4,3)/(1,3) for ABM, Sources/RungeKutta4thOrder.cpp:209,
    // Sources/AdamsMoulton.cpp:398); x_k is read from slot k - 1
    if (solver_ == kRK4) {
        launch_output(Y, dV_, Np_, 0, n, mu_, p_, dC_, dD_, sys_.zeroC, sys_.zeroD, dU_, 2, 0, nScan_, 0, s);
    } else {
        launch_output(Y, dV_, Np_, 3 * n, n, mu_, p_, dC_, dD_, sys_.zeroC, sys_.zeroD, dU_, 1, 3, nScan_, 3, s);
        PARODE_CUDA(cudaMemcpyAsync(Y, dYpre_, sizeof(double) * 3 * p_, cudaMemcpyDeviceToDevice, s));
    }
    ++launches;
    mark("output", s);
    launches_ = launches;
    last_y_ = Y;
}

void Plan::execute_general(double* Y, cudaStream_t s)
{
    // the reference's pipeline (Sources/RungeKutta4thOrder.cpp:234-288,
    // Sources/AdamsMoulton.cpp:403-461, Sources/GPUFixedStepIterative.cpp:236-446):
    // a copy of Phi per step (DistributeA), the forcing vectors, the scan
    // composing every pair (matrices and vectors), the outputs
    int launches = 0;
    marks_.clear();
    mark("start", s);
    fill_inputs(s);
    launches += mu_ > 0 ? 1 : 0;
    mark("inputs", s);
    double* V1 = dV_ + Np_;
    launch_forcing(V1, Np_, sys_.n, sys_.zeroB ? 0 : sys_.m, solver_, dBbar_, dU_, nScan_, Tp_, s);
    launch_distribute(dMs_, dPow_, Np_, nScan_, sms_, s);
    launches += 2;
    mark("maps", s);
    general_scan(dMs_, V1, dX0_, Np_, nScan_, precision_used_, dXs_, dStatus_, s);
    launches += 2 * ilog2(Tp_) + 2;
    mark("scan", s);
    if (solver_ == kRK4) {
        launch_output(Y, dXs_, Np_, 0, sys_.n, mu_, p_, dC_, dD_, sys_.zeroC, sys_.zeroD, dU_, 2, 0, nScan_, 0, s);
    } else {
        launch_output(Y, dXs_, Np_, 3 * sys_.n, sys_.n, mu_, p_, dC_, dD_, sys_.zeroC, sys_.zeroD, dU_, 1, 3,
                      nScan_, 3, s);
        PARODE_CUDA(cudaMemcpyAsync(Y, dYpre_, sizeof(double) * 3 * p_, cudaMemcpyDeviceToDevice, s));
    }
    ++launches;
    mark("output", s);
    launches_ = launches;
    last_y_ = Y;
}

int Plan::carry(cudaStream_t s)
{
    // the exclusive scan of the block aggregates (kernels_carry.cu)
    return launch_chunk_carry(Np_, dG_, nblocks_, dPow_, shape_.R, 0, dX0_, dWork_, s);
}

LevelArgs Plan::response_agg_args() const
{
    // FP64 aggregates G = W_agg [sample window] per block (tiled DMMA GEMM)
    const long ld = brKpad_ + Np_;
    LevelArgs g;
    g.P = dW_ + (long)shape_.B * p_ * ld;
    g.ldp = ld;
    g.Np = Np_;
    g.M = Np_;
    g.K = brKpad_;
    g.ncols = nblocks_;
    g.src = dU_;
    g.src_gs = (solver_ == kRK4 ? 2L : 1L) * shape_.B * mu_;
    g.src_ks = 1;
    g.dst = dG_;
    g.dst_gs = Np_;
    g.dst_is = 1;
    return g;
}

LevelArgs Plan::response_out_args(double* Y) const
{
    // FP64 outputs y = W_out [sample window ; X_b] per block, written into y
    // (rows (j, o) of block b are contiguous there)
    const long ld = brKpad_ + Np_;
    const int ybase = solver_ == kRK4 ? 0 : 3;
    LevelArgs h = response_agg_args();
    h.P = dW_;
    h.M = shape_.B * p_;
    h.K = (int)ld;
    h.K1 = brKpad_;
    h.src2 = dG_;
    h.src2_gs = Np_;
    h.dst = Y + ybase * p_;
    h.dst_gs = (long)shape_.B * p_;
    h.dst_limit = nScan_ * p_;
    return h;
}

void Plan::state_part(double* Y, long c0, long c1, cudaStream_t s)
{
    // mixed: y = windows + (C Phi^j) X_b over blocks [c0, c1), W's state
    // columns resident in shared memory (kernels_state.cu); the general tiled
    // GEMM where they do not fit.  A block's result does not depend on the
    // range it is formed in.
    const int ybase = solver_ == kRK4 ? 0 : 3;
    const long ld = brKpad_ + Np_;
    const long gs = (long)shape_.B * p_;
    const long off = ybase * p_ + c0 * gs;
    if (launch_state_out(Np_, dW_ + brKpad_, ld, shape_.B * p_, dG_ + c0 * Np_, dY_ + off, Y + off, gs, c1 - c0,
                         nScan_ * p_ - c0 * gs, sms_, s))
        return;
    LevelArgs x;
    x.P = dW_ + brKpad_;
    x.ldp = ld;
    x.Np = Np_;
    x.M = shape_.B * p_;
    x.K = Np_;
    x.ncols = c1 - c0;
    x.src = dG_ + c0 * Np_;
    x.src_gs = Np_;
    x.src_ks = 1;
    x.acc = dY_ + off;
    x.acc_gs = gs;
    x.dst = Y + off;
    x.dst_gs = gs;
    x.dst_limit = nScan_ * p_ - c0 * gs;
    launch_gemm_tiled(x, s);
}

int Plan::response_head(cudaStream_t s)
{
    // leaf = W x [sample window; initial state] per block (kernels_br.cu):
    // aggregates first (the state columns are not used), then the carry.  The
    // power table P_1..P_levels was formed with W when the plan was made.
    int launches = 0;
    marks_.clear();
    mark("start", s);
    fill_inputs(s);
    ++launches;
    mark("inputs", s);
    if (br_tc_) {
        // mixed: aggregates and output windows on the tensor cores
        launch_resp_tc(dResp_, dTcStart_, 2, dTcCta_, tcCtas_, dStatus_, one_pass_, s);
        ++launches;
        mark("aggregates+windows", s);
    } else {
        launch_gemm_tiled(response_agg_args(), s);
        ++launches;
        mark("aggregates", s);
    }
    if (tables_pending_) {
        PARODE_CUDA(cudaStreamWaitEvent(s, fork_[1], 0));
        tables_pending_ = false;
    }
    launches += carry(s);
    mark("carry", s);
    return launches;
}

void Plan::response_outputs(double* Y, long c0, long c1, cudaStream_t s)
{
    // the outputs of blocks [c0, c1) with their carried states, written
    // straight into y (rows (j, o) of block b are contiguous there)
    if (br_tc_) {
        state_part(Y, c0, c1, s);  // y = windows + C Phi^j X_b (FP64)
        return;
    }
    LevelArgs h = response_out_args(Y);
    h.src += c0 * h.src_gs;
    h.src2 += c0 * h.src2_gs;
    h.dst += c0 * h.dst_gs;
    h.dst_limit -= c0 * h.dst_gs;
    h.ncols = c1 - c0;
    launch_gemm_tiled(h, s);
}

void Plan::execute_response(double* Y, cudaStream_t s)
{
    int launches = response_head(s);
    response_outputs(Y, 0, nblocks_, s);
    ++launches;
    if (solver_ == kABM)
        PARODE_CUDA(cudaMemcpyAsync(Y, dYpre_, sizeof(double) * 3 * p_, cudaMemcpyDeviceToDevice, s));
    mark("outputs", s);
    launches_ = launches;
    last_y_ = Y;
}

void Plan::solve_to_host(double* yd, float* yf)
{
    void* y = yf ? (void*)yf : (void*)yd;
    if (!y || batch_ || shards_ > 1 || path_ != kPathBlocked || !br_ || profiling_ || nblocks_ < 8) {
        execute(nullptr, nullptr);
        if (yf)
            get_output_f32(nullptr, yf);
        else
            get_output(nullptr, yd);
        return;
    }
    PARODE_CUDA(cudaSetDevice(device_));
    cudaStream_t s = stream_;
    int launches = response_head(s);
    float* dF = nullptr;
    const long total = nOut_ * (long)p_;
    if (yf) {
        if (fault_alloc_now()) throw Error(kNotEnoughResources, "device allocation failed (injected)");
        if (cudaMallocAsync((void**)&dF, sizeof(float) * (size_t)std::max<long>(total, 1), s) != cudaSuccess) {
            cudaGetLastError();
            throw Error(kNotEnoughResources, "device allocation failed");
        }
    }
    // block ranges: an eighth first (its copy starts soonest), then two
    // quarters and the rest; range k's rows of y are [r[k], r[k + 1]) (the
    // first also holds the ABM start-up rows, the last the ragged tail)
    const long gs = (long)shape_.B * p_, base = (solver_ == kRK4 ? 0 : 3) * (long)p_;
    const long cut[5] = {0, nblocks_ / 8, 3 * nblocks_ / 8, 5 * nblocks_ / 8, nblocks_};
    long r[5] = {0, 0, 0, 0, total};
    for (int k = 1; k < 4; ++k) r[k] = std::min(total, base + cut[k] * gs);
    for (int k = 0; k < 4; ++k) {
        response_outputs(dY_, cut[k], cut[k + 1], s);
        ++launches;
        if (k == 0 && solver_ == kABM)
            PARODE_CUDA(cudaMemcpyAsync(dY_, dYpre_, sizeof(double) * 3 * p_, cudaMemcpyDeviceToDevice, s));
        if (dF) {
            launch_to_float(dY_ + r[k], dF + r[k], r[k + 1] - r[k], s);
            ++launches;
        }
        PARODE_CUDA(cudaEventRecord(fork_[k], s));
    }
    // the copies on the side stream, each after its range (issued after all
    // the ranges, so a pageable destination that blocks the host per copy
    // does not hold back the device's work)
    const size_t es = dF ? sizeof(float) : sizeof(double);
    for (int k = 0; k < 4; ++k) {
        if (r[k + 1] <= r[k]) continue;
        PARODE_CUDA(cudaStreamWaitEvent(side_, fork_[k], 0));
        const void* src = dF ? (const void*)(dF + r[k]) : (const void*)(dY_ + r[k]);
        PARODE_CUDA(cudaMemcpyAsync((char*)y + es * (size_t)r[k], src, es * (size_t)(r[k + 1] - r[k]),
                                    cudaMemcpyDeviceToHost, side_));
    }
    PARODE_CUDA(cudaEventRecord(fork_[0], side_));
    PARODE_CUDA(cudaStreamWaitEvent(s, fork_[0], 0));
    if (dF) PARODE_CUDA(cudaFreeAsync(dF, s));
    PARODE_CUDA(cudaEventRecord(done_, s));
    launches_ = launches;
    last_y_ = dY_;
    PARODE_CUDA(cudaStreamSynchronize(s));
    int status = 0;
    PARODE_CUDA(cudaMemcpy(&status, dStatus_, sizeof(int), cudaMemcpyDeviceToHost));
    if (status != 0) throw Error(kDeviceError, "a device-side wait gave up (tensor-core completion not observed)");
}

void Plan::setup_shard(const PlanOptions& opt)
{
    // Time shard `shard` of `shards` (the reference's multi-device split of
    // the horizon, Sources/RungeKutta4thOrder.cpp:96-125, with its carry
    // between devices, Sources/GPUFixedStepIterative.cpp:296-337): every
    // shard but the last holds S = c 16^k whole blocks, so the chunked
    // carry's first k levels stay inside a shard and the shards' level-k
    // chunk aggregates (c per shard) line up as one sequence; that sequence
    // is scanned by every shard (it is small) after an all-gather, and each
    // shard down-sweeps its own levels from its items' prefixes.
    if (opt.shards < 1 || opt.shard < 0 || opt.shard >= opt.shards)
        throw Error(kInvalidArgument, "shard index out of range");
    if (!br_ || batch_)
        throw Error(kInvalidArgument, "a time shard runs on the block-response path (scan dimension <= 64, inputs)");
    const long B = shape_.B;
    const long nbG = (nScan_ + B - 1) / B;
    const long per = (nbG + opt.shards - 1) / opt.shards;
    int k = 0;
    long p16 = 1;  // 16^k, with c = per / 16^k in [16, 256) once per >= 256
    while (p16 * 256 <= per) {
        p16 *= 16;
        ++k;
    }
    const long c = (per + p16 - 1) / p16;
    const long Sb = p16 * c;
    const long b0 = (long)opt.shard * Sb;
    if (b0 >= nbG) throw Error(kInvalidArgument, "more shards than the horizon's blocks fill");
    shard_ = opt.shard;
    shards_ = opt.shards;
    shard_k_ = k;
    shard_c_ = (int)c;
    shard_begin_ = b0 * B;
    nScanGlobal_ = nScan_;
    nScan_ = std::min(Sb * B, nScan_ - shard_begin_);
    nOut_ = nScan_ + (solver_ == kABM ? 3 : 0);
    nblocks_ = (nScan_ + B - 1) / B;
    // the power table reaches the top scan's levels: P_{R + 4 (k + h) + 3}
    levels_ = shape_.R + 4 * k + chunk_carry_table_levels((long)shards_ * c);
}

void Plan::shard_info(long long info[5]) const
{
    info[0] = shard_begin_;
    info[1] = nScan_;
    info[2] = shard_c_;
    info[3] = Np_;
    info[4] = shards_;
}

void Plan::shard_up(double* dTop, cudaStream_t s)
{
    if (shards_ < 1 || !dTop_) throw Error(kInvalidArgument, "not a time-shard plan");
    PARODE_CUDA(cudaSetDevice(device_));
    if (!s) s = stream_;
    fill_inputs(s);
    if (br_tc_) launch_resp_tc(dResp_, dTcStart_, 2, dTcCta_, tcCtas_, dStatus_, one_pass_, s);
    else launch_gemm_tiled(response_agg_args(), s);
    // the first k chunk levels, from a zero state: the shard's level-k chunk
    // aggregates (fewer than c in a short last shard: zeros after them)
    launch_chunk_up(Np_, dG_, nblocks_, dPow_, shape_.R, dWork_, shard_k_, &shard_levels_, s);
    const ChunkLevels& L = shard_levels_;
    PARODE_CUDA(cudaMemsetAsync(dTop, 0, sizeof(double) * (size_t)shard_c_ * Np_, s));
    PARODE_CUDA(cudaMemcpyAsync(dTop, L.arr[L.h], sizeof(double) * (size_t)L.cnt[L.h] * Np_, cudaMemcpyDeviceToDevice,
                                s));
    shard_up_done_ = true;
}

void Plan::shard_down(const double* dGathered, double* Y, cudaStream_t s)
{
    if (!shard_up_done_) throw Error(kInvalidArgument, "shard_down before shard_up");
    PARODE_CUDA(cudaSetDevice(device_));
    if (!s) s = stream_;
    if (!Y) Y = dY_;
    const long items = (long)shards_ * shard_c_;
    // every shard scans the gathered sequence (exclusive, seeded with the
    // initial state) and keeps the prefixes of its own items
    PARODE_CUDA(cudaMemcpyAsync(dTop_, dGathered, sizeof(double) * (size_t)items * Np_, cudaMemcpyDeviceToDevice, s));
    launch_chunk_carry(Np_, dTop_, items, dPow_, shape_.R + 4 * shard_k_, shard_k_, dX0_, dTop_ + items * Np_, s);
    ChunkLevels L = shard_levels_;
    const double* mine = dTop_ + (long)shard_ * shard_c_ * Np_;
    if (L.h == 0) {
        PARODE_CUDA(cudaMemcpyAsync(dG_, mine, sizeof(double) * (size_t)L.cnt[0] * Np_, cudaMemcpyDeviceToDevice, s));
    } else {
        L.arr[L.h] = const_cast<double*>(mine);
        launch_chunk_down(Np_, L, dPow_, shape_.R, s);
    }
    response_outputs(Y, 0, nblocks_, s);
    if (solver_ == kABM && shard_ == 0)
        PARODE_CUDA(cudaMemcpyAsync(Y, dYpre_, sizeof(double) * 3 * p_, cudaMemcpyDeviceToDevice, s));
    PARODE_CUDA(cudaEventRecord(done_, s));
    last_y_ = Y;
    shard_up_done_ = false;
}

void Plan::execute_blocked(double* Y, cudaStream_t s)
{
    if (br_) {
        execute_response(Y, s);
        return;
    }
    int launches = 0;
    marks_.clear();
    mark("start", s);
    // Two streams: the side stream produces the input samples while the
    // main stream squares the leaf's powers P_1..P_{R-1} (one CTA), then
    // squares the carry's powers P_R.. (one CTA) while the leaf runs on the
    // other SMs.  Events fork from and join back into the caller's stream.
    PARODE_CUDA(cudaEventRecord(fork_[0], s));
    PARODE_CUDA(cudaStreamWaitEvent(side_, fork_[0], 0));
    if (mu_ > 0 && !gen_) {
        fill_inputs(side_);
        ++launches;
    }
    PARODE_CUDA(cudaEventRecord(fork_[1], side_));
    launch_blocked_tables(shape_, dPow_, 1, shape_.R, dCP_, dCext_, p_, s);
    ++launches;
    PARODE_CUDA(cudaEventRecord(fork_[2], s));
    PARODE_CUDA(cudaStreamWaitEvent(side_, fork_[2], 0));
    const bool more_levels = levels_ > shape_.R;
    if (more_levels) {
        launch_blocked_tables(shape_, dPow_, shape_.R, levels_, nullptr, nullptr, p_, side_);
        ++launches;
    }
    PARODE_CUDA(cudaEventRecord(fork_[3], side_));
    PARODE_CUDA(cudaStreamWaitEvent(s, fork_[1], 0));
    mark("inputs+tables", s);

    LeafArgs a;
    a.solver = solver_;
    a.n = sys_.n;
    a.m = mu_;
    a.p = p_;
    a.zeroB = sys_.zeroB;
    a.zeroC = sys_.zeroC;
    a.zeroD = sys_.zeroD;
    a.nScan = nScan_;
    a.ntiles = ntiles_;
    a.ybase = solver_ == kRK4 ? 0 : 3;
    a.P = dPow_;
    a.Bbar = dBbar_;
    a.C = dC_;
    a.D = dD_;
    a.U = dU_;
    a.gen = gen_ ? 1 : 0;
    if (gen_) {
        const double* d = inputs_->sinusoid_device(input_, device_);
        const long q = (long)input_->m * input_->K;
        a.sa = d;
        a.sf = d + q;
        a.sphi = d + 2 * q;
        a.K = input_->K;
    }
    a.u_base = u_base_;
    a.u_dt = u_dt_;
    a.Y = Y;
    a.G = dG_;
    a.stage = stage_bytes_ > 0 ? 1 : 0;
    a.status = dStatus_;
    // one SM stays free for the side stream's power-table kernel
    const int grid = more_levels ? std::max(1, sms_ - 1) : sms_;
    if (precision_used_ == kMixed) launch_blocked_leaf_tc(shape_, a, grid, s);
    else launch_blocked_leaf(shape_, a, grid, s);
    ++launches;
    mark("leaf", s);
    PARODE_CUDA(cudaStreamWaitEvent(s, fork_[3], 0));
    // exclusive scan of the block aggregates, seeded with the initial state
    launches += launch_blocked_carry(shape_, dG_, nblocks_, shape_.R, dPow_, dX0_, dWork_, sms_, s);
    mark("carry", s);
    // y += C Phi^j X_block
    launch_blocked_fixup(shape_, Y, a.ybase, nScan_, p_, dCP_, dG_, s);
    ++launches;
    if (solver_ == kABM)
        PARODE_CUDA(cudaMemcpyAsync(Y, dYpre_, sizeof(double) * 3 * p_, cudaMemcpyDeviceToDevice, s));
    mark("fixup", s);
    launches_ = launches;
    last_y_ = Y;
}

void Plan::get_output_f32(float* t, float* y)
{
    PARODE_CUDA(cudaSetDevice(device_));
    if (batch_ || shards_ > 1) {
        // through the FP64 copy
        std::vector<double> td(t ? (size_t)nOut_ : 0), yd(y ? (size_t)nOut_ * p_ : 0);
        get_output(t ? td.data() : nullptr, y ? yd.data() : nullptr);
        for (size_t k = 0; k < td.size(); ++k) t[k] = (float)td[k];
        for (size_t k = 0; k < yd.size(); ++k) y[k] = (float)yd[k];
        return;
    }
    // y rounded to float on the device, then half the bytes cross the link;
    // the host writes the float time vector meanwhile
    PARODE_CUDA(cudaStreamWaitEvent(stream_, done_, 0));
    float* dF = nullptr;
    const long ny = nOut_ * (long)p_;
    if (y) {
        if (fault_alloc_now()) throw Error(kNotEnoughResources, "device allocation failed (injected)");
        if (cudaMallocAsync((void**)&dF, sizeof(float) * (size_t)std::max<long>(ny, 1), stream_) != cudaSuccess) {
            cudaGetLastError();
            throw Error(kNotEnoughResources, "device allocation failed");
        }
        launch_to_float(last_y_ ? last_y_ : dY_, dF, ny, stream_);
        PARODE_CUDA(cudaMemcpyAsync(y, dF, sizeof(float) * (size_t)ny, cudaMemcpyDeviceToHost, stream_));
        PARODE_CUDA(cudaFreeAsync(dF, stream_));
    }
    if (t) time_vector_f(solver_, t0_, tEnd_, h_, t);
    PARODE_CUDA(cudaStreamSynchronize(stream_));
    int status = 0;
    PARODE_CUDA(cudaMemcpy(&status, dStatus_, sizeof(int), cudaMemcpyDeviceToHost));
    if (status != 0) throw Error(kDeviceError, "a device-side wait gave up (tensor-core completion not observed)");
}

void Plan::get_output(double* t, double* y)
{
    PARODE_CUDA(cudaSetDevice(device_));
    if (batch_) {
        PARODE_CUDA(cudaStreamWaitEvent(stream_, done_, 0));
        PARODE_CUDA(cudaStreamSynchronize(stream_));
        batch_->get_output(0, t, y);
        return;
    }
    // the copy of y queues behind the last execute (whatever its stream); the
    // host computes the time vector meanwhile (into pinned memory the copy
    // runs asynchronously; into pageable memory cudaMemcpyAsync returns when
    // it is done)
    PARODE_CUDA(cudaStreamWaitEvent(stream_, done_, 0));
    if (y)
        PARODE_CUDA(cudaMemcpyAsync(y, last_y_ ? last_y_ : dY_, sizeof(double) * nOut_ * p_, cudaMemcpyDeviceToHost,
                                    stream_));
    if (t && shards_ > 1) {
        // the shard's slice of the horizon's time vector (its first ybase rows
        // are the start-up rows' times, as on shard 0)
        long ns = 0;
        const long nt = parode::num_outputs(solver_, t0_, tEnd_, h_, &ns);
        std::vector<double> tg((size_t)std::max(nt, 1L));
        time_vector(solver_, t0_, tEnd_, h_, tg.data());
        const long ybase = nt - ns;
        for (long i = 0; i < ybase; ++i) t[i] = tg[(size_t)i];
        for (long j = 0; j < nScan_; ++j) t[ybase + j] = tg[(size_t)(ybase + shard_begin_ + j)];
    } else if (t) {
        time_vector(solver_, t0_, tEnd_, h_, t);
    }
    PARODE_CUDA(cudaStreamSynchronize(stream_));
    int status = 0;
    PARODE_CUDA(cudaMemcpy(&status, dStatus_, sizeof(int), cudaMemcpyDeviceToHost));
    if (status != 0) throw Error(kDeviceError, "a device-side wait gave up (tensor-core completion not observed)");
}

}  // namespace parode
