"""Benchmark of the parallel-in-time LTI scan (ParODE hot path) on B200.

Workload (one step = one full solve): RK4, n=64 states, m=8 inputs, p=8
outputs, h=1e-4, T=2^20 steps, seeded synthetic system and sum-of-sinusoids
input (parode_b200/workloads.py: cfg2).  Metric: state*steps/s = n*T per solve
/ solve time, for the mixed-precision form (3xTF32 tensor-core leaf, FP64
carry), with the plain FP64 form timed beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
  python bench.py --impl reference ...   # the reference's CPU path, timed on host cores

Under torchrun every rank solves its own replica of the workload on its GPU
(the solve has no cross-system exchange: replicas only); rank 0 prints one
JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "state*steps/s (RK4 n=64 T=2^20 solve, mixed 3xTF32 form, rel err <= 1e-6 vs FP64)"
UNIT = "state*steps/s"
WORKLOAD = "cfg2: RK4 n=64 m=8 p=8 h=1e-4 T=2^20, seeded system + sum-of-sinusoids input"
# DRAM bytes (read + write) of one launch of the dominant kernel at T = 2^20
# (key: (T, mixed)), from the ncu captures summarised under profiles/.
# serving: the p99 latency the serving loop is specified to hold (cfg5 requests)
SERVE_P99_TARGET_MS = 20.0
DOMINANT_TRAFFIC = {(1 << 20, False): 168.18e6 + 45.27e6, (1 << 20, True): 134.87e6 + 60.82e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--T", type=int, default=1 << 20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--min-warmup-s", type=float, default=0.5, help="least warm-up time under load (clock sampling)")
    ap.add_argument("--no-extra", action="store_true", help="skip the batched (4096 systems) and serving runs")
    ap.add_argument("--time-partition", action="store_true",
                    help="with N > 1 GPUs also time one cfg2 solve split by time over the ranks "
                         "(parode_b200.multi.solve_time_partitioned: one all-gather per solve)")
    ap.add_argument("--serve-requests", type=int, default=256)
    ap.add_argument("--no-tune", action="store_true", help="time with the untuned block length of the response leaf")
    ap.add_argument("--ref-T", type=int, default=1 << 20,
                    help="reference arm: steps of the cfg2 horizon solved per timed step (default: all 2^20)")
    return ap.parse_args()


def bench_config(args, world):
    """The `config` object of both arms' JSON lines (identical by construction)."""
    return {"workload": WORKLOAD, "precision": args.precision,
            "l2": "256 MB flush between timed solves (outside the events)",
            "parallelism": f"replicas x{world}"}


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


# ---------------------------------------------------------------------------
# reference arm: the reference's CPU path (its test harness' sequential RK4
# loop, TestsSources/TestParODEStaticLibCInterface.cpp:158-204), restated in C
# under oracle/ and run on the host cores.
# ---------------------------------------------------------------------------

def rel_err(y, yref):
    """Per output channel max_k |y - yref| / max_k |yref|, maximum over channels
    (the comparison of two of this library's own results, e.g. mixed vs FP64)."""
    y = np.asarray(y, dtype=np.float64)
    yref = np.asarray(yref, dtype=np.float64)
    num = np.max(np.abs(y - yref), axis=0)
    den = np.max(np.abs(yref), axis=0)
    return float(np.max(np.where(den > 0, num / np.where(den > 0, den, 1.0), num)))


def reference_sample(T_sample):
    from oracle import oracle
    from parode_b200 import workloads as wl

    case = wl.cfg2(T=T_sample)
    sysd = oracle.System(case.A, case.B, case.C, case.D, case.x0)
    inp = oracle.Input.sinusoid(case.u.a, case.u.f, case.u.phi)

    def run():
        oracle.stepper(sysd, inp, 0, 0.0, case.h, T_sample, use_float=True)

    return case, run


def cpu_batched_sample(wl):
    """The batched workload's CPU baseline: every 8th cfg4 system (512 of 4096)
    by the FP64 affine recurrence (the oracle's O1), OpenMP across systems on
    all host threads."""
    from oracle import oracle

    sample = wl.cfg4()[::8]
    jobs = [(oracle.System(c.A, c.B, c.C, c.D, c.x0), oracle.Input.sinusoid(c.u.a, c.u.f, c.u.phi), c.solver, c.t0,
             c.t_end, c.h) for c in sample]
    t0 = time.perf_counter()
    ys = oracle.simulate_affine_many(jobs)
    dt = time.perf_counter() - t0
    work = float(sum(c.n * y.shape[0] for c, y in zip(sample, ys)))
    cores = int(oracle.lib().po_threads())
    return {"value": work / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"512 of the 4096 cfg4 systems (every 8th, {work:.3g} state*steps), FP64 affine recurrence, "
                      f"OpenMP across systems, {dt:.1f} s on {cores} host threads"}


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    # each timed step solves the whole cfg2 horizon (2^20 steps, ~8 s on one
    # core), so the line's config is the GPU arm's; --ref-T shortens it
    T_sample = max(1, min(args.ref_T, args.T))
    case, run = reference_sample(T_sample)
    times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        run()
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt)
    per = statistics.mean(times)
    value = case.n * T_sample / per
    sample = (f"cfg2 system (RK4 n=64 m=8 p=8), {T_sample} of its {args.T} steps per timed step; the reference's "
              f"sequential FP32 RK4 test loop restated in C (one system is one sequential chain: 1 thread)")
    config = bench_config(args, world)
    if T_sample < args.T:
        config["sampled_steps_per_step"] = T_sample
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded system and input)",
        "config": config,
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the GPU is busy."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="clocks", suffix=".csv")
        os.close(fd)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            with open(self.path) as fh:
                for ln in fh:
                    parts = [q.strip() for q in ln.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        smax = [v for v in (num(r[2]) for r in rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def gemm_peak_tflops(torch, dev, dtype, tf32=False):
    """Dense GEMM throughput measured here with cuBLAS (torch.matmul)."""
    N = 8192 if dtype != torch.float64 else 4096
    torch.backends.cuda.matmul.allow_tf32 = tf32
    a = torch.randn(N, N, dtype=dtype, device=dev)
    b = torch.randn(N, N, dtype=dtype, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.backends.cuda.matmul.allow_tf32 = False
    return 2.0 * N ** 3 / best / 1e12


def response_flops(case, shape, mixed):
    """Algorithmic FLOPs of one solve on the block-response path, per launch
    kind.  shape = (B, K, NP, blocks) from the plan.  The aggregate GEMM
    costs 2 NP K per block; the output GEMM 2 B p (K + NP) per block (window
    part 2 B p K, initial-state part 2 B p NP); the carry over blocks 4 NP^2
    per block (up- and down-sweep).  The dominant launch is the output GEMM
    in FP64 and, in the mixed form, the tensor-core launch that computes the
    aggregates and the output windows together."""
    B, K, NP, blocks = shape
    p = case.p
    agg, win, state, carry = 2.0 * NP * K * blocks, 2.0 * B * p * K * blocks, 2.0 * B * p * NP * blocks, \
        4.0 * NP * NP * blocks
    dominant = (agg + win) if mixed else (win + state)
    return {"dominant": dominant, "solve": agg + win + state + carry}


def _spec(pb, c):
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    return {"A": c.A, "B": c.B, "C": c.C, "D": c.D, "x0": c.x0, "u": u, "t0": c.t0, "t_end": c.t_end, "h": c.h,
            "solver": c.solver}


def _cheap_sample(cases, k):
    """k systems whose mixed result is compared with the FP64 one: half from
    the scan dimensions <= 64 (blocked path) and half from the larger ones
    (level-synchronous path, where the mixed form runs its tensor-core levels)."""
    cost = lambda i: cases[i].scan_dim ** 2 * cases[i].T
    small = sorted((i for i in range(len(cases)) if cases[i].scan_dim <= 64), key=cost)
    large = sorted((i for i in range(len(cases)) if cases[i].scan_dim > 64), key=cost)
    return small[: k // 2] + large[: k - k // 2]


def _over_ranks(torch, dev, world, value, op="max"):
    """value reduced over the ranks (max or sum); itself on one rank."""
    if world == 1:
        return value
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def measure_batched(pb, wl, torch, dev, reps=3, tune_classes=0, rank=0, world=1):
    """The batched form: 4096 independent systems (cfg4) in one batch, FP64 and
    mixed; on N ranks each solves its cost-balanced shard of the systems
    (parode_b200.multi.shard, no data-path collective) and the time is the
    slowest rank's."""
    from parode_b200 import multi

    cases_all = wl.cfg4()
    cases = [cases_all[i] for i in multi.shard(cases_all, rank, world, multi.system_cost)]
    specs = [_spec(pb, c) for c in cases]
    check = _cheap_sample(cases, 8)
    out = {"workload": "cfg4: 4096 systems, n log-uniform [4,96], T log-uniform [2^10,2^16], RK4/ABM 50/50",
           "state_steps": None, "ranks": world, "systems_on_rank0": len(cases)}
    stream = torch.cuda.Stream(device=dev)
    y64 = {}
    # freed batch memory stays mapped in the device pool: the FP64 batch's
    # set-up is the process's first (pool and pinned staging grown cold), the
    # mixed batch's reuses what the FP64 batch freed, the tuned batch's is the
    # mixed batch set up again
    pb.set_option(pb.OPT_POOL_KEEP, 64 << 30)
    out["setup_note"] = ("fp64.setup_s: first batch set-up of the process (device pool and pinned staging grow); "
                         "mixed.setup_s: after the FP64 batch freed its memory to the pool; "
                         "mixed.setup_again_s: the mixed batch set up again right after")
    for name, prec in (("fp64", pb.FP64), ("mixed", pb.MIXED)):
        t0 = time.perf_counter()
        b = pb.Batch(specs, precision=prec)
        setup_s = time.perf_counter() - t0
        b.execute(stream.cuda_stream)
        b.execute(stream.cuda_stream)  # the second execute captures the launch graph
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            b.execute(stream.cuda_stream)
            e.record(stream)
            e.synchronize()
            ts.append(s.elapsed_time(e))
        ms = statistics.median(ts)
        worst = None
        for i in check:
            _, y = b.output(i)
            if name == "fp64":
                y64[i] = y
            else:
                worst = max(worst or 0.0, rel_err(y, y64[i]))
        ms = _over_ranks(torch, dev, world, ms)
        work = _over_ranks(torch, dev, world, b.state_steps, "sum")
        setup_s = _over_ranks(torch, dev, world, setup_s)
        out["state_steps"] = work
        out[name] = {"ms": ms, "value": work / (ms / 1e3), "unit": UNIT, "launches": b.launch_count,
                     "setup_s": setup_s}
        if worst is not None:
            out[name].update(rel_err_vs_fp64_sampled=worst, sampled_systems=len(check))
        b.close()
        if name == "mixed":
            # the same batch set up again (device pool and pinned staging warm)
            t0 = time.perf_counter()
            b = pb.Batch(specs, precision=prec)  # returns with the device's set-up work queued, as above
            out[name]["setup_again_s"] = _over_ranks(torch, dev, world, time.perf_counter() - t0)
            b.close()
    out["mixed_over_fp64"] = out["fp64"]["ms"] / out["mixed"]["ms"]
    if tune_classes > 0:
        # the block length measured for the classes that carry most of the
        # work (ParODE_TuneResponseBlock), then the mixed batch again
        tuned = tune_batch_classes(pb, cases, pb.MIXED, tune_classes)
        b = pb.Batch(specs, precision=pb.MIXED)
        b.execute(stream.cuda_stream)
        b.execute(stream.cuda_stream)  # the second execute captures the launch graph
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            b.execute(stream.cuda_stream)
            e.record(stream)
            e.synchronize()
            ts.append(s.elapsed_time(e))
        ms = _over_ranks(torch, dev, world, statistics.median(ts))
        out["mixed_tuned"] = {"ms": ms, "value": out["state_steps"] / (ms / 1e3), "unit": UNIT,
                              "launches": b.launch_count,
                              "classes_tuned": len(tuned), "share_of_work_tuned": sum(w for _, w in tuned),
                              "gain_over_untuned": out["mixed"]["ms"] / ms}
        b.close()
        pb.tune_clear()
    pb.set_option(pb.OPT_POOL_KEEP, 0)
    return out


def _tune_key(c):
    pw = lambda v: 1 << max(0, int(v - 1).bit_length())
    ns = c.scan_dim
    nscan = c.T if c.solver == 0 else c.T - 3
    return (c.solver, pw(max(8, ns)), pw(c.m), pw(c.p), max(0, int(nscan - 1).bit_length()))


def tune_batch_classes(pb, cases, precision, count):
    """Tunes the `count` classes of systems with the most state*steps; returns
    [(class, share of the batch's state*steps)]."""
    work, rep = {}, {}
    for c in cases:
        k = _tune_key(c)
        work[k] = work.get(k, 0.0) + c.n * c.T
        if k not in rep or c.n * c.T > rep[k].n * rep[k].T:
            rep[k] = c
    total = sum(work.values())
    top = sorted(work, key=lambda k: -work[k])[:count]
    for k in top:
        c = rep[k]
        pb.tune_response_block(c.solver, c.n, c.m, c.p, c.T, precision)
    return [(k, work[k] / total) for k in top]


def measure_cfg1(pb, wl, torch, reps=200):
    """The small single solve (cfg1: RK4 n=8 m=2 p=2, T=4096): latency of
    one execute (CUDA events, inputs resident) and of the whole C-ABI call
    with host buffers, as p50 / p99 over `reps` solves."""
    c = wl.cfg1()
    u = pb.register_sinusoid(c.u.a, c.u.f, c.u.phi)
    plan = pb.Plan(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver)
    stream = torch.cuda.Stream()
    for _ in range(10):
        plan.execute(0, stream.cuda_stream)
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        plan.execute(0, stream.cuda_stream)
        e.record(stream)
        e.synchronize()
        ts.append(s.elapsed_time(e))
    launches = plan.launch_count
    plan.close()
    T_out = pb.num_outputs(c.solver, c.t0, c.t_end, c.h)
    t_host = torch.empty(T_out, dtype=torch.float64, pin_memory=True).numpy()
    y_host = torch.empty((T_out, c.p), dtype=torch.float64, pin_memory=True).numpy()
    es = []
    for it in range(reps // 4 + 5):
        t0 = time.perf_counter()
        pb.simulate(c.A, c.B, c.C, c.D, c.x0, u, c.t0, c.t_end, c.h, solver=c.solver, t_out=t_host, y_out=y_host)
        if it >= 5:
            es.append((time.perf_counter() - t0) * 1e3)
    return {"workload": "cfg1: RK4 n=8 m=2 p=2 h=1e-3 T=4096", "precision": "fp64", "launches": launches,
            "solve_ms": {"p50": float(np.percentile(ts, 50)), "p99": float(np.percentile(ts, 99))},
            "value": c.n * c.T / (float(np.percentile(ts, 50)) / 1e3), "unit": UNIT,
            "e2e_ms": {"p50": float(np.percentile(es, 50)), "p99": float(np.percentile(es, 99))}}


def measure_cfg3(pb, wl, torch, reps=3):
    """ABM4, n=128 (scan dimension 512), m=p=16, h=5e-4, T=2^18: the level-
    synchronous path, FP64 and mixed (one-system batch), rel err mixed vs FP64."""

    c = wl.cfg3()
    out = {"workload": "cfg3: ABM4 n=128 (N_s=512) m=p=16 h=5e-4 T=2^18"}
    stream = torch.cuda.Stream()
    ys = {}
    for name, prec in (("fp64", pb.FP64), ("mixed", pb.MIXED)):
        b = pb.Batch([_spec(pb, c)], precision=prec)
        b.execute(stream.cuda_stream)
        b.execute(stream.cuda_stream)  # the second execute captures the launch graph
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            b.execute(stream.cuda_stream)
            e.record(stream)
            e.synchronize()
            ts.append(s.elapsed_time(e))
        ms = statistics.median(ts)
        ys[name] = b.output(0)[1]
        flops = 4.0 * c.scan_dim ** 2 * c.T
        out[name] = {"ms": ms, "value": b.state_steps / (ms / 1e3), "unit": UNIT,
                     "sweep_tflops": flops / (ms / 1e3) / 1e12, "launches": b.launch_count}
        b.close()
    out["mixed_over_fp64"] = out["fp64"]["ms"] / out["mixed"]["ms"]
    out["rel_err_mixed_vs_fp64"] = rel_err(ys["mixed"], ys["fp64"])
    return out


def measure_serving(pb, wl, torch, count=64, rates=(500.0, 1000.0, 2000.0, 8000.0), dev=None, rank=0, world=1):
    """The serving loop on cfg5-shaped requests (Poisson arrivals), mixed form,
    beside one offline batch of the same requests.  On N ranks each serves its
    share of every request stream (round robin in arrival order) with its own
    server; latencies are the worst rank's percentiles, throughput the summed
    work over the longest span."""
    from parode_b200 import multi

    out = {"workload": f"cfg5: {count} requests per rate, n log-uniform [8,256], T log-uniform [1e3,1e6], "
                       f"RK4/ABM 50/50, Poisson arrivals", "budget_bytes": 150e9, "precision": "mixed",
           "rates": {}}
    reqs_all = {}
    for rate in rates:
        reqs = wl.cfg5(count, rate)
        reqs = [reqs[i] for i in multi.shard(reqs, rank, world)]
        reqs_all[rate] = reqs
        server = pb.Server(precision=pb.MIXED, hbm_budget_bytes=150e9, max_batch=32, max_inflight=8)
        specs = [(arr, c, _spec(pb, c)) for arr, c in reqs]
        ids = []
        t0 = time.monotonic()
        for arr, c, s in specs:
            d = t0 + arr - time.monotonic()
            if d > 0:
                time.sleep(d)
            ids.append(server.submit(s["A"], s["B"], s["C"], s["D"], s["x0"], s["u"], s["t0"], s["t_end"], s["h"],
                                     solver=s["solver"]))
        for rid in ids:
            server.wait(rid, timeout_s=600)
        st = server.stats()
        server.close()
        red = {k: _over_ranks(torch, dev, world, st[k]) for k in ("p50_ms", "p99_ms", "mean_ms", "span_s", "peak_bytes")}
        work = _over_ranks(torch, dev, world, st["state_steps"], "sum")
        batches = _over_ranks(torch, dev, world, st["batches"], "sum")
        out["rates"][str(int(rate))] = {"p50_ms": red["p50_ms"], "p99_ms": red["p99_ms"], "mean_ms": red["mean_ms"],
                                        "value": work / red["span_s"] if red["span_s"] else None,
                                        "unit": UNIT, "batches": int(batches),
                                        "peak_gb": red["peak_bytes"] / 1e9, "span_s": red["span_s"]}
    # offline: all requests of the middle rate in one batch (set-up excluded and included)
    reqs = reqs_all[rates[len(rates) // 2]]
    t0 = time.perf_counter()
    b = pb.Batch([_spec(pb, c) for _, c in reqs], precision=pb.MIXED)
    setup = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    b.execute(stream.cuda_stream)
    b.execute(stream.cuda_stream)  # the second execute captures the launch graph
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    b.execute(stream.cuda_stream)
    e.record(stream)
    e.synchronize()
    ms = _over_ranks(torch, dev, world, s.elapsed_time(e))
    setup = _over_ranks(torch, dev, world, setup)
    work = _over_ranks(torch, dev, world, b.state_steps, "sum")
    out["offline"] = {"value": work / (ms / 1e3), "value_with_setup": work / (ms / 1e3 + setup),
                      "unit": UNIT, "ms": ms, "setup_s": setup}
    b.close()
    # the stated latency target: the highest measured arrival rate whose p99
    # stays within it
    held = [r for r in rates if out["rates"][str(int(r))]["p99_ms"] <= SERVE_P99_TARGET_MS]
    out["p99_target_ms"] = SERVE_P99_TARGET_MS
    out["highest_rate_holding_p99_target"] = max(held) if held else None
    mid = out["rates"][str(int(rates[len(rates) // 2]))]
    # against the offline batch's execute alone, and against the offline batch
    # with its set-up (discretisation, W, arena), which every served request pays
    out["serving_over_offline"] = (mid["value"] / out["offline"]["value"]) if mid["value"] else None
    out["serving_over_offline_with_setup"] = (mid["value"] / out["offline"]["value_with_setup"]) if mid["value"] else None
    return out


def measure_time_partition(pb, torch, dev, case, u, precision, steps):
    """One cfg2 solve split by time over all ranks (strong scaling of a single
    system): each rank's shard plan, its up phase, one NCCL all-gather of the
    shards' chunk aggregates, its down phase; the slowest rank's time."""
    import torch.distributed as dist

    rank, world = dist.get_rank(), dist.get_world_size()
    plan = pb.Plan(case.A, case.B, case.C, case.D, case.x0, u, case.t0, case.t_end, case.h, solver=case.solver,
                   precision=precision, shard=rank, shards=world)
    _, steps_local, c, np_, _ = plan.shard_info
    top = torch.zeros(c * np_, dtype=torch.float64, device=dev)
    gathered = torch.empty(world * c * np_, dtype=torch.float64, device=dev)
    y = torch.empty((plan.num_outputs, plan.channels), dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream(dev)

    def solve():
        plan.shard_up(top.data_ptr(), s.cuda_stream)
        dist.all_gather_into_tensor(gathered, top)
        plan.shard_down(gathered.data_ptr(), y.data_ptr(), s.cuda_stream)

    for _ in range(3):
        solve()
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(steps):
        solve()
    e1.record(s)
    torch.cuda.synchronize()
    ms = torch.tensor([e0.elapsed_time(e1) / steps], dtype=torch.float64, device=dev)
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    plan.close()
    ms = float(ms.item())
    return {"workload": "cfg2 split by time over the ranks", "ms_per_solve": ms, "ranks": world,
            "steps_on_rank0": steps_local, "value": case.n * case.T / (ms / 1e3), "unit": UNIT,
            "scaling": "strong"}


def run_ours(args):
    import torch

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        import datetime
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    import parode_b200 as pb
    from parode_b200 import workloads as wl

    pb.init([local_rank])
    case = wl.cfg2(T=args.T)
    u = pb.register_sinusoid(case.u.a, case.u.f, case.u.phi)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    clk = ClockSampler(local_rank)

    def time_plan(precision, sample_clocks):
        plan = pb.Plan(case.A, case.B, case.C, case.D, case.x0, u, case.t0, case.t_end, case.h,
                       solver=case.solver, precision=precision)
        y = torch.empty((plan.num_outputs, plan.channels), dtype=torch.float64, device=dev)
        run = lambda: plan.execute(y.data_ptr(), stream.cuda_stream)
        if sample_clocks:
            clk.start()  # sampled through the warm-up and the timed region, both under load
        with torch.cuda.stream(stream):
            t_end = time.perf_counter() + args.min_warmup_s  # warm-up under load, sampled by the clock monitor
            it = 0
            while it < args.warmup or time.perf_counter() < t_end:
                run()
                flush.zero_()
                it += 1
                if it % 8 == 0:
                    stream.synchronize()
        torch.cuda.synchronize()
        plan.set_profiling(True)
        with torch.cuda.stream(stream):
            run()
        stages = dict(plan.stage_times())
        plan.set_profiling(False)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        pairs = []
        with torch.cuda.stream(stream):
            for _ in range(args.steps):
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record(stream)
                run()
                e.record(stream)
                flush.zero_()  # L2 flush between timed solves, outside the events
                pairs.append((s, e))
        torch.cuda.synchronize()
        if sample_clocks:
            clk.stop()
        if world > 1:
            torch.distributed.barrier()
        total = torch.tensor([sum(s.elapsed_time(e) for s, e in pairs)], dtype=torch.float64, device=dev)
        if world > 1:
            torch.distributed.all_reduce(total, op=torch.distributed.ReduceOp.MAX)
        per = sorted(s.elapsed_time(e) for s, e in pairs)
        info = {"ms_per_step": float(total.item()) / args.steps, "stages_ms": stages, "launches": plan.launch_count,
                "solve_ms": {"p50": float(np.percentile(per, 50)), "p99": float(np.percentile(per, 99))},
                "precision_used": plan.precision, "path": plan.path, "response_shape": plan.response_shape}
        y_host = y.cpu().numpy()
        plan.close()
        return info, y_host

    precision = pb.MIXED if args.precision == "mixed" else pb.FP64
    # the response leaf's block length measured for this class of systems
    # (ParODE_TuneResponseBlock); the plans below use it
    tuner = None
    if not args.no_tune:
        tuner = {}
        for name, prec in (("mixed", pb.MIXED), ("fp64", pb.FP64)):
            if name == "fp64" and args.no_plain and precision != pb.FP64:
                continue
            R, best, untuned = pb.tune_response_block(case.solver, case.n, case.m, case.p, case.T, prec)
            tuner[name] = {"block": 1 << R, "ms_tuned": best, "ms_untuned": untuned, "gain": untuned / best}
    main, y_main = time_plan(precision, True)
    plain, y_plain = (None, None)
    if not args.no_plain and precision != pb.FP64:
        plain, y_plain = time_plan(pb.FP64, False)
    # the single-pass TF32 form of the same solve (operands rounded to TF32 once)
    single = None
    if not args.no_plain and precision == pb.MIXED:
        single, y_single = time_plan(pb.TF32, False)
        single["rel_err_vs_fp64"] = None
        if y_plain is not None:
            single["rel_err_vs_fp64"] = rel_err(y_single, y_plain)
        single["value"] = world * case.n * case.T / (single["ms_per_step"] / 1e3)
        del y_single
    value = world * case.n * case.T / (main["ms_per_step"] / 1e3)

    # e2e: the reference's C-ABI call with host buffers (plan set-up, H2D,
    # solve, D2H of y into host arrays the caller keeps across calls, pinned):
    # SimulateODE with its float arrays (fType), the precision mode set by
    # PARODE_OPT_PRECISION; beside it the FP64 extension ParODE_SimulateODE_d
    def time_calls(call):
        ms = []
        # 1 warm-up + 7 timed calls; the median, since the host side (page
        # cache, other processes on the host cores) adds outliers of 10-600 ms
        for it in range(1 + 7):
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            call()
            e.record()
            e.synchronize()
            if it > 0:
                ms.append(s.elapsed_time(e))
        t_ = torch.tensor([statistics.median(ms)], dtype=torch.float64, device=dev)
        if world > 1:
            torch.distributed.all_reduce(t_, op=torch.distributed.ReduceOp.MAX)
        return float(t_.item()), ms

    e2e = None
    e2e_f64 = None
    if not args.no_e2e:
        T_out = pb.num_outputs(case.solver, case.t0, case.t_end, case.h)
        t32 = torch.empty(T_out, dtype=torch.float32, pin_memory=True).numpy()
        y32 = torch.empty((T_out, case.p), dtype=torch.float32, pin_memory=True).numpy()
        prev = pb.get_option(pb.OPT_PRECISION)
        pb.set_option(pb.OPT_PRECISION, precision)
        try:
            def call32():
                _, _, err = pb.simulate_f32(case.A, case.B, case.C, case.D, case.x0, u, case.t0, case.t_end, case.h,
                                            solver=case.solver, t_out=t32, y_out=y32)
                if err != 0:
                    raise RuntimeError(f"SimulateODE error {err}")
            med, ms = time_calls(call32)
        finally:
            pb.set_option(pb.OPT_PRECISION, prev)
        h2d = 4 * (case.A.size + case.B.size + case.C.size + case.D.size + case.x0.size) + 8 * 3 * case.u.a.size
        d2h = 4 * case.T * case.p
        e2e = {"value": world * case.n * case.T / (med / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "ms_per_step": med,
               "statistic": f"median of {len(ms)} calls", "mean_ms": statistics.mean(ms), "max_ms": max(ms),
               "call": "SimulateODE, the reference's C ABI (float arrays in, t and y out into pinned host memory "
                       "reused across calls; y rounded to float on the device and copied out in four block ranges, "
                       "each while the later ones are formed), precision mode mixed"}
        t64 = torch.empty(T_out, dtype=torch.float64, pin_memory=True).numpy()
        y64 = torch.empty((T_out, case.p), dtype=torch.float64, pin_memory=True).numpy()
        med, ms = time_calls(lambda: pb.simulate(case.A, case.B, case.C, case.D, case.x0, u, case.t0, case.t_end,
                                                 case.h, solver=case.solver, precision=precision, t_out=t64, y_out=y64))
        e2e_f64 = {"value": world * case.n * case.T / (med / 1e3), "unit": UNIT, "ms_per_step": med,
                   "h2d_bytes_per_step": int(8 * (case.A.size + case.B.size + case.C.size + case.D.size +
                                                  case.x0.size + 3 * case.u.a.size)),
                   "d2h_bytes_per_step": int(2 * d2h), "statistic": f"median of {len(ms)} calls",
                   "call": "ParODE_SimulateODE_d (double arrays in, y out into pinned host memory reused across calls, "
                           "in four block ranges as above)"}

    # the e2e call's parts, each timed on its own: plan creation (host
    # discretisation, W and power tables on the device), the solve, the copy
    # of y into pinned host memory, the host time vector
    e2e_split = None
    if not args.no_e2e:
        T_out = pb.num_outputs(case.solver, case.t0, case.t_end, case.h)
        t_host = torch.empty(T_out, dtype=torch.float64, pin_memory=True).numpy()
        y_host = torch.empty((T_out, case.p), dtype=torch.float64, pin_memory=True).numpy()
        parts = {"plan_ms": [], "solve_ms": [], "copy_ms": []}
        for it in range(4):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            plan = pb.Plan(case.A, case.B, case.C, case.D, case.x0, u, case.t0, case.t_end, case.h,
                           solver=case.solver, precision=precision)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            plan.execute()
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            plan.output(t_out=t_host, y_out=y_host)  # y by DMA while the host builds t
            t3 = time.perf_counter()
            plan.close()
            if it > 0:
                parts["plan_ms"].append((t1 - t0) * 1e3)
                parts["solve_ms"].append((t2 - t1) * 1e3)
                parts["copy_ms"].append((t3 - t2) * 1e3)
        med = {k: statistics.median(v) for k, v in parts.items()}
        e2e_split = dict(med, d2h_gbs=8.0 * case.T * case.p / (med["copy_ms"] / 1e3) / 1e9,
                         note="parts timed separately with host clocks (synchronised), the copy as one piece after "
                              "the solve; the e2e call overlaps the host time vector with plan creation, the solve "
                              "and the copy, and each output range's copy with the forming of the later ranges")
    cfg1 = measure_cfg1(pb, wl, torch) if world == 1 and not args.no_extra else None
    tpart = measure_time_partition(pb, torch, dev, case, u, precision, args.steps) \
        if (world > 1 and args.time_partition) else None

    batched = serving = cfg3 = None
    if not args.no_extra:
        # independent systems shard across the ranks (no data-path collective)
        batched = measure_batched(pb, wl, torch, dev, tune_classes=0 if args.no_tune else 16, rank=rank, world=world)
        if world == 1:
            cfg3 = measure_cfg3(pb, wl, torch)
        serving = measure_serving(pb, wl, torch, count=args.serve_requests, dev=dev, rank=rank, world=world)

    if rank == 0:
        peaks, peaks_kind = measured_peaks()
        used_mixed = main["precision_used"] == pb.MIXED
        fl = response_flops(case, main["response_shape"], used_mixed) if main["path"] == 3 else None
        stage = "aggregates+windows" if used_mixed else "outputs"
        dom_ms = main["stages_ms"].get(stage)
        tf32_run = None
        if used_mixed:
            # dense TF32 is half the bf16 rate; 3xTF32 spends three tensor
            # products per algorithmic product
            peak = peaks["bf16_tflops"] / 2.0 / 3.0
            tf32_run = gemm_peak_tflops(torch, dev, torch.float32, tf32=True)
            peak_src = (f"MEASURED_PEAKS.json bf16_tflops ({peaks['bf16_tflops']:.1f}, {peaks_kind}) / 2 (dense TF32) "
                        f"/ 3 (three products per 3xTF32 product); cuBLAS TF32 measured in this run: "
                        f"{tf32_run:.0f} TFLOP/s")
        else:
            peak = gemm_peak_tflops(torch, dev, torch.float64)
            peak_src = "dense FP64 GEMM measured in this run (cuBLAS DGEMM via torch.matmul)"
        achieved = fl["dominant"] / (dom_ms / 1e3) / 1e12 if (fl and dom_ms) else None
        roofline = {"bound": "tensor",
                    "kernel": ("k_resp_tc: 3xTF32 tcgen05 GEMMs of the block aggregates and output windows"
                               if used_mixed else "k_level_tiled: FP64 DMMA output GEMM y = W [window; X_b]"),
                    "stage": stage, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": (achieved / peak) if achieved else None, "peak_source": peak_src,
                    "algorithmic_flops_per_launch": fl["dominant"] if fl else None,
                    "traffic": DOMINANT_TRAFFIC.get((case.T, used_mixed)),
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch (profiles/)",
                    "stages_ms": main["stages_ms"],
                    "whole_solve_tflops": fl["solve"] / (main["ms_per_step"] / 1e3) / 1e12 if fl else None}
        rel_vs_fp64 = None
        if y_plain is not None:
            rel_vs_fp64 = rel_err(y_main, y_plain)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            T_cpu = 1 << 20
            c2, run = reference_sample(T_cpu)
            t0 = time.perf_counter()
            run()
            dt = time.perf_counter() - t0
            cpu = {"value": c2.n * T_cpu / dt, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"the reference's CPU path (its tests' sequential FP32 RK4 loop, restated in C) on the "
                             f"full cfg2 horizon, {T_cpu} steps in {dt:.1f} s on 1 host core"}
            if not args.no_extra:
                cpu["batched"] = cpu_batched_sample(wl)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": main["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "tf32x3+f64" if used_mixed else "f64", "data": "synthetic (seeded system and input)",
            "config": bench_config(args, world),
            "precision_used": "mixed" if used_mixed else "fp64",
            "path": {1: "level-synchronous", 2: "blocked, in-block sweeps",
                     3: "blocked, block-response GEMMs"}.get(main["path"], "?"),
            "gpu_launches": main["launches"] * args.steps, "solve_ms": main["solve_ms"],
            "clocks": clk.summary(), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "plain_fp64": None if plain is None else {
                "value": world * case.n * case.T / (plain["ms_per_step"] / 1e3), "ms_per_step": plain["ms_per_step"],
                "stages_ms": plain["stages_ms"],
                "output_gemm_tflops": (response_flops(case, plain["response_shape"], False)["dominant"] /
                                       (plain["stages_ms"]["outputs"] / 1e3) / 1e12)
                if plain["path"] == 3 and plain["stages_ms"].get("outputs") else None},
            "mixed_over_plain": None if plain is None else plain["ms_per_step"] / main["ms_per_step"],
            "tf32_single_pass": None if single is None else {
                k: single[k] for k in ("value", "ms_per_step", "stages_ms", "precision_used", "rel_err_vs_fp64")},
            "rel_err_mixed_vs_fp64": rel_vs_fp64,
            "peaks": {k: peaks.get(k) for k in ("hbm_gbs", "bf16_tflops", "bf16_tflops_sustained")},
            "peaks_source": peaks_kind,
            "tuner": tuner,
            "e2e_split": e2e_split,
            "e2e_f64": e2e_f64,
            "cfg1": cfg1,
            "batched": batched,
            "serving": serving,
            "abm_n128": cfg3,
            "time_partitioned": tpart,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
