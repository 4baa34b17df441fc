"""Benchmark of the parallel-in-time LTI scan (ParODE hot path) on B200.

Workload (one step = one full solve): RK4, n=64 states, m=8 inputs, p=8
outputs, h=1e-4, T=2^20 steps, seeded synthetic system and sum-of-sinusoids
input (parode_b200/workloads.py: cfg2).  Metric: state*steps/s = n*T per solve
/ solve time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
  python bench.py --impl reference ...   # the reference's CPU path, timed on host cores

Under torchrun every rank solves its own replica of the workload on its GPU
(the path has no cross-system exchange: replicas only); rank 0 prints one
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

METRIC = "state*steps/s (RK4 n=64 T=2^20 solve, rel err <= 1e-6 vs FP64 oracle)"
UNIT = "state*steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "mixed", "fp64"])
    ap.add_argument("--T", type=int, default=1 << 20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


# ---------------------------------------------------------------------------
# reference arm: the reference's CPU path (its test harness' sequential RK4
# loop, TestsSources/TestParODEStaticLibCInterface.cpp:158-204), restated in C
# under oracle/ and run on the host cores.
# ---------------------------------------------------------------------------

def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    from oracle import oracle
    from parode_b200 import workloads as wl

    T_sample = 1 << 16
    case = wl.cfg2(T=T_sample)
    sysd = oracle.System(case.A, case.B, case.C, case.D, case.x0)
    inp = oracle.Input.sinusoid(case.u.a, case.u.f, case.u.phi)
    times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.stepper(sysd, inp, 0, 0.0, case.h, T_sample, use_float=True)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt)
    per = statistics.mean(times)
    value = case.n * T_sample / per
    sample = f"cfg2 system, first {T_sample} of 2^20 steps per step; sequential FP32 RK4 loop (1 system => 1 thread)"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "RK4 n=64 m=8 p=8 h=1e-4 T=2^20 (sampled)", "sample_steps": T_sample},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
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
                    parts = [p.strip() for p in ln.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
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


def fp64_peak_tflops(torch, dev):
    """FP64 tensor throughput measured here with a cuBLAS DGEMM (torch.matmul)."""
    N = 4096
    a = torch.randn(N, N, dtype=torch.float64, device=dev)
    b = torch.randn(N, N, dtype=torch.float64, device=dev)
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
    return 2.0 * N ** 3 / best / 1e12


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
    precision = {"auto": pb.FP64, "mixed": pb.MIXED, "fp64": pb.FP64}[args.precision]
    case = wl.cfg2(T=args.T)
    u = pb.register_sinusoid(case.u.a, case.u.f, case.u.phi)
    plan = pb.Plan(case.A, case.B, case.C, case.D, case.x0, u, case.t0, case.t_end, case.h, solver=case.solver,
                   precision=precision)
    T, p, n = plan.num_outputs, plan.channels, case.n
    stream = torch.cuda.Stream(device=dev)
    y_dev = torch.empty((T, p), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def one(prof=False):
        plan.execute(y_dev.data_ptr(), stream.cuda_stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            one()
            flush.zero_()
    torch.cuda.synchronize()

    # stage split of one solve (CUDA events inside the library, same stream)
    plan.set_profiling(True)
    with torch.cuda.stream(stream):
        one()
    stages = plan.stage_times()
    plan.set_profiling(False)
    torch.cuda.synchronize()

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    step_ms = []
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            for _ in range(args.steps):
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record(stream)
                one()
                e.record(stream)
                flush.zero_()  # L2 flush between timed solves, outside the events
                step_ms.append((s, e))
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ms = [s.elapsed_time(e) for s, e in step_ms]
    total_ms = float(sum(ms))
    clocks = clk.summary()

    # parity of the timed configuration against the last result
    _, y_host = None, y_dev.cpu().numpy()

    total = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(total, op=torch.distributed.ReduceOp.MAX)
    total_ms = float(total.item())
    value = world * n * case.T * args.steps / (total_ms / 1e3)

    # e2e: the C-ABI call with host buffers (plan set-up, H2D, solve, D2H of y)
    e2e = None
    if not args.no_e2e:
        A, B, Cm, D, x0 = case.A, case.B, case.C, case.D, case.x0
        e2e_ms = []
        for it in range(1 + max(1, min(args.steps, 3))):
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            _, y_e2e = pb.simulate(A, B, Cm, D, x0, u, case.t0, case.t_end, case.h, solver=case.solver,
                                   precision=precision)
            e.record()
            e.synchronize()
            if it > 0:
                e2e_ms.append(s.elapsed_time(e))
        e2e_t = torch.tensor([statistics.mean(e2e_ms)], dtype=torch.float64, device=dev)
        if world > 1:
            torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
        h2d = 8 * (A.size + B.size + Cm.size + D.size + x0.size + 3 * case.u.a.size)
        d2h = 8 * T * p
        e2e = {"value": world * n * case.T / (float(e2e_t.item()) / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "ms_per_step": float(e2e_t.item())}

    line = None
    if rank == 0:
        peaks, peaks_kind = measured_peaks()
        fp64_tf = fp64_peak_tflops(torch, dev)
        st = dict(stages)
        sweep_ms = st.get("sweeps", total_ms / args.steps)
        Ns = case.scan_dim
        flops_sweep = 4.0 * Ns * Ns * case.T  # up + down vector sweeps (algorithmic)
        achieved = flops_sweep / (sweep_ms / 1e3) / 1e12
        roofline = {"bound": "tensor", "kernel": "affine-level sweeps (DMMA FP64)", "achieved": achieved,
                    "peak": fp64_tf, "unit": "TFLOP/s", "frac": achieved / fp64_tf,
                    "peak_source": "FP64 DGEMM measured in this run (torch.matmul float64 4096^3)",
                    "traffic": None, "stages_ms": st}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            from oracle import oracle

            T_cpu = 1 << 20
            c2 = wl.cfg2(T=T_cpu)
            sysd = oracle.System(c2.A, c2.B, c2.C, c2.D, c2.x0)
            inp = oracle.Input.sinusoid(c2.u.a, c2.u.f, c2.u.phi)
            t0 = time.perf_counter()
            oracle.stepper(sysd, inp, 0, 0.0, c2.h, T_cpu, use_float=True)
            dt = time.perf_counter() - t0
            cpu = {"value": c2.n * T_cpu / dt, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"reference CPU path (sequential FP32 RK4 loop of the reference tests) on cfg2, "
                             f"{T_cpu} steps, {dt:.1f} s"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if precision == pb.FP64 else "tf32x3+f64",
            "data": "synthetic",
            "config": {"workload": "cfg2: RK4 n=64 m=8 p=8 h=1e-4 T=2^20, seeded system + sinusoid input",
                       "precision": "fp64" if precision == pb.FP64 else "mixed", "path": plan_path_name(pb),
                       "l2": "256 MB flush between timed solves", "parallelism": f"replicas x{world}"},
            "gpu_launches": plan.launch_count * args.steps,
            "clocks": clocks, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "peaks": {k: peaks.get(k) for k in ("hbm_gbs", "bf16_tflops", "bf16_tflops_sustained")},
            "peaks_source": peaks_kind,
        }
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def plan_path_name(pb):
    return {0: "auto", 1: "level-synchronous", 2: "blocked"}.get(pb.get_option(pb.OPT_PATH), "?")


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
