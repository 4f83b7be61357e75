#!/usr/bin/env python3
"""Benchmark of the batched 1D FFT hot path on B200.

Default workload (the configuration the headline metric is quoted on):
plain C2C FP32 forward, N=1024, batch=4096, unit stride, contiguous,
out-of-place, no scaling; re/im i.i.d. U[-1,1) from a seed.

  python bench.py --gpus N --steps K --warmup W [--impl reference]

One JSON line on rank 0.  `value` = algorithmic GB/s (one read of the input
+ one write of the output per transform) over all ranks, device-timed with
CUDA events on the launching stream, max over ranks.  Inputs rotate over
buffer sets whose total size exceeds L2 so no step starts L2-warm.
`e2e` = the same metric through plfft_plan_execute() on pinned host buffers
(host->device and device->host copies inside the timed region).
`--impl reference` times the CPU implementation of the path (the FP64 port
of the reference's transform definitions, `oracle/`; the reference itself is
AArch64-only and cannot be built on this x86_64 host).
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "perf-libs-fft_b200"))

WORKLOADS = {
    "c2c_n1024_b4096": dict(kind="c2c", n=1024, batch=4096, desc="plain C2C FP32 forward N=1024 batch=4096"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2c_n1024_b4096", choices=list(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def algo_bytes(w):
    n, b = w["n"], w["batch"]
    if w["kind"] == "c2c":
        return 2 * n * b * 8
    raise ValueError(w["kind"])


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """dram bytes per launch from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the workload runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference(w, steps, warmup, sample_transforms):
    """Time the FP64 CPU port (oracle) on a bounded sample of the workload."""
    import numpy as np

    import oracle

    threads = oracle.max_threads()
    n = w["n"]
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, (sample_transforms, n)) + 1j * rng.uniform(-1, 1, (sample_transforms, n))
    for _ in range(warmup):
        oracle.c2c(x, -1, method="fft", threads=threads)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        oracle.c2c(x, -1, method="fft", threads=threads)
        times.append(time.perf_counter() - t0)
    per_step = sum(times) / len(times)
    gbs = 2 * n * sample_transforms * 8 / per_step / 1e9
    return gbs, threads, per_step


def main():
    args = parse()
    w = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    n, batch = w["n"], w["batch"]
    config = {"workload": w["desc"], "n": n, "batch": batch, "layout": "unit stride, contiguous, out-of-place",
              "l2": "inputs rotate over buffer sets totalling > 4x L2", "parallelism": f"batch-replica x{args.gpus}"}

    if args.impl == "reference":
        if rank != 0:
            return
        sample = 256
        gbs, threads, per_step = cpu_reference(w, max(1, min(args.steps, 20)), min(args.warmup, 3), sample)
        line = {"metric": "batched C2C FP32 GB/s (algorithmic bytes)", "value": gbs, "unit": "GB/s",
                "impl": "reference", "n_gpus": args.gpus, "steps": max(1, min(args.steps, 20)),
                "warmup": min(args.warmup, 3), "ms_per_step": per_step * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded U[-1,1))",
                "config": config,
                "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": threads, "kind": "port",
                                 "sample": f"{sample} of {batch} transforms per step, FP64 mixed-radix FFT port of "
                                           "the reference conventions (the reference is AArch64-only and does not "
                                           "build on this x86_64 host)"},
                "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import numpy as np
    import torch

    import plfft

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    plan = plfft.make_plan("c2c", n, batch, direction=plfft.FORWARD)
    launches = plan.launch_count()
    abytes = algo_bytes(w)
    l2 = 126 << 20
    sets = max(2, int(np.ceil(4 * l2 / abytes)))
    g = torch.Generator(device="cuda")
    g.manual_seed(1234 + rank)
    ins, outs = [], []
    for _ in range(sets):
        re_ = torch.rand(batch * n, device="cuda", generator=g) * 2 - 1
        im_ = torch.rand(batch * n, device="cuda", generator=g) * 2 - 1
        ins.append(torch.complex(re_, im_))
        outs.append(torch.empty(batch * n, dtype=torch.complex64, device="cuda"))
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    ws = torch.empty(max(1, plan.workspace_size()), dtype=torch.uint8, device="cuda")

    sampler = ClockSampler(local)
    sampler.start()
    for i in range(args.warmup):
        plan.execute_async(ins[i % sets].data_ptr(), outs[i % sets].data_ptr(), ws.data_ptr(), sh)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for i in range(args.steps):
        plan.execute_async(ins[i % sets].data_ptr(), outs[i % sets].data_ptr(), ws.data_ptr(), sh)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    # per-launch duration of the dominant kernel (one launch per step here)
    kev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * min(args.steps, 50))]
    for i in range(len(kev) // 2):
        kev[2 * i].record(stream)
        plan.execute_async(ins[i % sets].data_ptr(), outs[i % sets].data_ptr(), ws.data_ptr(), sh)
        kev[2 * i + 1].record(stream)
    torch.cuda.synchronize()
    kms = [kev[2 * i].elapsed_time(kev[2 * i + 1]) for i in range(len(kev) // 2)]
    kernel_ms = statistics.median(kms) / launches

    # end to end through the public API on pinned host buffers
    hx = ins[0].cpu().pin_memory()
    hy = torch.empty(batch * n, dtype=torch.complex64).pin_memory()
    plan.execute(hx.data_ptr(), hy.data_ptr())  # warm the staging buffers
    e2e_steps = max(3, min(args.steps, 20))
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(torch.cuda.default_stream())
    for _ in range(e2e_steps):
        plan.execute(hx.data_ptr(), hy.data_ptr())
    e1.record(torch.cuda.default_stream())
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    clocks = sampler.stop()

    if dist is not None:
        t = torch.tensor([ms, e2e_ms, kernel_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms, kernel_ms = [float(v) for v in t.tolist()]

    ms_per_step = ms / args.steps
    value = abytes * world / (ms_per_step * 1e-3) / 1e9
    peak, peak_kind = peaks()
    achieved = abytes / launches / (kernel_ms * 1e-3) / 1e9
    traffic = profile_traffic("c2c_reg_n1024_b4096")

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        sample = 256
        gbs, threads, _ = cpu_reference(w, 10, 2, sample)
        cpu = {"value": gbs, "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"{sample} of {batch} transforms, FP64 mixed-radix FFT port (oracle/), 10 timed reps"}

    if rank == 0:
        line = {
            "metric": "batched C2C FP32 GB/s (algorithmic bytes)", "value": value, "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded U[-1,1) re/im)", "config": config,
            "gflops": 5 * n * np.log2(n) * batch * world / (ms_per_step * 1e-3) / 1e9,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                         "kernel_ms": kernel_ms, "algorithmic_bytes_per_launch": abytes // launches},
            "e2e": {"value": abytes * world / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s",
                    "h2d_bytes_per_step": batch * n * 8, "d2h_bytes_per_step": batch * n * 8,
                    "ms_per_step": e2e_ms, "api": "plfft_plan_execute(host pinned buffers)"},
            "gpu_launches": launches * args.steps,
            "plan": plan.describe(),
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    plan.destroy()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
