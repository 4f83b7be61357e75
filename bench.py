#!/usr/bin/env python3
"""Benchmark of PLFFT's batched 1D transform path on B200.

  python bench.py --gpus N --steps K --warmup W [--impl reference] [--workload NAME]

Default workload (the configuration the headline metric is quoted on):
plain C2C FP32 forward, N=1024, batch=4096, unit stride, contiguous,
out-of-place, no scaling; re/im i.i.d. U[-1,1) from a seed.  Other workloads
(--workload) cover the remaining configurations: R2C/C2R round trip, DCT-II,
DST-II, Q0.15, the long C2C lengths in plain FP32 and split-BF16 precision,
the grouped mixed-length batch and the differentiation step.

One JSON line on rank 0.  `value` = algorithmic GB/s (one read of every input
plus one write of every output per step) summed over ranks, device-timed
with CUDA events on the launching stream, max over ranks.
Inputs rotate over buffer sets totalling more than 4x the 126 MB L2, so no
step starts L2-warm.  `e2e` is the same metric through the public entry point
with pinned host buffers (host->device and device->host copies inside the
timed region).  `--impl reference` times the CPU implementation of the path:
the FP64 port of the reference's transform definitions in oracle/ (the
reference itself is AArch64-only and does not build on an x86_64 host), on
all host cores, as K steps of a calibrated sample of the same workload.

The CPU-baseline leg runs the FP64 oracle on a sample of members taken from
the last buffer set the timed loop transformed, and compares the device's
outputs for those members with it: the line's `parity` field (worst member
rel-L2 against the FP32 gate, or bit-exactness for Q0.15).  A failed check
prints the line and exits with status 1.

Multi-GPU (torchrun, one rank per GPU): every rank runs the full workload on
its own GPU (batch replicas, weak scaling); there is no data-path collective.
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
sys.path.insert(0, os.path.join(ROOT, "tests"))

L2_BYTES = 126 << 20
QUEUE_DELAY_CYCLES = 1_000_000  # ~0.5 ms at 1.965 GHz, before the timed region


# --------------------------------------------------------------------------
# workloads
# --------------------------------------------------------------------------
class Workload:
    """One step = one pass of the hot path over one batch."""

    name = ""
    desc = ""
    dtype = "f32"
    data = "synthetic (seeded U[-1,1) re/im)"
    profile = None  # profiles/<name>.md holding traffic_bytes_per_launch

    def config(self):
        return {}

    def extra(self, stream, steps):
        """Additional keys for the JSON line (measured after the timed region)."""
        return {}


def _rand_complex(count, gen):
    import torch

    re_ = torch.rand(count, device="cuda", generator=gen) * 2 - 1
    im_ = torch.rand(count, device="cuda", generator=gen) * 2 - 1
    return torch.complex(re_, im_)


def spread_members(howmany, m, seed=0):
    """m member indices spread over the batch, always with the first and the
    last few (the final partial group of the last CTAs)."""
    import numpy as np

    m = max(1, min(m, howmany))
    tail = list(range(max(0, howmany - min(8, m // 2)), howmany))
    rng = np.random.default_rng(seed)
    rest = m - len(tail)
    body = rng.choice(max(1, howmany - len(tail)), max(0, min(rest, howmany - len(tail))), replace=False)
    return np.array(sorted(set(body.tolist()) | set(tail) | {0}))[:m] if m < howmany else np.arange(howmany)


def _rows(t, idx, width, np_dtype):
    """Members idx of a flat device buffer of contiguous rows, as a host array."""
    import numpy as np
    import torch

    v = t.view(-1)
    sel = torch.as_tensor(idx, device=v.device, dtype=torch.int64)
    if np_dtype == np.complex64:
        v = v.view(torch.complex64)
    elif np_dtype == np.int16:
        v = v.view(torch.int32)
    out = v.view(-1, width).index_select(0, sel).cpu().numpy()
    return out.view(np.int16).reshape(len(idx), width, 2) if np_dtype == np.int16 else out


def _parity(got, ref, tol, what):
    """Worst member rel-L2 of got against ref (rows), checked against tol."""
    import numpy as np

    num = np.linalg.norm(np.asarray(got, np.complex128) - ref, axis=-1)
    den = np.maximum(np.linalg.norm(ref, axis=-1), 1e-300)
    worst = float((num / den).max())
    return {"members": int(got.shape[0]), "worst_member_rel_l2": worst, "tol": tol, "ok": bool(worst <= tol),
            "against": what}


class PlanWorkload(Workload):
    """A single plfft plan executed per step."""

    def __init__(self, name, desc, kind, n, batch, r2r=None, precision=0, profile=None):
        self.name, self.desc, self.kind, self.n, self.batch = name, desc, kind, n, batch
        if kind != "c2c":
            self.data = "synthetic (seeded real U[-1,1))"
        self.r2r, self.precision, self.profile = r2r, precision, profile
        self.last_set = None

    def sizes(self):
        n, b = self.n, self.batch
        h = n // 2 + 1
        if self.kind == "c2c":
            return n * b * 8, n * b * 8
        if self.kind == "r2c":
            return n * b * 4, h * b * 8
        if self.kind == "c2r":
            return h * b * 8, n * b * 4
        return n * b * 4, n * b * 4

    def algo_bytes(self):
        i, o = self.sizes()
        return i + o

    def flops(self):
        import math

        f = 5 * self.n * math.log2(max(self.n, 2)) * self.batch
        return f if self.kind == "c2c" else f / 2

    def config(self):
        return {"workload": self.desc, "kind": self.kind, "n": self.n, "batch": self.batch,
                "layout": "unit stride, contiguous, out-of-place",
                "precision": "split_bf16" if self.precision else "fp32"}

    def setup(self, gen):
        import torch

        import plfft

        kw = {}
        if self.kind == "r2r":
            kw["r2r_kind"] = plfft.R2RKind[self.r2r]
        self.plan = plfft.make_plan(self.kind, self.n, self.batch, precision=self.precision, **kw)
        ib, ob = self.sizes()
        self.sets = max(2, -(-4 * L2_BYTES // (ib + ob)))
        self.ins = [torch.empty(ib // 4, dtype=torch.float32, device="cuda").uniform_(-1, 1, generator=gen)
                    for _ in range(self.sets)]
        self.outs = [torch.empty(ob // 4, dtype=torch.float32, device="cuda") for _ in range(self.sets)]
        self.ws = torch.empty(max(1, self.plan.workspace_size()), dtype=torch.uint8, device="cuda")
        self.launches = self.plan.launch_count()

    def step(self, i, stream):
        self.last_set = i % self.sets
        self.plan.execute_async(self.ins[i % self.sets].data_ptr(), self.outs[i % self.sets].data_ptr(),
                                self.ws.data_ptr(), stream)

    def e2e(self, steps):
        import torch

        ib, ob = self.sizes()
        hx = self.ins[0].cpu().pin_memory()
        hy = torch.empty(ob // 4, dtype=torch.float32).pin_memory()
        self.plan.execute(hx.data_ptr(), hy.data_ptr())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        for _ in range(steps):
            self.plan.execute(hx.data_ptr(), hy.data_ptr())
        e1.record(torch.cuda.default_stream())
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, ib, ob, "plfft_plan_execute(host pinned buffers)"

    def describe(self):
        return self.plan.describe()

    def sample_count(self):
        import numpy as np

        # about 2e6 n log n of oracle work, and at least 4 members
        m = max(4, min(self.batch, int(2e6 // max(1, self.n * max(1, np.log2(self.n))))))
        if self.kind == "r2r" and self.r2r not in ("DCT_2", "DST_2"):
            m = max(1, min(self.batch, int(4e7 // (self.n * self.n))))
        elif self.kind == "r2r":
            m = max(1, min(self.batch, int(2e6 // max(1, 2 * self.n * np.log2(2 * self.n)))))
        return m

    def device_rows(self, idx):
        """(inputs, outputs) of members idx of the last timed buffer set."""
        import numpy as np

        k = self.last_set
        n, h = self.n, self.n // 2 + 1
        if self.kind == "c2c":
            return _rows(self.ins[k], idx, n, np.complex64), _rows(self.outs[k], idx, n, np.complex64)
        if self.kind == "r2c":
            return _rows(self.ins[k], idx, n, np.float32), _rows(self.outs[k], idx, h, np.complex64)
        if self.kind == "c2r":
            return _rows(self.ins[k], idx, h, np.complex64), _rows(self.outs[k], idx, n, np.float32)
        return _rows(self.ins[k], idx, n, np.float32), _rows(self.outs[k], idx, n, np.float32)

    def cpu_sample(self, threads, from_device=False):
        """FP64 oracle over a bounded sample of members.  Returns (run the
        sample, sample bytes, text, check): with from_device the sample is the
        members of the last timed set and check(result) compares the device's
        outputs for them with the oracle's."""
        import numpy as np

        import oracle

        m = self.sample_count()
        idx = spread_members(self.batch, m)
        m = len(idx)
        rng = np.random.default_rng(0)
        y = None
        if from_device:
            x, y = self.device_rows(idx)
            x = x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)
        elif self.kind == "c2c":
            x = rng.uniform(-1, 1, (m, self.n)) + 1j * rng.uniform(-1, 1, (m, self.n))
        else:
            x = rng.uniform(-1, 1, (m, self.n))
        tol = 1e-6 if self.precision else oracle.fp32_tol(self.n)
        if self.kind == "c2c":
            fn = lambda: oracle.c2c(x, -1, method="fft", threads=threads)  # noqa: E731
        elif self.kind == "r2c":
            fn = lambda: oracle.r2c(x, method="fft", threads=threads)  # noqa: E731
        elif self.r2r in ("DCT_2", "DST_2"):
            # FP64 FFT of the length-2N even / odd extension, then the
            # post-rotation (the same mapping as the device path)
            k = np.arange(self.n)
            sign = 1.0 if self.r2r == "DCT_2" else -1.0
            tol = oracle.fp32_tol(2 * self.n)

            def fn():
                ext = np.concatenate([x, sign * x[:, ::-1]], axis=1).astype(np.complex128)
                F = oracle.c2c(ext, -1, method="fft", threads=threads)
                if self.r2r == "DCT_2":
                    return (np.exp(-1j * np.pi * k / (2 * self.n)) * F[:, : self.n]).real
                return -(np.exp(-1j * np.pi * (k + 1) / (2 * self.n)) * F[:, 1: self.n + 1]).imag
        else:
            tol = oracle.fp32_tol(2 * self.n)
            fn = lambda: oracle.r2r(x, self.r2r, threads=threads)  # noqa: E731
        frac = m / self.batch
        how = "direct sums" if (self.kind == "r2r" and self.r2r not in ("DCT_2", "DST_2")) else "mixed-radix FFT"
        check = None
        if y is not None:
            check = lambda ref: _parity(y, ref, tol, "FP64 oracle (oracle/)")  # noqa: E731
        return fn, self.algo_bytes() * frac, f"{m} of {self.batch} transforms, FP64 {how} (oracle/)", check


class RoundTripWorkload(PlanWorkload):
    """R2C forward then C2R with 1/N scale (one step = both)."""

    def __init__(self, name, desc, n, batch, profile=None):
        super().__init__(name, desc, "r2c", n, batch, profile=profile)

    def algo_bytes(self):
        n, b = self.n, self.batch
        return 2 * (n * b * 4 + (n // 2 + 1) * b * 8)

    def flops(self):
        import math

        return 5 * self.n * math.log2(self.n) * self.batch

    def config(self):
        c = super().config()
        c["kind"] = "r2c + c2r (1/N)"
        return c

    def setup(self, gen):
        import torch

        import plfft

        n, b = self.n, self.batch
        self.plan = plfft.make_plan("r2c", n, b)
        self.inv = plfft.make_plan("c2r", n, b, scale=1.0 / n)
        rb, cb = n * b * 4, (n // 2 + 1) * b * 8
        self.sets = max(2, -(-4 * L2_BYTES // (2 * rb + cb)))
        self.ins = [torch.empty(rb // 4, device="cuda").uniform_(-1, 1, generator=gen) for _ in range(self.sets)]
        self.mid = [torch.empty(cb // 4, device="cuda") for _ in range(self.sets)]
        self.outs = [torch.empty(rb // 4, device="cuda") for _ in range(self.sets)]
        self.ws = torch.empty(max(1, self.plan.workspace_size(), self.inv.workspace_size()), dtype=torch.uint8,
                              device="cuda")
        self.launches = self.plan.launch_count() + self.inv.launch_count()

    def step(self, i, stream):
        k = i % self.sets
        self.last_set = k
        self.plan.execute_async(self.ins[k].data_ptr(), self.mid[k].data_ptr(), self.ws.data_ptr(), stream)
        self.inv.execute_async(self.mid[k].data_ptr(), self.outs[k].data_ptr(), self.ws.data_ptr(), stream)

    def e2e(self, steps):
        import torch

        n, b = self.n, self.batch
        hx = self.ins[0].cpu().pin_memory()
        hy = torch.empty(n * b, dtype=torch.float32).pin_memory()
        dmid = self.mid[0]

        def one():
            self.plan.execute(hx.data_ptr(), dmid.data_ptr())
            self.inv.execute(dmid.data_ptr(), hy.data_ptr())

        one()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        for _ in range(steps):
            one()
        e1.record(torch.cuda.default_stream())
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, n * b * 4, n * b * 4, "plfft_plan_execute x2 (host pinned in/out)"

    def describe(self):
        return self.plan.describe() + " + " + self.inv.describe()

    def cpu_sample(self, threads, from_device=False):
        import numpy as np

        import oracle

        n, h = self.n, self.n // 2 + 1
        idx = spread_members(self.batch, self.sample_count())
        m = len(idx)
        if from_device:
            k = self.last_set
            x = _rows(self.ins[k], idx, n, np.float32).astype(np.float64)
            spec = _rows(self.mid[k], idx, h, np.complex64)
            back = _rows(self.outs[k], idx, n, np.float32)
        else:
            x = np.random.default_rng(0).uniform(-1, 1, (m, n))

        def fn():
            X = oracle.r2c(x, method="fft", threads=threads)
            return X, oracle.c2r(X, n, method="fft", threads=threads) / n

        check = None
        if from_device:
            def check(ref):
                a = _parity(spec, ref[0], oracle.fp32_tol(n), "FP64 oracle (oracle/): R2C")
                b = _parity(back, ref[1], oracle.fp32_tol(n), "FP64 oracle (oracle/): C2R(R2C)/N")
                worst = a if a["worst_member_rel_l2"] >= b["worst_member_rel_l2"] else b
                return dict(worst, ok=a["ok"] and b["ok"], against="FP64 oracle (oracle/): R2C and C2R(1/N)")
        return (fn, self.algo_bytes() * m / self.batch,
                f"{m} of {self.batch} transforms, FP64 R2C + C2R mixed-radix FFT (oracle/)", check)


class GroupedWorkload(Workload):
    """The grouped mixed-length batch in one persistent launch per phase
    (per_length=False), or the same transforms as one plain plan per
    distinct length executed back to back (per_length=True)."""

    desc = ("grouped C2C FP32: 4000 transforms, log-uniform 16..65536 (60% pow2, 20% 2^a3^b5^c7^d, "
            "10% Rader primes, 10% Bluestein)")
    profile = "grouped_4000"

    def __init__(self, count=4000, per_length=False):
        import numpy as np

        from helpers import grouped_lengths

        self.count = count
        self.per_length = per_length
        self.name = "grouped_4000_per_length" if per_length else "grouped_4000"
        if per_length:
            self.desc = self.desc.replace("in one", "") + "; one plain plan per distinct length"
        L = np.array(sorted(grouped_lengths(self.count, seed=2026)), np.int64)
        self.lengths = L
        self.offs = np.concatenate([[0], np.cumsum(L)[:-1]]).astype(np.int64)
        self.total = int(L.sum())
        self.last_set = None

    def _make_per_length(self):
        """One plan per distinct length over the contiguous members of that length."""
        import numpy as np

        import plfft

        plans = []
        uniq, first, cnt = np.unique(self.lengths, return_index=True, return_counts=True)
        for n, f, c in zip(uniq, first, cnt):
            plans.append((plfft.make_plan("c2c", int(n), int(c)), int(self.offs[f]) * 8))
        return plans

    def setup(self, gen):
        import torch

        import plfft

        L = self.lengths
        self.sets = max(2, -(-4 * L2_BYTES // (16 * self.total)))
        self.ins = [_rand_complex(self.total, gen) for _ in range(self.sets)]
        self.outs = [torch.empty(self.total, dtype=torch.complex64, device="cuda") for _ in range(self.sets)]
        if self.per_length:
            self.plans = self._make_per_length()
            self.ws = torch.empty(max(1, max(p.workspace_size() for p, _ in self.plans)), dtype=torch.uint8,
                                  device="cuda")
            self.launches = sum(p.launch_count() for p, _ in self.plans)
        else:
            self.group = plfft.Group(L, self.offs, self.offs, plfft.FORWARD)
            self.launches = self.group.launch_count()

    def algo_bytes(self):
        return 16 * self.total

    def flops(self):
        import numpy as np

        return float(np.sum(5 * self.lengths * np.log2(self.lengths)))

    def config(self):
        import numpy as np

        return {"workload": self.desc, "count": self.count, "distinct_lengths": int(len(np.unique(self.lengths))),
                "total_elements": self.total, "layout": "transforms contiguous, sorted by length"}

    def _run_per_length(self, k, stream):
        xi, yo, ws = self.ins[k].data_ptr(), self.outs[k].data_ptr(), self.ws.data_ptr()
        for p, off in self.plans:
            p.execute_async(xi + off, yo + off, ws, stream)

    def step(self, i, stream):
        k = i % self.sets
        self.last_set = k
        if self.per_length:
            self._run_per_length(k, stream)
        else:
            self.group.execute_async(self.ins[k].data_ptr(), self.outs[k].data_ptr(), stream)

    def extra(self, stream, steps):
        """Grouped line: the same transforms as per-length plain plans on the
        same buffers, timed the same way, and the grouped launch's speed-up."""
        if self.per_length:
            return {}
        import torch

        self.plans = self._make_per_length()
        self.ws = torch.empty(max(1, max(p.workspace_size() for p, _ in self.plans)), dtype=torch.uint8,
                              device="cuda")
        sh = stream.cuda_stream
        for i in range(3):
            self._run_per_length(i % self.sets, sh)
        torch.cuda.synchronize()
        reps = max(3, min(steps, 20))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(reps):
            self._run_per_length(i % self.sets, sh)
        e1.record(stream)
        torch.cuda.synchronize()
        per_ms = e0.elapsed_time(e1) / reps
        launches = sum(p.launch_count() for p, _ in self.plans)
        del self.plans
        return {"per_length": {"ms_per_step": per_ms, "value": self.algo_bytes() / (per_ms * 1e-3) / 1e9,
                               "unit": "GB/s", "plans": int(len(set(self.lengths.tolist()))),
                               "launches_per_step": launches},
                "_per_length_ms": per_ms}

    def e2e(self, steps):
        import torch

        hx = self.ins[0].cpu().pin_memory()
        hy = torch.empty(self.total, dtype=torch.complex64).pin_memory()
        s = torch.cuda.current_stream()

        def one():
            self.ins[0].copy_(hx, non_blocking=True)
            if self.per_length:
                self._run_per_length(0, s.cuda_stream)
            else:
                self.group.execute_async(self.ins[0].data_ptr(), self.outs[0].data_ptr(), s.cuda_stream)
            hy.copy_(self.outs[0], non_blocking=True)

        one()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(steps):
            one()
        e1.record(s)
        torch.cuda.synchronize()
        api = "H2D + " + ("plfft_plan_execute_async per length" if self.per_length
                          else "plfft_cuda_group_execute_async") + " + D2H (pinned)"
        return e0.elapsed_time(e1) / steps, 8 * self.total, 8 * self.total, api

    def describe(self):
        if self.per_length:
            return f"{len(self.plans)} per-length plans"
        return self.group.describe()

    def cpu_sample(self, threads, from_device=False):
        import numpy as np

        import oracle

        sel = np.arange(0, len(self.lengths), max(1, len(self.lengths) // 200))
        sel = np.union1d(sel, [len(self.lengths) - 1])
        pick = self.lengths[sel]
        if from_device:
            xin = self.ins[self.last_set]
            yout = self.outs[self.last_set]
            xs = [xin[int(o):int(o) + int(n)].cpu().numpy().astype(np.complex128)
                  for o, n in zip(self.offs[sel], pick)]
            ys = [yout[int(o):int(o) + int(n)].cpu().numpy() for o, n in zip(self.offs[sel], pick)]
        else:
            xs = [np.random.default_rng(int(n)).standard_normal(n) + 0j for n in pick]

        def fn():
            return [oracle.c2c(x[None], -1, method="fft", threads=threads)[0] for x in xs]

        check = None
        if from_device:
            def check(refs):
                ratios = []
                for y, r, n in zip(ys, refs, pick):
                    ratios.append(oracle.rel_l2(y, r) / oracle.fp32_tol(int(n)))
                worst = float(max(ratios))
                return {"members": len(ys), "worst_rel_l2_over_tol": worst, "tol": "4*log2(N)*2^-24 per length",
                        "ok": bool(worst <= 1.0), "against": "FP64 oracle (oracle/)"}
        return fn, 16 * float(np.sum(pick)), f"{len(pick)} of {self.count} transforms, FP64 FFT (oracle/)", check


class AdjointWorkload(PlanWorkload):
    """Differentiation step: R2C forward + adjoint (C2R with Hermitian-fold
    weights) of the weighted power loss, x FP32 1024 x 8192.  The adjoint
    writes a gradient buffer of its own, so the inputs stay the seeded data."""

    def __init__(self):
        super().__init__("diff_r2c_n8192_b1024", "loss = sum W |R2C(x)|^2 forward + adjoint, N=8192 batch=1024",
                         "r2c", 8192, 1024, profile="real_fused_diff_n8192_b1024")

    def algo_bytes(self):
        n, b = self.n, self.batch
        return 2 * (n * b * 4 + (n // 2 + 1) * b * 8)

    def step(self, i, stream):
        k = i % self.sets
        self.last_set = k
        self.plan.execute_async(self.ins[k].data_ptr(), self.outs[k].data_ptr(), self.ws.data_ptr(), stream)
        self.plan.execute_adjoint(self.outs[k].data_ptr(), self.grads[k].data_ptr(), 0, stream)

    def setup(self, gen):
        import torch

        super().setup(gen)
        self.grads = [torch.empty_like(x) for x in self.ins]
        self.launches *= 2

    def cpu_sample(self, threads, from_device=False):
        import numpy as np

        import oracle

        n, h = self.n, self.n // 2 + 1
        idx = spread_members(self.batch, self.sample_count())
        m = len(idx)
        if from_device:
            k = self.last_set
            x = _rows(self.ins[k], idx, n, np.float32).astype(np.float64)
            spec = _rows(self.outs[k], idx, h, np.complex64)
            grad = _rows(self.grads[k], idx, n, np.float32)
        else:
            x = np.random.default_rng(0).uniform(-1, 1, (m, n))
        # adjoint of R2C under <a, b> = Re sum conj(a) b: x_j = Re sum_k g_k e^{+2 pi i jk/n}
        # over the stored bins, i.e. C2R with the interior bins halved
        wgt = np.full(h, 0.5)
        wgt[0] = 1.0
        if n % 2 == 0:
            wgt[-1] = 1.0

        def fn():
            X = oracle.r2c(x, method="fft", threads=threads)
            return X, oracle.c2r(X * wgt, n, method="fft", threads=threads)

        check = None
        if from_device:
            def check(ref):
                a = _parity(spec, ref[0], oracle.fp32_tol(n), "R2C")
                b = _parity(grad, oracle.c2r(spec.astype(np.complex128) * wgt, n, method="fft", threads=threads),
                            oracle.fp32_tol(n), "adjoint")
                worst = a if a["worst_member_rel_l2"] >= b["worst_member_rel_l2"] else b
                return dict(worst, ok=a["ok"] and b["ok"], against="FP64 oracle (oracle/): R2C and its adjoint")
        return (fn, self.algo_bytes() * m / self.batch,
                f"{m} of {self.batch} transforms, FP64 R2C + adjoint mixed-radix FFT (oracle/)", check)


class Q15Workload(PlanWorkload):
    """Q0.15 fixed-point C2C (int16 re/im pairs, scaled by 1/N)."""

    dtype = "int16"
    data = "synthetic (seeded int16 re/im uniform in [-2^14, 2^14))"

    def __init__(self, name, desc, n, batch):
        super().__init__(name, desc, "c2c", n, batch, profile="fx_two_stage_q15_n256_b16384")

    def sizes(self):
        return self.n * self.batch * 4, self.n * self.batch * 4

    def config(self):
        c = super().config()
        c["precision"] = "q15 (bit-exact to the reference's fixed-point codelets)"
        return c

    def setup(self, gen):
        import torch

        import plfft

        self.plan = plfft.make_plan("c2c", self.n, self.batch, data_type=plfft.DataType.Q15)
        ib, ob = self.sizes()
        self.sets = max(2, -(-4 * L2_BYTES // (ib + ob)))
        # int16 re/im uniform in [-2^14, 2^14), two per 32-bit word
        self.ins = [torch.randint(-(1 << 14), 1 << 14, (ib // 2,), dtype=torch.int16, device="cuda",
                                  generator=gen).view(torch.int32) for _ in range(self.sets)]
        self.outs = [torch.empty(ob // 4, dtype=torch.int32, device="cuda") for _ in range(self.sets)]
        self.ws = torch.empty(1, dtype=torch.uint8, device="cuda")
        self.launches = self.plan.launch_count()

    def e2e(self, steps):
        import torch

        ib, ob = self.sizes()
        hx = self.ins[0].cpu().pin_memory()
        hy = torch.empty(ob // 4, dtype=torch.int32).pin_memory()
        self.plan.execute(hx.data_ptr(), hy.data_ptr())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        for _ in range(steps):
            self.plan.execute(hx.data_ptr(), hy.data_ptr())
        e1.record(torch.cuda.default_stream())
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, ib, ob, "plfft_plan_execute(host pinned buffers)"

    def cpu_sample(self, threads, from_device=False):
        import numpy as np

        import oracle

        idx = spread_members(self.batch, min(self.batch, 4096))
        m = len(idx)
        y = None
        if from_device:
            k = self.last_set
            x = _rows(self.ins[k], idx, self.n, np.int16)
            y = _rows(self.outs[k], idx, self.n, np.int16)
        else:
            rng = np.random.default_rng(0)
            x = rng.integers(-(1 << 14), 1 << 14, (m, self.n, 2)).astype(np.int16)
        check = None
        if y is not None:
            def check(ref):
                bad = int(np.count_nonzero(np.any(y != ref, axis=(1, 2))))
                return {"members": m, "mismatched_members": bad, "bit_exact": bad == 0, "ok": bad == 0,
                        "against": "bit-exact Q0.15 restatement (oracle/fixed.c)"}
        return (lambda: oracle.q15_c2c(x, -1), self.algo_bytes() * m / self.batch,
                f"{m} of {self.batch} transforms, bit-exact Q0.15 C restatement (oracle/fixed.c, {threads} threads)", check)


class Q15RealWorkload(PlanWorkload):
    """Q0.15 fixed-point R2C (int16 reals in, bins 0..N/2 as int16 re/im
    pairs out, scaled by 1/N)."""

    dtype = "int16"
    data = "synthetic (seeded int16 reals uniform in [-2^15, 2^15))"

    def __init__(self, name, desc, n, batch):
        super().__init__(name, desc, "r2c", n, batch, profile="fx_r2c_two_stage_q15_n256_b16384")
        self.data = Q15RealWorkload.data  # the real-kind default set by the base is for float data

    def sizes(self):
        return self.n * self.batch * 2, (self.n // 2 + 1) * self.batch * 4

    def config(self):
        c = super().config()
        c["precision"] = "q15 (bit-exact to the reference's fixed-point real-input plans)"
        return c

    def setup(self, gen):
        import torch

        import plfft

        self.plan = plfft.make_plan("r2c", self.n, self.batch, data_type=plfft.DataType.Q15)
        ib, ob = self.sizes()
        self.sets = max(2, -(-4 * L2_BYTES // (ib + ob)))
        self.ins = [torch.randint(-(1 << 15), 1 << 15, (ib // 2,), dtype=torch.int16, device="cuda", generator=gen)
                    for _ in range(self.sets)]
        self.outs = [torch.empty(ob // 4, dtype=torch.int32, device="cuda") for _ in range(self.sets)]
        self.ws = torch.empty(1, dtype=torch.uint8, device="cuda")
        self.launches = self.plan.launch_count()

    def e2e(self, steps):
        import torch

        ib, ob = self.sizes()
        hx = self.ins[0].cpu().pin_memory()
        hy = torch.empty(ob // 4, dtype=torch.int32).pin_memory()
        self.plan.execute(hx.data_ptr(), hy.data_ptr())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        for _ in range(steps):
            self.plan.execute(hx.data_ptr(), hy.data_ptr())
        e1.record(torch.cuda.default_stream())
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, ib, ob, "plfft_plan_execute(host pinned buffers)"

    def cpu_sample(self, threads, from_device=False):
        import numpy as np
        import torch

        import oracle

        idx = spread_members(self.batch, min(self.batch, 4096))
        m = len(idx)
        h = self.n // 2 + 1
        y = None
        if from_device:
            k = self.last_set
            sel = torch.as_tensor(idx, device="cuda", dtype=torch.int64)
            x = self.ins[k].view(-1, self.n).index_select(0, sel).cpu().numpy()
            y = _rows(self.outs[k], idx, h, np.int16)
        else:
            rng = np.random.default_rng(0)
            x = rng.integers(-(1 << 15), 1 << 15, (m, self.n)).astype(np.int16)
        check = None
        if y is not None:
            def check(ref):
                bad = int(np.count_nonzero(np.any(y != ref, axis=(1, 2))))
                return {"members": m, "mismatched_members": bad, "bit_exact": bad == 0, "ok": bad == 0,
                        "against": "bit-exact Q0.15 restatement (oracle/fixed.c)"}
        return (lambda: oracle.q15_r2c(x), self.algo_bytes() * m / self.batch,
                f"{m} of {self.batch} transforms, bit-exact Q0.15 C restatement (oracle/fixed.c, {threads} threads)", check)


def make_workload(name):
    table = {
        "c2c_n1024_b4096": lambda: PlanWorkload("c2c_n1024_b4096", "plain C2C FP32 forward N=1024 batch=4096",
                                                "c2c", 1024, 4096, profile="c2c_pow2_n1024_b4096"),
        "r2c_c2r_n4096_b8192": lambda: RoundTripWorkload("r2c_c2r_n4096_b8192",
                                                         "R2C + C2R(1/N) FP32 round trip N=4096 batch=8192",
                                                         4096, 8192, profile="real_fused_n4096_b8192"),
        "dct2_n1024_b4096": lambda: PlanWorkload("dct2_n1024_b4096", "R2R DCT-II FP32 N=1024 batch=4096", "r2r",
                                                 1024, 4096, r2r="DCT_2", profile="real_fused_dct2_n1024_b4096"),
        "dst2_n1024_b4096": lambda: PlanWorkload("dst2_n1024_b4096", "R2R DST-II FP32 N=1024 batch=4096", "r2r",
                                                 1024, 4096, r2r="DST_2", profile="real_fused_dst2_n1024_b4096"),
        "c2c_n1m_b64": lambda: PlanWorkload("c2c_n1m_b64", "C2C FP32 N=2^20 batch=64", "c2c", 1 << 20, 64,
                                            profile="fourstep_ring_n1m_b64"),
        "c2c_n64k_b1024": lambda: PlanWorkload("c2c_n64k_b1024", "C2C FP32 N=2^16 batch=1024", "c2c", 1 << 16, 1024,
                                               profile="fourstep_ring_n64k_b1024"),
        "c2c_n1m_b64_split_bf16": lambda: PlanWorkload("c2c_n1m_b64_split_bf16",
                                                       "C2C N=2^20 batch=64, split-BF16 tensor-core stages",
                                                       "c2c", 1 << 20, 64, precision=1,
                                                       profile="split_bf16_pass_n1m_b64"),
        "c2c_n64k_b1024_split_bf16": lambda: PlanWorkload("c2c_n64k_b1024_split_bf16",
                                                          "C2C N=2^16 batch=1024, split-BF16 tensor-core stages",
                                                          "c2c", 1 << 16, 1024, precision=1,
                                                          profile="split_bf16_pass_n64k_b1024"),
        "grouped_4000": lambda: GroupedWorkload(),
        "grouped_4000_per_length": lambda: GroupedWorkload(per_length=True),
        "q15_n256_b16384": lambda: Q15Workload("q15_n256_b16384", "C2C Q0.15 forward N=256 batch=16384", 256, 16384),
        "q15_r2c_n256_b16384": lambda: Q15RealWorkload("q15_r2c_n256_b16384", "R2C Q0.15 N=256 batch=16384", 256,
                                                       16384),
        "diff_r2c_n8192_b1024": lambda: AdjointWorkload(),
        # kernel-coverage workloads (not benchmark configurations): the
        # smooth non-power-of-two, Rader, Bluestein and real-wrap schedules
        "c2c_n1000_b16384": lambda: PlanWorkload("c2c_n1000_b16384", "C2C FP32 N=1000 (2^3 5^3) batch=16384",
                                                 "c2c", 1000, 16384, profile="c2c_tile_n1000_b16384"),
        "c2c_n1009_b8192": lambda: PlanWorkload("c2c_n1009_b8192", "C2C FP32 N=1009 (Rader) batch=8192",
                                                "c2c", 1009, 8192, profile="conv_rader_n1009_b8192"),
        "c2c_n1031_b8192": lambda: PlanWorkload("c2c_n1031_b8192", "C2C FP32 N=1031 (Bluestein) batch=8192",
                                                "c2c", 1031, 8192, profile="conv_bluestein_n1031_b8192"),
        "r2c_n1000_b16384": lambda: PlanWorkload("r2c_n1000_b16384", "R2C FP32 N=1000 (half length) batch=16384",
                                                 "r2c", 1000, 16384, profile="real_half_r2c_n1000_b16384"),
    }
    return table[name]()


WORKLOAD_NAMES = ["c2c_n1024_b4096", "r2c_c2r_n4096_b8192", "dct2_n1024_b4096", "dst2_n1024_b4096", "c2c_n1m_b64",
                  "c2c_n64k_b1024", "c2c_n1m_b64_split_bf16", "c2c_n64k_b1024_split_bf16", "grouped_4000",
                  "grouped_4000_per_length",
                  "diff_r2c_n8192_b1024", "q15_n256_b16384", "q15_r2c_n256_b16384",
                  "c2c_n1000_b16384", "c2c_n1009_b8192", "c2c_n1031_b8192", "r2c_n1000_b16384"]


# --------------------------------------------------------------------------
# measurement helpers
# --------------------------------------------------------------------------
def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """Steady-state DRAM bytes (read + write) of one step from the committed
    ncu summary: all of the step's kernels, three consecutive steps captured
    without cache flushing, averaged."""
    if not name:
        return None
    path = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_step:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the workload runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []  # (host time, csv line)
        self.t_mark = self.t_end = None

    def mark(self):
        """The timed region starts."""
        self.t_mark = time.perf_counter()

    def mark_end(self):
        self.t_end = time.perf_counter()

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
            self.lines.append((time.perf_counter(), line.strip()))

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
        # samples inside the timed region (with one sampling period of slack);
        # a region shorter than the period falls back to every sample taken
        # while the workload ran (warm-up, timed loop, per-step timing)
        lines = [ln for t, ln in self.lines
                 if self.t_mark is not None and self.t_mark - 0.1 <= t <= (self.t_end or t) + 0.1]
        window = "timed region"
        if len(lines) < 2:
            lines, window = [ln for _, ln in self.lines], "warm-up through per-step timing"
        for ln in lines:
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
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm),
                "window": window}


def _calibrate(fn):
    """Seconds of one sample after a warm-up call."""
    fn()
    t0 = time.perf_counter()
    fn()
    return max(time.perf_counter() - t0, 1e-6)


def cpu_baseline(w, target_s=10.0, from_device=True):
    """The CPU oracle on repetitions of a bounded sample, about target_s
    seconds.  The sample is members of the last timed buffer set; the
    oracle's result for it is also the parity check of the device outputs."""
    import platform

    import oracle

    threads = oracle.max_threads()
    fn, sbytes, text, check = w.cpu_sample(threads, from_device=from_device)
    ref = fn()
    parity = check(ref) if check is not None else None
    t0 = time.perf_counter()
    fn()
    one = max(time.perf_counter() - t0, 1e-6)
    reps = max(1, min(100000, int(target_s / one)))
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    dt = (time.perf_counter() - t0) / reps
    return {"value": sbytes / dt / 1e9, "unit": "GB/s", "cores": threads, "kind": "port",
            "host_arch": platform.machine(),
            "sample": f"{text}, {reps} repetitions ({reps * dt:.1f} s)"}, parity


def reference_arm(w, steps, warmup, budget_s=120.0):
    """The reference's CPU path (the oracle port: the reference cannot be
    built on this host) timed as `steps` steps of a bounded sample after
    `warmup` untimed ones; the whole run stays within about budget_s seconds."""
    import platform

    import oracle

    threads = oracle.max_threads()
    fn, sbytes, text, _ = w.cpu_sample(threads)
    one = _calibrate(fn)
    per_step = min(10.0, max(0.05, budget_s / max(1, steps + warmup)))
    reps = max(1, int(per_step / one))
    for _ in range(warmup * reps):
        fn()
    t0 = time.perf_counter()
    for _ in range(steps * reps):
        fn()
    dt = time.perf_counter() - t0
    value = steps * reps * sbytes / dt / 1e9
    return value, {"value": value, "unit": "GB/s", "cores": threads, "kind": "port",
                   "host_arch": platform.machine(),
                   "sample": f"{text}, {reps} repetitions per step"}, dt * 1e3 / steps


def max_over_ranks(dist, values, device):
    """Element-wise maximum over ranks of per-rank figures (step counts,
    device-timed milliseconds).  Every rank makes the same collective call
    in the same order; without a process group the values pass through."""
    import torch

    if dist is None:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


# --------------------------------------------------------------------------
def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: enough for about 1 s of timed work, at least 200)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2c_n1024_b4096", choices=WORKLOAD_NAMES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    w = make_workload(args.workload)

    if args.impl == "reference":
        if rank != 0:
            return
        steps = args.steps if args.steps is not None else 10
        value, cpu, ms = reference_arm(w, steps, args.warmup)
        line = {"metric": f"{w.name} GB/s (algorithmic bytes)", "value": value, "unit": "GB/s",
                "impl": "reference", "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
                "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64" if w.dtype == "f32" else w.dtype,
                "data": w.data, "config": w.config(), "cpu_baseline": cpu,
                "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import numpy as np
    import torch

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

    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234 + rank)
    w.setup(gen)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream

    # the clock sampler runs from before the warm-up, so starting it costs
    # the timed region nothing
    sampler = ClockSampler(local)
    sampler.start()
    # the step index picks the buffer set; it runs on through every phase so
    # that no timed step finds its set still in L2 from an earlier one
    nxt = 0
    for i in range(args.warmup):
        w.step(nxt, sh)
        nxt += 1
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.steps is None:
        # size the timed region to about one second (clock samples need it)
        ev0.record(stream)
        for i in range(20):
            w.step(nxt, sh)
            nxt += 1
        ev1.record(stream)
        torch.cuda.synchronize()
        est = ev0.elapsed_time(ev1) / 20
        steps = max(200, min(200000, int(1000.0 / max(est, 1e-4))))
        # every rank times the same number of steps
        args.steps = int(max_over_ranks(dist, [steps], "cuda")[0])
    barrier()
    torch.cuda.synchronize()
    sampler.mark()
    # the device idles ~0.5 ms before the start event while the host queues
    # the first steps, so the timed region holds the K steps back to back and
    # not the host's latency of the first launch (the host keeps ahead after
    # that: it submits a step faster than the device runs one)
    torch.cuda._sleep(QUEUE_DELAY_CYCLES)
    first_timed = nxt
    ev0.record(stream)
    for i in range(args.steps):
        w.step(first_timed + i, sh)
    ev1.record(stream)
    nxt = first_timed + args.steps
    torch.cuda.synchronize()
    sampler.mark_end()
    barrier()
    ms = ev0.elapsed_time(ev1)
    last_timed_set = getattr(w, "last_set", None)
    # per-step device time (each step bracketed by events)
    nk = min(args.steps, 50)
    kev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * nk)]
    for i in range(nk):
        kev[2 * i].record(stream)
        w.step(nxt + i, sh)
        kev[2 * i + 1].record(stream)
    torch.cuda.synchronize()
    step_ms = statistics.median(kev[2 * i].elapsed_time(kev[2 * i + 1]) for i in range(nk))
    clocks = sampler.stop()
    extra = w.extra(stream, args.steps)
    per_length_ms = extra.pop("_per_length_ms", None)
    e2e = None
    if not args.no_e2e:
        e2e_ms, hb, db, api = w.e2e(max(3, min(args.steps, 20)))
        e2e = {"value": w.algo_bytes() * world / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s",
               "h2d_bytes_per_step": hb, "d2h_bytes_per_step": db, "ms_per_step": e2e_ms, "api": api}

    if dist is not None:
        ms, step_ms, e2e_max = max_over_ranks(dist, [ms, step_ms, e2e["ms_per_step"] if e2e else 0.0], "cuda")
        if e2e:
            e2e["ms_per_step"] = e2e_max
            e2e["value"] = w.algo_bytes() * world / (e2e_max * 1e-3) / 1e9

    ms_per_step = ms / args.steps
    abytes = w.algo_bytes()
    value = abytes * world / (ms_per_step * 1e-3) / 1e9
    peak, peak_kind = peaks()
    # one launch per step: its average duration over the timed region;
    # several: the median event-bracketed step (all of the step's kernels)
    kernel_ms = ms_per_step if w.launches == 1 else step_ms
    achieved = abytes / (kernel_ms * 1e-3) / 1e9
    cpu, parity = None, None
    if rank == 0 and not args.no_cpu_baseline:
        # the per-step timing loop above ran other buffer sets last (and may
        # have wrapped onto the timed one): redo the final timed step so the
        # checked buffer set holds the timed step's outputs
        if last_timed_set is not None:
            w.step(first_timed + args.steps - 1, sh)
            torch.cuda.synchronize()
        cpu, parity = cpu_baseline(w)
    if rank == 0:
        line = {
            "metric": f"{w.name} GB/s (algorithmic bytes)", "value": value, "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": w.dtype,
            "data": w.data,
            "config": dict(w.config(), l2="inputs rotate over buffer sets totalling > 4x L2",
                           parallelism=f"batch replicas x{world}, no collective",
                           queue="steps queued behind a ~0.5 ms device delay before the start event"),
            "gflops": w.flops() * world / (ms_per_step * 1e-3) / 1e9,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": profile_traffic(w.profile), "kernel_ms": kernel_ms,
                         "algorithmic_bytes_per_step": abytes, "launches_per_step": w.launches},
            "e2e": e2e,
            "gpu_launches": w.launches * args.steps,
            "plan": w.describe(),
            "clocks": clocks,
            "cpu_baseline": cpu,
            "parity": parity,
        }
        line.update(extra)
        if per_length_ms is not None:
            line["speedup_vs_per_length"] = per_length_ms / ms_per_step
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    if parity is not None and not parity["ok"]:
        print(f"bench: parity check failed: {parity}", file=sys.stderr)
        sys.exit(1)


if __name__ == "__main__":
    main()
