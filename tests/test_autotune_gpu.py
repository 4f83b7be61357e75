"""Planner rigor levels: MEASURE / PATIENT / EXHAUSTIVE time candidate
schedules and keep the fastest (reference src/plfft.cpp:149-184,
src/planner/benchmarker.hpp:33-93), remembered as wisdom
(src/planner/wisdom.hpp:23-37).  Whatever schedule wins, results must meet
the FP32 parity gate.
"""
import os

import numpy as np
import pytest

import oracle
from helpers import c2c_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,howmany,rigor", [(1024, 512, "MEASURE"), (256, 300, "PATIENT"),
                                             (4096, 64, "MEASURE"), (65536, 4, "EXHAUSTIVE"),
                                             (1000, 40, "PATIENT")])
def test_autotuned_plans_are_correct(n, howmany, rigor):
    import plfft

    plfft.wisdom_forget()
    got, ref, plan = c2c_case(n, howmany, seed=n, rigor=plfft.Rigor[rigor], method="fft")
    assert "autotuned" in plan.describe() or "c2c" in plan.describe()
    assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(n), plan.describe()


def test_wisdom_reuse_export_import(tmp_path):
    import plfft

    plfft.wisdom_forget()
    a = plfft.make_plan("c2c", 1024, 256, rigor=plfft.Rigor.MEASURE)
    assert "autotuned" in a.describe(), a.describe()
    b = plfft.make_plan("c2c", 1024, 256, rigor=plfft.Rigor.MEASURE)
    assert "[wisdom]" in b.describe()
    assert b.describe().split(" [")[0] == a.describe().split(" [")[0]
    path = os.path.join(tmp_path, "wisdom.txt")
    plfft.wisdom_export(path)
    lines = open(path).read().splitlines()
    assert any(line.startswith("c2c n=1024 hm=256") for line in lines)
    plfft.wisdom_forget()
    c = plfft.make_plan("c2c", 1024, 256, rigor=plfft.Rigor.MEASURE)
    assert "autotuned" in c.describe()
    plfft.wisdom_forget()
    plfft.wisdom_import(path)
    d = plfft.make_plan("c2c", 1024, 256, rigor=plfft.Rigor.MEASURE)
    assert "[wisdom]" in d.describe()


def test_estimate_is_not_tuned():
    import plfft

    p = plfft.make_plan("c2c", 1024, 64, rigor=plfft.Rigor.ESTIMATE)
    assert "autotuned" not in p.describe() and "wisdom" not in p.describe()


@pytest.mark.parametrize("kind,n,howmany,r2r,rigor", [
    ("r2c", 4096, 256, None, "MEASURE"), ("c2r", 1024, 300, None, "PATIENT"), ("r2c", 1000, 64, None, "MEASURE"),
    ("r2r", 1024, 200, "DCT_2", "MEASURE"), ("r2r", 256, 100, "DST_3", "EXHAUSTIVE"), ("r2r", 33, 50, "DCT_1", "MEASURE"),
])
def test_autotuned_real_plans_are_correct(kind, n, howmany, r2r, rigor):
    """Real-data kinds are tuned too (fused-kernel launch shapes and the
    real-wrap schedule); the winner must meet the parity gate."""
    import plfft
    import torch

    plfft.wisdom_forget()
    rng = np.random.default_rng(n)
    h = n // 2 + 1
    kw = {"r2r_kind": plfft.R2RKind[r2r]} if r2r else {}
    plan = plfft.make_plan(kind, n, howmany, rigor=plfft.Rigor[rigor], **kw)
    assert "autotuned" in plan.describe() or "[" not in plan.describe(), plan.describe()
    if kind == "c2r":
        x = (rng.uniform(-1, 1, (howmany, h)) + 1j * rng.uniform(-1, 1, (howmany, h))).astype(np.complex64)
        y = torch.empty(howmany * n, dtype=torch.float32, device="cuda")
        ref = oracle.c2r(x.astype(np.complex128), n)
    else:
        x = rng.uniform(-1, 1, (howmany, n)).astype(np.float32)
        y = torch.empty(howmany * (h if kind == "r2c" else n), dtype=torch.complex64 if kind == "r2c" else torch.float32,
                        device="cuda")
        ref = oracle.r2c(x.astype(np.float64)) if kind == "r2c" else oracle.r2r(x.astype(np.float64), r2r)
    d = torch.from_numpy(np.ascontiguousarray(x).ravel()).cuda()
    plan.execute(d.data_ptr(), y.data_ptr())
    got = y.cpu().numpy().reshape(ref.shape)
    tol = oracle.fp32_tol(2 * n if kind == "r2r" else n)
    assert oracle.rel_l2(got, ref) <= tol, plan.describe()
    again = plfft.make_plan(kind, n, howmany, rigor=plfft.Rigor[rigor], **kw)
    if "autotuned" in plan.describe():
        assert "[wisdom]" in again.describe(), again.describe()
