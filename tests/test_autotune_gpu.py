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
