"""C2C FP32 parity: CUDA path (through the C-ABI) vs the FP64 oracle.

Gate: rel-L2 <= 4*log2(N)*2^-24 per case (FP32 tolerance of the spec).
Cases include the reference's own C2C list (test/c2c_f32.cpp:10-27).
"""
import numpy as np
import pytest

import oracle
from helpers import c2c_case

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 4, 5, 7, 8, 9, 11, 12, 13, 15, 16, 25, 32, 49, 64, 100, 128, 143, 256, 360, 512,
         1000, 1024, 2048, 2187, 4096, 8192, 16384]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("direction", [-1, 1])
def test_c2c_sizes(n, direction):
    howmany = max(1, min(64, 65536 // n))
    got, ref, plan = c2c_case(n, howmany, direction=direction, seed=n)
    err = oracle.rel_l2(got, ref)
    assert err <= oracle.fp32_tol(n), (n, err, plan.describe())


# reference test/c2c_f32.cpp:10-27 (those with on-chip smooth lengths)
REF_CASES = [
    (2, 1, 1, 2, 1, 2), (8, 1, 1, 8, 1, 8), (16, 4, 1, 16, 1, 16), (8, 3, 2, 20, 2, 20),
    (64, 2, 8, 600, 8, 600), (24, 4, 1, 32, 1, 32), (512, 1, 1, 512, 1, 512), (512, 3, 1, 512, 1, 512),
    (512, 3, 3, 1, 3, 1), (1024, 4, 1, 1024, 1, 1024), (1024, 4, 1, 1024, 1024, 1),
]


@pytest.mark.parametrize("case", REF_CASES)
@pytest.mark.parametrize("direction", [-1, 1])
def test_c2c_reference_layouts(case, direction):
    n, hm, is_, id_, os_, od = case
    got, ref, plan = c2c_case(n, hm, is_, id_, os_, od, direction=direction, seed=7)
    assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(n), plan.describe()


# reference test/c2c_f32.cpp:17,24 -- prime and large-prime-factor layouts
REF_CONV_CASES = [(23, 49, 441, 9, 441, 9), (1058, 4, 1058, 1, 1058, 1), (23, 3, 1, 23, 1, 23)]


@pytest.mark.parametrize("case", REF_CONV_CASES)
@pytest.mark.parametrize("direction", [-1, 1])
def test_c2c_reference_conv_layouts(case, direction):
    n, hm, is_, id_, os_, od = case
    got, ref, plan = c2c_case(n, hm, is_, id_, os_, od, direction=direction, seed=17)
    assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(n), plan.describe()


# (n, schedule): Rader for primes p with smooth p - 1, Bluestein otherwise
# (the reference planner's rule); one fused launch while the convolution fits
# a power-of-two m <= 8192 (Rader: m >= 2p - 3, Bluestein: m >= 2n - 1),
# multi-launch convolutions beyond
CONV_CASES = [(17, "rader-fused"), (23, "rader-fused"), (97, "rader-fused"), (1009, "rader-fused"),
              (4001, "rader-fused"), (47, "bluestein-fused"), (94, "bluestein-fused"), (1031, "bluestein-fused"),
              (1058, "bluestein-fused"), (2870, "bluestein-fused"), (4093, "bluestein-fused"),
              (4094, "bluestein-fused"), (4099, "(bluestein n="), (2 * 8191, "(bluestein n="), (65537, "(rader n="),
              (8191 * 3, "(bluestein n=")]


@pytest.mark.parametrize("n,expect", CONV_CASES)
@pytest.mark.parametrize("direction", [-1, 1])
def test_c2c_rader_bluestein(n, expect, direction):
    howmany = 3
    got, ref, plan = c2c_case(n, howmany, direction=direction, seed=n, method="fft")
    assert expect in plan.describe(), plan.describe()
    assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(n), plan.describe()


# the fused convolution kernel's launch shapes: 16 or 32 elements per thread,
# each register budget, several members per CTA (the last CTA partly
# filled), strided members
@pytest.mark.parametrize("e,minb", [(16, 2), (16, 3), (16, 4), (32, 2)])
@pytest.mark.parametrize("n,hm,layout", [(17, 37, (1, 17, 1, 17)), (1009, 11, (1, 1009, 1, 1009)),
                                         (1031, 9, (9, 1, 9, 1)), (4093, 5, (1, 4093, 1, 4093)),
                                         (4001, 3, (1, 4003, 1, 4001)), (3001, 4, (3, 9003, 1, 3001)),
                                         (300 * 7 - 1, 4, (1, 2099, 1, 2100)), (263, 33, (2, 600, 1, 263))])
def test_c2c_conv_fused_shapes(monkeypatch, e, minb, n, hm, layout):
    monkeypatch.setenv("PLFFT_B200_CONV_E", str(e))
    monkeypatch.setenv("PLFFT_B200_CONV_MINB", str(minb))
    monkeypatch.setenv("PLFFT_B200_CONV_G", "4")
    is_, id_, os_, od = layout
    for direction in (-1, 1):
        got, ref, plan = c2c_case(n, hm, is_, id_, os_, od, direction=direction, seed=n + e, method="fft")
        assert "fused" in plan.describe(), plan.describe()
        assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(n), plan.describe()


@pytest.mark.parametrize("n", [32768, 65536, 1 << 18, 1 << 20])
def test_c2c_four_step(n):
    howmany = 2
    got, ref, plan = c2c_case(n, howmany, seed=3, method="fft")
    assert "four-step" in plan.describe()
    assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(n), plan.describe()


# the bulk-copy ring passes (dense batches): every supported tile width and
# slot count, both directions, more tiles than CTAs so each CTA's ring wraps
@pytest.mark.parametrize("n,c,slots", [(1 << 14, 16, 3), (1 << 15, 8, 2), (1 << 16, 16, 3), (1 << 16, 16, 2),
                                       (1 << 16, 8, 3), (1 << 17, 16, 3), (1 << 18, 8, 3), (1 << 19, 8, 3),
                                       (1 << 20, 8, 2), (1 << 20, 4, 3)])
def test_c2c_four_step_ring(monkeypatch, n, c, slots):
    import plfft

    monkeypatch.setenv("PLFFT_B200_FSR_C", str(c))
    monkeypatch.setenv("PLFFT_B200_FSR_SLOTS", str(slots))
    howmany = max(2, (1 << 22) // n)
    for direction in (-1, 1):
        got, ref, plan = c2c_case(n, howmany, direction=direction, seed=n + c, method="fft")
        assert "bulk-ring" in plan.describe(), plan.describe()
        assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(n), plan.describe()


# strided or unaligned members keep the per-element four-step passes
@pytest.mark.parametrize("case", [(1 << 16, 3, 1, 65537, 1, 65536), (1 << 16, 2, 2, 2 * 65536, 1, 65536)])
def test_c2c_four_step_strided(case):
    n, hm, is_, id_, os_, od = case
    got, ref, plan = c2c_case(n, hm, is_, id_, os_, od, seed=5, method="fft")
    assert "four-step" in plan.describe(), plan.describe()
    assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(n), plan.describe()


@pytest.mark.parametrize("n", [16, 1024, 1000, 4096])
def test_c2c_in_place(n):
    got, ref, _ = c2c_case(n, 8, alias=True, seed=11)
    assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(n)


@pytest.mark.parametrize("n", [1024, 77 * 13])
def test_c2c_host_pointers(n):
    got, ref, _ = c2c_case(n, 5, host=True, seed=5)
    assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(n)


def test_c2c_scale_round_trip():
    import plfft
    import torch

    n, hm = 4096, 16
    rng = np.random.default_rng(1)
    x = (rng.uniform(-1, 1, n * hm) + 1j * rng.uniform(-1, 1, n * hm)).astype(np.complex64)
    fwd = plfft.make_plan("c2c", n, hm, direction=-1)
    bwd = plfft.make_plan("c2c", n, hm, direction=1, scale=1.0 / n)
    d = torch.from_numpy(x).cuda()
    y = torch.empty_like(d)
    z = torch.empty_like(d)
    fwd.execute(d.data_ptr(), y.data_ptr())
    bwd.execute(y.data_ptr(), z.data_ptr())
    assert oracle.rel_l2(z.cpu().numpy(), x) <= oracle.fp32_tol(n)


def test_c2c_known_pairs():
    """delta -> constant and pure tone (reference test/delta_constant_test.hpp:38-63,
    test/pure_tone_test.hpp:36-62)."""
    import plfft
    import torch

    n = 1024
    plan = plfft.make_plan("c2c", n, 2, direction=-1)
    x = np.zeros(2 * n, np.complex64)
    x[0] = 1.0
    k0 = 37
    x[n + k0] = 1.0
    d = torch.from_numpy(x).cuda()
    y = torch.empty_like(d)
    plan.execute(d.data_ptr(), y.data_ptr())
    y = y.cpu().numpy()
    assert np.allclose(y[:n], 1.0, atol=1e-6)
    k = np.arange(n)
    tone = np.exp(-2j * np.pi * k * k0 / n)
    assert np.abs(y[n:] - tone).max() < 1e-5


def test_c2c_output_guard_band():
    """Strided output: bytes between outputs and past the span stay untouched."""
    import plfft
    import torch

    n, hm, os_, od = 256, 3, 2, 600
    plan = plfft.make_plan("c2c", n, hm, 1, n, os_, od)
    x = torch.randn(hm * n, dtype=torch.complex64, device="cuda")
    sentinel = complex(1234.5, -987.25)
    total = (hm - 1) * od + (n - 1) * os_ + 1 + 64
    y = torch.full((total,), sentinel, dtype=torch.complex64, device="cuda")
    plan.execute(x.data_ptr(), y.data_ptr())
    yc = y.cpu().numpy()
    mask = np.ones(total, bool)
    idx = (np.arange(hm)[:, None] * od + np.arange(n)[None, :] * os_).ravel()
    mask[idx] = False
    assert np.all(yc[mask] == np.complex64(sentinel))


@pytest.mark.parametrize("kind,n,howmany", [("c2c", 1024, 2501), ("r2c", 4096, 1500), ("c2r", 4096, 1500)])
def test_host_buffers_pipelined_chunks(kind, n, howmany):
    """plfft_plan_execute on large host batches runs as overlapped chunks
    (copies and kernels on several streams), with a shorter last chunk."""
    import plfft

    rng = np.random.default_rng(21)
    h = n // 2 + 1
    plan = plfft.make_plan(kind, n, howmany)
    if kind == "c2c":
        x = (rng.uniform(-1, 1, (howmany, n)) + 1j * rng.uniform(-1, 1, (howmany, n))).astype(np.complex64)
        y = np.zeros_like(x)
        plan.execute(x.ctypes.data, y.ctypes.data)
        ref = oracle.c2c(x.astype(np.complex128), -1, method="fft")
    elif kind == "r2c":
        x = rng.uniform(-1, 1, (howmany, n)).astype(np.float32)
        y = np.zeros((howmany, h), np.complex64)
        plan.execute(x.ctypes.data, y.ctypes.data)
        ref = oracle.r2c(x.astype(np.float64), method="fft")
    else:
        spec = oracle.r2c(rng.uniform(-1, 1, (howmany, n)), method="fft")
        x = spec.astype(np.complex64)
        y = np.zeros((howmany, n), np.float32)
        plan.execute(x.ctypes.data, y.ctypes.data)
        ref = oracle.c2r(x.astype(np.complex128), n, method="fft")
    assert oracle.rel_l2(y, ref) <= oracle.fp32_tol(n), plan.describe()


@pytest.fixture
def cluster_form(monkeypatch):
    """Select the one-pass cluster form of n = 65536 (an autotuner candidate)."""
    monkeypatch.setenv("PLFFT_B200_CLUSTER", "1")


@pytest.mark.parametrize("direction", [-1, 1])
@pytest.mark.parametrize("layout", [(41, 1, None, 1, None), (3, 2, 1, 3, 1)])
def test_c2c_cluster_four_step(cluster_form, direction, layout):
    """n = 65536 in one pass on 8-CTA clusters: more members than resident
    clusters (the clusters loop), and interleaved strided members."""
    hm, is_, id_, os_, od = layout
    got, ref, plan = c2c_case(65536, hm, is_, id_, os_, od, direction=direction, seed=4, method="fft")
    assert "cluster" in plan.describe(), plan.describe()
    assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(65536), plan.describe()


def test_c2c_cluster_four_step_in_place(cluster_form):
    got, ref, plan = c2c_case(65536, 5, alias=True, seed=8, method="fft")
    assert "cluster" in plan.describe(), plan.describe()
    assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(65536), plan.describe()
