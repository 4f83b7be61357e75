"""R2C / C2R / R2R FP32 parity: CUDA path (C-ABI) vs the FP64 oracle.

Gate: rel-L2 <= 4*log2(N)*2^-24.  Cases follow the reference's real-data
tests (test/simple_test.hpp:16-95 round trips and sums, test/r2r_test.hpp:
82-178 all 11 kinds, test/plfft_interface_test.cpp:360-413 in-place R2C/C2R).
"""
import numpy as np
import pytest

import oracle
import plfft
from helpers import gather, span

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_plan(plan, x, nout_elems, out_dtype):
    import torch

    d = _dev(x)
    y = torch.zeros(nout_elems, dtype=out_dtype, device="cuda")
    plan.execute(d.data_ptr(), y.data_ptr())
    return y.cpu().numpy()


R2C_SIZES = [1, 2, 3, 4, 5, 8, 16, 17, 64, 100, 128, 1000, 1024, 4096, 8192, 32768]


@pytest.mark.parametrize("n", R2C_SIZES)
def test_r2c(n):
    import torch

    hm = max(1, min(32, 65536 // n))
    h = n // 2 + 1
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, hm * n).astype(np.float32)
    plan = plfft.make_plan("r2c", n, hm)
    y = run_plan(plan, x, hm * h, torch.complex64).reshape(hm, h)
    ref = oracle.r2c(x.reshape(hm, n).astype(np.float64))
    assert oracle.rel_l2(y, ref) <= oracle.fp32_tol(n), plan.describe()


@pytest.mark.parametrize("n", R2C_SIZES)
def test_c2r(n):
    import torch

    hm = max(1, min(32, 65536 // n))
    h = n // 2 + 1
    rng = np.random.default_rng(n + 1)
    X = (rng.uniform(-1, 1, (hm, h)) + 1j * rng.uniform(-1, 1, (hm, h))).astype(np.complex64)
    plan = plfft.make_plan("c2r", n, hm)
    y = run_plan(plan, X.ravel(), hm * n, torch.float32).reshape(hm, n)
    ref = oracle.c2r(X.astype(np.complex128), n)
    assert oracle.rel_l2(y, ref) <= oracle.fp32_tol(n), plan.describe()


@pytest.mark.parametrize("n", [4096, 1000, 17])
def test_r2c_c2r_round_trip_scaled(n):
    import torch

    hm = 8
    h = n // 2 + 1
    rng = np.random.default_rng(9)
    x = rng.uniform(-1, 1, hm * n).astype(np.float32)
    f = plfft.make_plan("r2c", n, hm)
    b = plfft.make_plan("c2r", n, hm, scale=1.0 / n)
    d = _dev(x)
    y = torch.empty(hm * h, dtype=torch.complex64, device="cuda")
    z = torch.empty(hm * n, dtype=torch.float32, device="cuda")
    f.execute(d.data_ptr(), y.data_ptr())
    b.execute(y.data_ptr(), z.data_ptr())
    assert oracle.rel_l2(z.cpu().numpy(), x) <= oracle.fp32_tol(n)


@pytest.mark.parametrize("n", [4, 5])
def test_in_place_real_complex_round_trip(n):
    """reference test/plfft_interface_test.cpp:360-413 (spans 6 real / 3 complex)."""
    hm, rspan, cspan = 2, 6, 3
    data = np.zeros(hm * rspan, np.float32)
    for b in range(hm):
        for e in range(n):
            data[b * rspan + e] = b * 10 + e + 1
    expected = data.copy() * n
    f = plfft.make_plan("r2c", n, hm, 1, rspan, 1, cspan, alias=plfft.IoAlias.MAY_ALIAS)
    c = plfft.make_plan("c2r", n, hm, 1, cspan, 1, rspan, alias=plfft.IoAlias.MAY_ALIAS)
    f.execute(data.ctypes.data, data.ctypes.data)
    c.execute(data.ctypes.data, data.ctypes.data)
    for b in range(hm):
        for e in range(n):
            i = b * rspan + e
            assert abs(data[i] - expected[i]) < 1e-4


KINDS = ["DCT_1", "DCT_2", "DCT_3", "DCT_4", "DST_1", "DST_2", "DST_3", "DST_4", "DHT", "R2HC", "HC2R"]


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n", [2, 3, 8, 17, 64, 128, 1024])
def test_r2r(kind, n):
    import torch

    hm = 4
    rng = np.random.default_rng(hash((kind, n)) % 2**32)
    x = rng.uniform(-1, 1, hm * n).astype(np.float32)
    plan = plfft.make_plan("r2r", n, hm, r2r_kind=plfft.R2RKind[kind])
    y = run_plan(plan, x, hm * n, torch.float32).reshape(hm, n)
    ref = oracle.r2r(x.reshape(hm, n).astype(np.float64), kind)
    assert oracle.rel_l2(y, ref) <= oracle.fp32_tol(2 * n), (kind, n, plan.describe())


def test_dct1_n1_rejected():
    with pytest.raises(plfft.PlfftError) as e:
        plfft.make_plan("r2r", 1, 1, r2r_kind=plfft.R2RKind.DCT_1)
    assert e.value.status == plfft.Status.PLAN_CREATION_FAILED


def test_r2r_in_place_r2hc():
    """reference test/plfft_interface_test.cpp:415-433."""
    data = np.array([1, 2, 3, 4], np.float32)
    p = plfft.make_plan("r2r", 4, 1, r2r_kind=plfft.R2RKind.R2HC, alias=plfft.IoAlias.MAY_ALIAS)
    p.execute(data.ctypes.data, data.ctypes.data)
    assert data[0] == 10.0


@pytest.mark.parametrize("kind", ["DCT_2", "DST_2"])
def test_r2r_strided(kind):
    import torch

    n, hm, is_, id_, os_, od = 64, 3, 2, 200, 3, 300
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, span(hm, id_, n, is_)).astype(np.float32)
    plan = plfft.make_plan("r2r", n, hm, is_, id_, os_, od, r2r_kind=plfft.R2RKind[kind])
    y = run_plan(plan, x, span(hm, od, n, os_), torch.float32)
    ref = oracle.r2r(gather(x, hm, id_, n, is_).astype(np.float64), kind)
    assert oracle.rel_l2(gather(y, hm, od, n, os_), ref) <= oracle.fp32_tol(2 * n)


FUSED_N = [128, 256, 512, 1024, 2048, 4096, 8192, 16384]


@pytest.mark.parametrize("n", FUSED_N)
@pytest.mark.parametrize("pad", [0, 1])
def test_fused_r2c_c2r(n, pad):
    """One-kernel R2C/C2R (N = 2M, M a power of two); pad=1 makes the real
    distance odd so real pairs are not 8-byte aligned (scalar path)."""
    import torch

    hm = 5
    h = n // 2 + 1
    rid, cid = n + pad, h + pad
    rng = np.random.default_rng(n + pad)
    x = rng.uniform(-1, 1, span(hm, rid, n, 1)).astype(np.float32)
    f = plfft.make_plan("r2c", n, hm, 1, rid, 1, cid)
    assert "fused" in f.describe(), f.describe()
    y = run_plan(f, x, span(hm, cid, h, 1), torch.complex64)
    ref = oracle.r2c(gather(x, hm, rid, n, 1).astype(np.float64))
    assert oracle.rel_l2(gather(y, hm, cid, h, 1), ref) <= oracle.fp32_tol(n)
    X = (rng.uniform(-1, 1, (hm, h)) + 1j * rng.uniform(-1, 1, (hm, h))).astype(np.complex64)
    b = plfft.make_plan("c2r", n, hm, 1, h, 1, rid)
    assert "fused" in b.describe(), b.describe()
    z = run_plan(b, X.ravel(), span(hm, rid, n, 1), torch.float32)
    refz = oracle.c2r(X.astype(np.complex128), n)
    assert oracle.rel_l2(gather(z, hm, rid, n, 1), refz) <= oracle.fp32_tol(n)


FUSED_R2R = ["DCT_2", "DST_2", "DCT_3", "DST_3", "DCT_4", "DST_4", "DHT", "R2HC", "HC2R"]


@pytest.mark.parametrize("kind", FUSED_R2R)
@pytest.mark.parametrize("n", [128, 1024, 2048, 4096, 16384])
def test_fused_r2r(kind, n):
    """One-kernel R2R kinds for N = 2M, M a power of two (real_fused.cu)."""
    import torch

    hm = 3
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, hm * n).astype(np.float32)
    plan = plfft.make_plan("r2r", n, hm, r2r_kind=plfft.R2RKind[kind])
    assert "fused" in plan.describe(), plan.describe()
    y = run_plan(plan, x, hm * n, torch.float32).reshape(hm, n)
    ref = oracle.r2r(x.reshape(hm, n).astype(np.float64), kind)
    assert oracle.rel_l2(y, ref) <= oracle.fp32_tol(2 * n)


@pytest.mark.parametrize("kind", ["DCT_2", "DST_2", "DCT_3", "DST_3"])
@pytest.mark.parametrize("n", [128, 1024, 2048])
@pytest.mark.parametrize("pad", [0, 1, 2, 4])
def test_fused_member_alignment(kind, n, pad):
    """Member distances n + pad on both sides: 16-byte aligned members take
    the float4 paths (DCT-II / DST-II input, DCT-III / DST-III output), the
    others the staged ones; both must agree with the oracle."""
    import torch

    hm = 5
    d = n + pad
    rng = np.random.default_rng(n + pad)
    x = rng.uniform(-1, 1, span(hm, d, n, 1)).astype(np.float32)
    plan = plfft.make_plan("r2r", n, hm, 1, d, 1, d, r2r_kind=plfft.R2RKind[kind])
    assert "fused" in plan.describe(), plan.describe()
    y = run_plan(plan, x, span(hm, d, n, 1), torch.float32)
    ref = oracle.r2r(gather(x, hm, d, n, 1).astype(np.float64), kind)
    assert oracle.rel_l2(gather(y, hm, d, n, 1), ref) <= oracle.fp32_tol(2 * n)


@pytest.mark.parametrize("n", [1024, 4096])
def test_fused_r2c_in_place(n):
    """In-place R2C with the padded layout (each member's output over its own input)."""
    import torch

    hm = 4
    h = n // 2 + 1
    rng = np.random.default_rng(3)
    buf = np.zeros(hm * 2 * h, np.float32)
    xs = rng.uniform(-1, 1, (hm, n)).astype(np.float32)
    for b in range(hm):
        buf[b * 2 * h: b * 2 * h + n] = xs[b]
    d = torch.from_numpy(buf).cuda()
    plan = plfft.make_plan("r2c", n, hm, 1, 2 * h, 1, h, alias=plfft.IoAlias.MAY_ALIAS)
    plan.execute(d.data_ptr(), d.data_ptr())
    y = d.cpu().numpy().view(np.complex64).reshape(hm, h)
    assert oracle.rel_l2(y, oracle.r2c(xs.astype(np.float64))) <= oracle.fp32_tol(n)


# half-length R2C / C2R (even n that is not twice a power of two): a length
# n/2 C2C over the real data read as complex pairs, with the split / merge
# kernel; odd real distances fall back to the full-length form.  Cases:
# smooth, Rader and Bluestein half lengths, a four-step half length over two
# chunks of members (the second one partial), strided complex sides.
HALF_CASES = [(6, 7, 6, 4, 1), (10, 5, 10, 6, 1), (100, 33, 100, 51, 1), (1000, 64, 1000, 501, 1),
              (2002, 9, 2002, 1002, 1), (2018, 6, 2018, 1010, 1), (2062, 6, 2062, 1032, 1),
              (1000, 5, 1001, 501, 1), (1000, 4, 1000, 1100, 2), (100000, 200, 100000, 50001, 1)]


@pytest.mark.parametrize("n,hm,rdist,cdist,cstride", HALF_CASES)
def test_real_half(n, hm, rdist, cdist, cstride):
    import torch

    h = n // 2 + 1
    rng = np.random.default_rng(n + hm)
    rows = np.unique(np.array([0, hm // 2, hm - 1]))
    x = rng.uniform(-1, 1, span(hm, rdist, n, 1)).astype(np.float32)
    f = plfft.make_plan("r2c", n, hm, 1, rdist, cstride, cdist)
    half = "half" in f.describe()
    assert half, f.describe()
    y = run_plan(f, x, span(hm, cdist, h, cstride), torch.complex64)
    got = gather(y, hm, cdist, h, cstride)[rows]
    ref = oracle.r2c(gather(x, hm, rdist, n, 1)[rows].astype(np.float64))
    assert oracle.rel_l2(got, ref) <= oracle.fp32_tol(n), f.describe()
    X = (rng.uniform(-1, 1, span(hm, cdist, h, cstride)) + 1j * rng.uniform(-1, 1, span(hm, cdist, h, cstride)))
    X = X.astype(np.complex64)
    b = plfft.make_plan("c2r", n, hm, cstride, cdist, 1, rdist, scale=1.0 / n)
    assert "half" in b.describe(), b.describe()
    z = run_plan(b, X, span(hm, rdist, n, 1), torch.float32)
    refz = oracle.c2r(gather(X, hm, cdist, h, cstride)[rows].astype(np.complex128), n) / n
    assert oracle.rel_l2(gather(z, hm, rdist, n, 1)[rows], refz) <= oracle.fp32_tol(n), b.describe()


@pytest.mark.parametrize("n", [1000, 2018])
def test_real_half_in_place(n):
    """In-place R2C then C2R over the padded layout (each member's complex
    output over its own real input)."""
    import torch

    hm = 7
    h = n // 2 + 1
    rng = np.random.default_rng(n)
    x = np.zeros((hm, 2 * h), np.float32)
    x[:, :n] = rng.uniform(-1, 1, (hm, n))
    d = torch.from_numpy(x.ravel().copy()).cuda()
    f = plfft.make_plan("r2c", n, hm, 1, 2 * h, 1, h, alias=plfft.IoAlias.MAY_ALIAS)
    assert "half" in f.describe(), f.describe()
    f.execute(d.data_ptr(), d.data_ptr())
    Y = d.cpu().numpy().view(np.complex64).reshape(hm, h)
    assert oracle.rel_l2(Y, oracle.r2c(x[:, :n].astype(np.float64))) <= oracle.fp32_tol(n)
    b = plfft.make_plan("c2r", n, hm, 1, h, 1, 2 * h, alias=plfft.IoAlias.MAY_ALIAS, scale=1.0 / n)
    b.execute(d.data_ptr(), d.data_ptr())
    z = d.cpu().numpy().reshape(hm, 2 * h)[:, :n]
    assert oracle.rel_l2(z, x[:, :n].astype(np.float64)) <= oracle.fp32_tol(n)
