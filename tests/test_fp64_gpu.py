"""FP64 data type through the C-ABI against the FP64 oracle.

The reference's FP64 tests bound batched R2C/C2R errors by 1e-11
(test/r2c_c2r_1d_batched.cpp:33-38); C2C uses eps * 4 * log2(n)
(test/test_utils.hpp:122-130 scaled to rel-L2).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def tol64(n):
    return 4 * max(1.0, np.log2(max(n, 2))) * 2.0 ** -52 * 8


def _run(kind, n, hm, x, direction=-1, istride=1, idist=None, ostride=1, odist=None, nout=None):
    import plfft
    import torch

    plan = plfft.make_plan(kind, n, hm, istride, idist, ostride, odist, direction=direction,
                           data_type=plfft.DataType.FP64)
    assert "fp64" in plan.describe()
    d_in = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    d_out = torch.zeros(nout, dtype=d_in.dtype if kind != "c2r" else torch.float64, device="cuda") \
        if kind != "r2c" else torch.zeros(nout, dtype=torch.complex128, device="cuda")
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    return d_out.cpu().numpy(), plan


@pytest.mark.parametrize("n", [1, 8, 60, 97, 1024, 4096, 1000, 3 * 4096, 1 << 16, 11 * 13])
@pytest.mark.parametrize("direction", [-1, 1])
def test_fp64_c2c(n, direction):
    rng = np.random.default_rng(n)
    hm = 3
    x = rng.uniform(-1, 1, (hm, n)) + 1j * rng.uniform(-1, 1, (hm, n))
    got, plan = _run("c2c", n, hm, x.ravel(), direction, nout=hm * n)
    ref = oracle.c2c(x, direction, method="fft")
    assert oracle.rel_l2(got.reshape(hm, n), ref) <= tol64(n), plan.describe()


def test_fp64_c2c_strided():
    n, hm, is_, os_ = 1024, 4, 2, 3
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, (hm, n)) + 1j * rng.uniform(-1, 1, (hm, n))
    buf = np.zeros(hm * n * is_, np.complex128)
    idx = np.arange(hm)[:, None] * n * is_ + np.arange(n)[None, :] * is_
    buf[idx] = x
    got, _ = _run("c2c", n, hm, buf, -1, is_, n * is_, os_, n * os_, nout=hm * n * os_)
    oidx = np.arange(hm)[:, None] * n * os_ + np.arange(n)[None, :] * os_
    assert oracle.rel_l2(got[oidx], oracle.c2c(x, -1, method="fft")) <= tol64(n)


@pytest.mark.parametrize("n", [16, 1000, 4096, 3 * 4096, 97])
def test_fp64_r2c_c2r(n):
    rng = np.random.default_rng(n + 1)
    hm, h = 6, n // 2 + 1
    x = rng.uniform(-1, 1, (hm, n))
    spec, plan = _run("r2c", n, hm, x.ravel(), nout=hm * h)
    ref = oracle.r2c(x, method="fft")
    assert oracle.rel_l2(spec.reshape(hm, h), ref) <= 1e-11, plan.describe()
    back, plan2 = _run("c2r", n, hm, spec, nout=hm * n)
    assert oracle.rel_l2(back.reshape(hm, n), n * x) <= 1e-11, plan2.describe()


R2R = ["DCT_1", "DCT_2", "DCT_3", "DCT_4", "DST_1", "DST_2", "DST_3", "DST_4", "DHT", "R2HC", "HC2R"]


@pytest.mark.parametrize("kind", R2R)
@pytest.mark.parametrize("n", [2, 17, 64, 1000])
def test_fp64_r2r(kind, n):
    """Every R2R kind in FP64: double pre/post passes around the FP64 C2C."""
    import plfft
    import torch

    rng = np.random.default_rng(hash((kind, n)) % 2**32)
    hm = 3
    x = rng.uniform(-1, 1, (hm, n))
    plan = plfft.make_plan("r2r", n, hm, r2r_kind=plfft.R2RKind[kind], data_type=plfft.DataType.FP64)
    assert "fp64" in plan.describe(), plan.describe()
    d_in = torch.from_numpy(x.ravel().copy()).cuda()
    d_out = torch.zeros(hm * n, dtype=torch.float64, device="cuda")
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    ref = oracle.r2r(x, kind)
    assert oracle.rel_l2(d_out.cpu().numpy().reshape(hm, n), ref) <= tol64(2 * n), plan.describe()


def test_fp64_r2r_strided_scaled():
    import plfft
    import torch

    n, hm, is_, os_ = 64, 2, 2, 3
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, (hm, n))
    buf = np.zeros(hm * n * is_)
    buf[np.arange(hm)[:, None] * n * is_ + np.arange(n)[None, :] * is_] = x
    plan = plfft.make_plan("r2r", n, hm, is_, n * is_, os_, n * os_, r2r_kind=plfft.R2RKind.DST_2,
                           data_type=plfft.DataType.FP64, scale=0.25)
    d_in = torch.from_numpy(buf).cuda()
    d_out = torch.zeros(hm * n * os_, dtype=torch.float64, device="cuda")
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    got = d_out.cpu().numpy()[np.arange(hm)[:, None] * n * os_ + np.arange(n)[None, :] * os_]
    assert oracle.rel_l2(got, 0.25 * oracle.r2r(x, "DST_2")) <= tol64(2 * n)


@pytest.mark.parametrize("n", [1024, 3 * 4096, 97])
def test_fp64_c2c_in_place_host(n):
    """In place on host buffers (staged through the device)."""
    import plfft

    rng = np.random.default_rng(n + 7)
    hm = 3
    x = rng.uniform(-1, 1, (hm, n)) + 1j * rng.uniform(-1, 1, (hm, n))
    buf = x.copy()
    plan = plfft.make_plan("c2c", n, hm, direction=1, data_type=plfft.DataType.FP64,
                           alias=plfft.IoAlias.MAY_ALIAS)
    plan.execute(buf.ctypes.data, buf.ctypes.data)
    assert oracle.rel_l2(buf, oracle.c2c(x, 1, method="fft")) <= tol64(n)
