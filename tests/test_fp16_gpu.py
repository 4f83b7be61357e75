"""FP16 (binary16) data type through the C-ABI: the device path widens the
caller's half data to FP32, runs the FP32 schedule and rounds the result to
half (round to nearest even), so the error against the FP64 oracle is the
half rounding of the output (~2^-11 relative per element).  The reference's
FP16 plans (include/plfft.h:143-154) take and return binary16 data with the
same layouts and conventions as FP32.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

TOL = 1e-3  # rel-L2: half output rounding (2^-11 ~ 4.9e-4 per element, worst case)


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).view(np.int16).ravel().copy()).cuda()


def _host(t, dtype, shape):
    return t.cpu().numpy().view(dtype).reshape(shape)


@pytest.mark.parametrize("n,howmany", [(1024, 16), (1000, 7), (97, 5), (65536, 2)])
@pytest.mark.parametrize("direction", [-1, 1])
def test_fp16_c2c(n, howmany, direction):
    import plfft
    import torch

    rng = np.random.default_rng(n)
    x = (rng.uniform(-1, 1, (howmany, n)) + 1j * rng.uniform(-1, 1, (howmany, n)))
    xh = np.stack([x.real, x.imag], -1).astype(np.float16)  # [hm, n, 2] halves
    plan = plfft.make_plan("c2c", n, howmany, direction=direction, data_type=plfft.DataType.FP16)
    assert "fp16" in plan.describe()
    d_in = _dev(xh)
    d_out = torch.zeros_like(d_in)
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    y = _host(d_out, np.float16, (howmany, n, 2)).astype(np.float64)
    ref = oracle.c2c(xh[..., 0].astype(np.float64) + 1j * xh[..., 1].astype(np.float64), direction, method="fft")
    assert oracle.rel_l2(y[..., 0] + 1j * y[..., 1], ref) <= TOL


@pytest.mark.parametrize("n", [4096, 1000])
def test_fp16_r2c_c2r_strided(n):
    import plfft
    import torch

    hm, h = 6, n // 2 + 1
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, (hm, n)).astype(np.float16)
    # input members interleaved (idist 1, istride hm), dense complex output
    r2c = plfft.make_plan("r2c", n, hm, hm, 1, 1, h, data_type=plfft.DataType.FP16)
    d_in = _dev(x.T.copy())
    d_spec = torch.zeros(hm * h * 2, dtype=torch.int16, device="cuda")
    r2c.execute(d_in.data_ptr(), d_spec.data_ptr())
    spec = _host(d_spec, np.float16, (hm, h, 2)).astype(np.float64)
    ref = oracle.r2c(x.astype(np.float64), method="fft")
    assert oracle.rel_l2(spec[..., 0] + 1j * spec[..., 1], ref) <= TOL
    c2r = plfft.make_plan("c2r", n, hm, data_type=plfft.DataType.FP16)
    d_back = torch.zeros(hm * n, dtype=torch.int16, device="cuda")
    c2r.execute(d_spec.data_ptr(), d_back.data_ptr())
    back = _host(d_back, np.float16, (hm, n)).astype(np.float64)
    ref2 = oracle.c2r(spec[..., 0] + 1j * spec[..., 1], n, method="fft")
    assert oracle.rel_l2(back, ref2) <= TOL


def test_fp16_dct2_in_place_and_host():
    import plfft

    n, hm = 1024, 4
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, (hm, n)).astype(np.float16)
    plan = plfft.make_plan("r2r", n, hm, r2r_kind=plfft.R2RKind.DCT_2, data_type=plfft.DataType.FP16,
                           alias=plfft.IoAlias.MAY_ALIAS)
    buf = x.copy()
    plan.execute(buf.ctypes.data, buf.ctypes.data)  # host pointers, in place
    ref = oracle.r2r(x.astype(np.float64), "DCT_2")
    assert oracle.rel_l2(buf.astype(np.float64), ref) <= TOL


def test_fp16_c2c_in_place():
    import plfft
    import torch

    n, hm = 4096, 8
    rng = np.random.default_rng(11)
    xh = np.stack([rng.uniform(-1, 1, (hm, n)), rng.uniform(-1, 1, (hm, n))], -1).astype(np.float16)
    plan = plfft.make_plan("c2c", n, hm, direction=-1, data_type=plfft.DataType.FP16,
                           alias=plfft.IoAlias.MAY_ALIAS)
    d = _dev(xh)
    plan.execute(d.data_ptr(), d.data_ptr())
    y = _host(d, np.float16, (hm, n, 2)).astype(np.float64)
    ref = oracle.c2c(xh[..., 0].astype(np.float64) + 1j * xh[..., 1].astype(np.float64), -1, method="fft")
    assert oracle.rel_l2(y[..., 0] + 1j * y[..., 1], ref) <= TOL
