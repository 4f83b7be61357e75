"""Fixed-point C2R (Q0.15, Q0.7) on the device, through the C-ABI, against
the reference's own kernels' outputs (tests/golden/*_c2r_reference.npz) and
the bit-exact restatement (oracle/fixed.c): every case bit for bit.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

SIZES = [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]
TYPES = {"q15": (16, np.int16, "Q15"), "q7": (8, np.int8, "Q7")}


def _device_c2r(dtype, n, buf, howmany, istride=1, idist=None, ostride=1, odist=None, out_len=None):
    """buf: complex lanes [elements, 2] laid out with the given strides;
    returns the flat real output."""
    import plfft
    import torch

    bits, lane, name = TYPES[dtype]
    h = n // 2 + 1
    idist = h if idist is None else idist
    odist = n if odist is None else odist
    plan = plfft.make_plan("c2r", n, howmany, istride, idist, ostride, odist, data_type=plfft.DataType[name])
    d_in = torch.from_numpy(np.ascontiguousarray(buf).view(np.uint8).ravel().copy()).cuda()
    nout = out_len if out_len is not None else howmany * n
    d_out = torch.zeros(nout * np.dtype(lane).itemsize, dtype=torch.uint8, device="cuda")
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    return d_out.cpu().numpy().view(lane), plan


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", SIZES)
def test_fixed_c2r_matches_reference_kernels(dtype, n):
    g = np.load(__file__.replace("test_fixed_c2r_gpu.py", f"golden/{dtype}_c2r_reference.npz"))
    X = g[f"x_{n}"]
    hm, h = X.shape[0], n // 2 + 1
    y, plan = _device_c2r(dtype, n, X.reshape(-1, 2), hm)
    assert "c2r-" in plan.describe(), plan.describe()
    assert np.array_equal(y.reshape(hm, n), g[f"y_{n}"]), plan.describe()
    if n <= 256:  # members adjacent: istride = ostride = howmany, idist = odist = 1
        buf = np.ascontiguousarray(X.transpose(1, 0, 2)).reshape(-1, 2)
        y, plan = _device_c2r(dtype, n, buf, hm, hm, 1, hm, 1)
        assert np.array_equal(y.reshape(n, hm).T, g[f"yu_{n}"]), plan.describe()


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", SIZES)
def test_fixed_c2r_random_batches_bit_exact(dtype, n):
    bits, lane, _ = TYPES[dtype]
    lo, hi = -(1 << (bits - 1)), (1 << (bits - 1)) - 1
    hm, h = 1003, n // 2 + 1  # ragged last CTA
    rng = np.random.default_rng(700 + n + bits)
    X = rng.integers(lo, hi + 1, (hm, h, 2)).astype(lane)
    X[:40] = np.where(rng.random((40, h, 2)) < 0.8, rng.choice([lo, hi, lo + 1, hi - 1], (40, h, 2)), X[:40])
    y, plan = _device_c2r(dtype, n, X.reshape(-1, 2), hm)
    ref = oracle.q15_c2r(X, n) if dtype == "q15" else oracle.q7_c2r(X, n)
    assert np.array_equal(y.reshape(hm, n), ref), plan.describe()


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", [8, 256, 2048])
def test_fixed_c2r_strided(dtype, n):
    """An input stride of 2 with gapped member distances, an output stride
    of 3 (the reference's batched layouts)."""
    bits, lane, _ = TYPES[dtype]
    lim = 1 << (bits - 1)
    hm, h = 7, n // 2 + 1
    idist, odist = 2 * h + 3, 3 * n + 1
    rng = np.random.default_rng(n)
    buf = rng.integers(-lim, lim, ((hm - 1) * idist + 2 * (h - 1) + 1, 2)).astype(lane)
    out_len = (hm - 1) * odist + 3 * (n - 1) + 1
    y, plan = _device_c2r(dtype, n, buf, hm, 2, idist, 3, odist, out_len=out_len)
    ref = oracle.fixed_c2r_strided(bits, buf, n, hm, 2, idist, 3, odist, out_len)
    assert np.array_equal(y, ref), plan.describe()


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", [8, 64, 256, 1024])
def test_fixed_c2r_in_place(dtype, n):
    """In place: each member's reals over its own bins (idist = n/2 + 1
    complex elements, odist = n + 2 reals)."""
    import plfft
    import torch

    bits, lane, name = TYPES[dtype]
    lim = 1 << (bits - 1)
    hm, h = 300, n // 2 + 1
    rng = np.random.default_rng(n + bits + 1)
    X = rng.integers(-lim, lim, (hm, h, 2)).astype(lane)
    d = torch.from_numpy(X.view(np.uint8).ravel().copy()).cuda()
    plan = plfft.make_plan("c2r", n, hm, 1, h, 1, 2 * h, alias=plfft.IoAlias.MAY_ALIAS,
                           data_type=plfft.DataType[name])
    plan.execute(d.data_ptr(), d.data_ptr())
    torch.cuda.synchronize()
    got = d.cpu().numpy().view(lane).reshape(hm, 2 * h)[:, :n]
    ref = oracle.q15_c2r(X, n) if dtype == "q15" else oracle.q7_c2r(X, n)
    assert np.array_equal(got, ref), plan.describe()
