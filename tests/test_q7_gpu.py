"""Q0.7 C2C on the device (through the C-ABI) vs the reference's own
kernels' outputs (tests/golden/q7_reference.npz) and the bit-exact oracle
(oracle/fixed.c): every case must match bit for bit.

Layouts follow the reference's own Q0.7 test list (test/c2c_q0_7.cpp:15-24:
single members, contiguous batches, element stride 2 with distance 20,
stride 8 with distance 600).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]


def _device_q7(n, buf, howmany, direction, istride=1, idist=None, ostride=1, odist=None, out_elems=None,
               alias=False, fill=0):
    """Runs a Q7 plan on int8 (re, im) pairs held as int16 words; returns the output words."""
    import plfft
    import torch

    idist = n if idist is None else idist
    odist = n if odist is None else odist
    plan = plfft.make_plan("c2c", n, howmany, istride, idist, ostride, odist, direction=direction,
                           data_type=plfft.DataType.Q7,
                           alias=plfft.IoAlias.MAY_ALIAS if alias else plfft.IoAlias.NO_ALIAS)
    d_in = torch.from_numpy(np.ascontiguousarray(buf).view(np.int16).reshape(-1).copy()).cuda()
    d_out = d_in if alias else torch.full((out_elems,), fill, dtype=torch.int16, device="cuda")
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    return d_out.cpu().numpy(), plan


@pytest.mark.parametrize("n", SIZES[1:])
@pytest.mark.parametrize("d", ["f", "b"])
def test_q7_matches_reference_kernels(n, d):
    g = np.load(__file__.replace("test_q7_gpu.py", "golden/q7_reference.npz"))
    x = g[f"x_{n}"]
    hm = x.shape[0]
    out, plan = _device_q7(n, x, hm, -1 if d == "f" else 1, out_elems=hm * n)
    assert np.array_equal(out.view(np.int8).reshape(x.shape), g[f"y_{n}_{d}"]), plan.describe()
    out1, _ = _device_q7(n, x[:1], 1, -1 if d == "f" else 1, out_elems=n)
    assert np.array_equal(out1.view(np.int8).reshape(1, n, 2), g[f"y1_{n}_{d}"])


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("direction", [-1, 1])
def test_q7_random_batches_bit_exact(n, direction):
    rng = np.random.default_rng(300 + n)
    hm = 1000 + 3  # ragged last CTA
    x = rng.integers(-128, 128, (hm, n, 2)).astype(np.int8)
    x[:7] = np.where(rng.random((7, n, 2)) < 0.5, -128, 127)  # saturating members
    out, plan = _device_q7(n, x, hm, direction, out_elems=hm * n)
    assert np.array_equal(out.view(np.int8).reshape(x.shape), oracle.q7_c2c(x, direction)), plan.describe()


@pytest.mark.parametrize("case", [(8, 3, 2, 20, 2, 20), (64, 2, 8, 600, 8, 600), (1024, 3, 2, 2100, 3, 3200)])
def test_q7_reference_strided_layouts_and_guard_words(case):
    """Strided members (test/c2c_q0_7.cpp:19-20); words between outputs stay untouched."""
    n, hm, is_, id_, os_, od = case
    rng = np.random.default_rng(n)
    xs = rng.integers(-128, 128, (hm, n, 2)).astype(np.int8)
    span_i = (hm - 1) * id_ + (n - 1) * is_ + 1
    buf = np.zeros((span_i, 2), np.int8)
    idx_i = np.arange(hm)[:, None] * id_ + np.arange(n)[None, :] * is_
    buf[idx_i] = xs
    total = (hm - 1) * od + (n - 1) * os_ + 1 + 8
    sentinel = np.int16(0x5AA5)
    out, plan = _device_q7(n, buf, hm, -1, is_, id_, os_, od, out_elems=total, fill=int(sentinel))
    idx_o = np.arange(hm)[:, None] * od + np.arange(n)[None, :] * os_
    ref = oracle.q7_c2c(xs, -1).view(np.int16).reshape(hm, n)
    assert np.array_equal(out[idx_o], ref), plan.describe()
    mask = np.ones(total, bool)
    mask[idx_o.ravel()] = False
    assert np.all(out[mask] == sentinel)


@pytest.mark.parametrize("n", [8, 256, 1024])
def test_q7_in_place(n):
    rng = np.random.default_rng(9)
    hm = 37
    x = rng.integers(-128, 128, (hm, n, 2)).astype(np.int8)
    out, _ = _device_q7(n, x, hm, 1, alias=True)
    assert np.array_equal(out.view(np.int8).reshape(x.shape), oracle.q7_c2c(x, 1))


def test_q7_host_buffers():
    import plfft

    n, hm = 512, 64
    rng = np.random.default_rng(4)
    x = rng.integers(-128, 128, (hm, n, 2)).astype(np.int8)
    y = np.zeros_like(x)
    plan = plfft.make_plan("c2c", n, hm, data_type=plfft.DataType.Q7)
    plan.execute(x.ctypes.data, y.ctypes.data)
    assert np.array_equal(y, oracle.q7_c2c(x, -1))


def test_q7_unsupported_configs_fail_plan_creation():
    import plfft

    for n in (8192, 24):
        with pytest.raises(plfft.PlfftError) as e:
            plfft.make_plan("c2c", n, 4, data_type=plfft.DataType.Q7)
        assert e.value.status == plfft.Status.PLAN_CREATION_FAILED
