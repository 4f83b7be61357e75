"""Q0.15 C2C on the device (through the C-ABI) vs the reference's own
kernels' outputs (tests/golden/q15_reference.npz) and the bit-exact oracle
(oracle/fixed.c): every case must match bit for bit.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]


def _device_q15(n, buf_in, howmany, direction, istride=1, idist=None, ostride=1, odist=None, out_words=None,
                alias=False):
    """Runs a Q15 plan on int16 (re, im) words held as int32; returns the output words."""
    import plfft
    import torch

    idist = n if idist is None else idist
    odist = n if odist is None else odist
    plan = plfft.make_plan("c2c", n, howmany, istride, idist, ostride, odist, direction=direction,
                           data_type=plfft.DataType.Q15,
                           alias=plfft.IoAlias.MAY_ALIAS if alias else plfft.IoAlias.NO_ALIAS)
    d_in = torch.from_numpy(buf_in.view(np.int32).copy()).cuda()
    if alias:
        d_out = d_in
    else:
        d_out = torch.zeros(out_words, dtype=torch.int32, device="cuda")
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    return d_out.cpu().numpy(), plan


@pytest.mark.parametrize("n", SIZES[1:])
@pytest.mark.parametrize("d", ["f", "b"])
def test_q15_matches_reference_kernels(n, d):
    g = np.load(__file__.replace("test_q15_gpu.py", "golden/q15_reference.npz"))
    x = g[f"x_{n}"]
    hm = x.shape[0]
    out, plan = _device_q15(n, x, hm, -1 if d == "f" else 1, out_words=hm * n)
    assert np.array_equal(out.view(np.int16).reshape(x.shape), g[f"y_{n}_{d}"]), plan.describe()
    out1, _ = _device_q15(n, x[:1], 1, -1 if d == "f" else 1, out_words=n)
    assert np.array_equal(out1.view(np.int16).reshape(1, n, 2), g[f"y1_{n}_{d}"])


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("direction", [-1, 1])
def test_q15_random_batches_bit_exact(n, direction):
    rng = np.random.default_rng(100 + n)
    hm = 2000 + 3  # ragged last CTA
    x = rng.integers(-32768, 32768, (hm, n, 2)).astype(np.int16)
    x[:7] = np.where(rng.random((7, n, 2)) < 0.5, -32768, 32767)  # saturating members
    out, plan = _device_q15(n, x, hm, direction, out_words=hm * n)
    ref = oracle.q15_c2c(x, direction)
    assert np.array_equal(out.view(np.int16).reshape(x.shape), ref), plan.describe()


@pytest.mark.parametrize("n", [4, 16, 256, 1024])
def test_q15_strided_layouts_and_guard_words(n):
    """Interleaved members (idist = 1, istride = howmany) in; strided out with
    gaps whose words must stay untouched."""
    rng = np.random.default_rng(5)
    hm, os_, od = 5, 2, 2 * n + 3
    xs = rng.integers(-32768, 32768, (hm, n, 2)).astype(np.int16)
    inter = np.ascontiguousarray(xs.transpose(1, 0, 2))  # element k of member b at k*hm + b
    total = (hm - 1) * od + (n - 1) * os_ + 1 + 8
    import plfft
    import torch

    plan = plfft.make_plan("c2c", n, hm, hm, 1, os_, od, direction=-1, data_type=plfft.DataType.Q15)
    d_in = torch.from_numpy(inter.view(np.int32).ravel().copy()).cuda()
    sentinel = np.int32(0x5A5AA5A5)
    d_out = torch.full((total,), int(sentinel), dtype=torch.int32, device="cuda")
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    got = d_out.cpu().numpy()
    idx = (np.arange(hm)[:, None] * od + np.arange(n)[None, :] * os_)
    ref = oracle.q15_c2c(xs, -1).view(np.int32).reshape(hm, n)
    assert np.array_equal(got[idx], ref)
    mask = np.ones(total, bool)
    mask[idx.ravel()] = False
    assert np.all(got[mask] == sentinel)


@pytest.mark.parametrize("n", [8, 128, 2048])
def test_q15_in_place(n):
    rng = np.random.default_rng(9)
    hm = 77
    x = rng.integers(-32768, 32768, (hm, n, 2)).astype(np.int16)
    out, _ = _device_q15(n, x, hm, 1, alias=True)
    assert np.array_equal(out.view(np.int16).reshape(x.shape), oracle.q15_c2c(x, 1))


def test_q15_unsupported_configs_fail_plan_creation():
    import plfft

    for kw in ({"n": 8192}, {"n": 24}):
        with pytest.raises(plfft.PlfftError) as e:
            plfft.make_plan("c2c", kw["n"], 4, data_type=plfft.DataType.Q15)
        assert e.value.status == plfft.Status.PLAN_CREATION_FAILED
    with pytest.raises(plfft.PlfftError) as e:  # fixed-point R2R (reference src/plfft.cpp:248-261)
        plfft.make_plan("r2r", 16, 1, r2r_kind=plfft.R2RKind.DCT_2, data_type=plfft.DataType.Q15)
    assert e.value.status == plfft.Status.PLAN_CREATION_FAILED
