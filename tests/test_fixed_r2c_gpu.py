"""Fixed-point R2C (Q0.15, Q0.7) on the device, through the C-ABI, against
the reference's own kernels' outputs (tests/golden/*_r2c_reference.npz) and
the bit-exact restatement (oracle/fixed.c): every case bit for bit.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

SIZES = [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]
TYPES = {"q15": (16, np.int16, np.int32, "Q15"), "q7": (8, np.int8, np.int16, "Q7")}


def _device_r2c(dtype, n, x, howmany, istride=1, idist=None, ostride=1, odist=None, out_words=None):
    """x: real lanes (int16 / int8) laid out with the given strides; returns
    the output buffer as (re, im) lane pairs."""
    import plfft
    import torch

    bits, lane, word, name = TYPES[dtype]
    h = n // 2 + 1
    idist = n if idist is None else idist
    odist = h if odist is None else odist
    plan = plfft.make_plan("r2c", n, howmany, istride, idist, ostride, odist, data_type=plfft.DataType[name])
    d_in = torch.from_numpy(np.ascontiguousarray(x).view(np.uint8).copy()).cuda()
    nout = out_words if out_words is not None else howmany * h
    d_out = torch.zeros(nout * 2 * np.dtype(lane).itemsize, dtype=torch.uint8, device="cuda")
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    return d_out.cpu().numpy().view(lane).reshape(nout, 2), plan


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", SIZES)
def test_fixed_r2c_matches_reference_kernels(dtype, n):
    g = np.load(__file__.replace("test_fixed_r2c_gpu.py", f"golden/{dtype}_r2c_reference.npz"))
    x = g[f"x_{n}"]
    hm = x.shape[0]
    y, plan = _device_r2c(dtype, n, x, hm)
    assert "r2c-" in plan.describe(), plan.describe()
    assert np.array_equal(y.reshape(hm, n // 2 + 1, 2), g[f"y_{n}"]), plan.describe()


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", [2, 4, 8, 16])
def test_fixed_r2c_odist_unit_matches_reference_kernels(dtype, n):
    """Members adjacent in the output (ostride = howmany, odist = 1): the
    reference's gu kernel variant, whose 4- and 8-point codelets round
    differently from the gs one."""
    g = np.load(__file__.replace("test_fixed_r2c_gpu.py", f"golden/{dtype}_r2c_reference.npz"))
    x = g[f"xu_{n}"]
    hm, h = x.shape[0], n // 2 + 1
    y, plan = _device_r2c(dtype, n, x, hm, 1, n, hm, 1)
    got = y.reshape(h, hm, 2).transpose(1, 0, 2)
    assert np.array_equal(got, g[f"yu_{n}"]), plan.describe()


# (istride, idist, ostride, odist) per kernel variant of the reference
# (providers/aot/aot_kernel_data.cpp:188-252), for howmany members of n
def _variant_layout(var, n, hm):
    h = n // 2 + 1
    return {"uu": (hm, 1, hm, 1), "us": (hm, 1, 1, h), "gu": (1, n, hm, 1), "gs": (1, n, 1, h)}[var]


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", [2, 4, 8, 16, 64, 128, 2048])
@pytest.mark.parametrize("var", ["uu", "us", "gu", "gs", "uun"])
def test_fixed_r2c_kernel_variants(dtype, n, var):
    """Every batch layout the reference picks a distinct kernel variant for,
    on extreme-heavy inputs, bit for bit against the restatement."""
    bits, lane, _, _ = TYPES[dtype]
    lo, hi = -(1 << (bits - 1)), (1 << (bits - 1)) - 1
    hm = 1 if var == "uun" else (257 if n <= 128 else 9)
    is_, id_, os_, od = _variant_layout("gs" if var == "uun" else var, n, hm)
    h = n // 2 + 1
    rng = np.random.default_rng(n * 7 + bits + len(var))
    ext = np.array([lo, lo + 1, hi - 1, hi])
    x = np.where(rng.random((hm, n)) < 0.85, rng.choice(ext, (hm, n)), rng.integers(lo, hi + 1, (hm, n))).astype(lane)
    buf = np.zeros((hm - 1) * id_ + (n - 1) * is_ + 1, lane)
    for b in range(hm):
        buf[b * id_:b * id_ + n * is_:is_][:n] = x[b]
    out_words = (hm - 1) * od + (h - 1) * os_ + 1
    y, plan = _device_r2c(dtype, n, buf, hm, is_, id_, os_, od, out_words=out_words)
    ref = oracle.fixed_r2c_strided(bits, buf, n, hm, is_, id_, os_, od, out_words)
    assert np.array_equal(y, ref), plan.describe()


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", SIZES)
def test_fixed_r2c_random_batches_bit_exact(dtype, n):
    bits, lane, _, _ = TYPES[dtype]
    lim = 1 << (bits - 1)
    rng = np.random.default_rng(300 + n + bits)
    hm = 1000 + 3  # ragged last CTA
    x = rng.integers(-lim, lim, (hm, n)).astype(lane)
    x[:5] = np.where(rng.random((5, n)) < 0.5, -lim, lim - 1)  # saturating members
    y, plan = _device_r2c(dtype, n, x, hm)
    ref = oracle.q15_r2c(x) if dtype == "q15" else oracle.q7_r2c(x)
    assert np.array_equal(y.reshape(hm, n // 2 + 1, 2), ref), plan.describe()


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", [8, 256, 2048])
def test_fixed_r2c_strided(dtype, n):
    """Member distances with gaps, an input stride of 2 and an output stride
    of 3 (the reference's batched layouts)."""
    bits, lane, _, _ = TYPES[dtype]
    lim = 1 << (bits - 1)
    hm, h = 7, n // 2 + 1
    idist, odist = 2 * n + 5, 3 * h + 2
    rng = np.random.default_rng(n)
    buf = rng.integers(-lim, lim, (hm - 1) * idist + 2 * (n - 1) + 1).astype(lane)
    y, plan = _device_r2c(dtype, n, buf, hm, 2, idist, 3, odist, out_words=(hm - 1) * odist + 3 * (h - 1) + 1)
    x = np.stack([buf[b * idist:b * idist + 2 * n:2] for b in range(hm)])
    ref = oracle.q15_r2c(x) if dtype == "q15" else oracle.q7_r2c(x)
    got = np.stack([y[b * odist:b * odist + 3 * h:3] for b in range(hm)])
    assert np.array_equal(got, ref), plan.describe()


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", [8, 64, 256, 1024])
def test_fixed_r2c_in_place(dtype, n):
    """In place over the padded layout (each member's bins over its own
    reals, idist = 2 (n/2 + 1) reals): the same bits as out of place."""
    import plfft
    import torch

    bits, lane, _, name = TYPES[dtype]
    lim = 1 << (bits - 1)
    hm, h = 300, n // 2 + 1
    rng = np.random.default_rng(n + bits)
    x = np.zeros((hm, 2 * h), lane)
    x[:, :n] = rng.integers(-lim, lim, (hm, n))
    d = torch.from_numpy(x.view(np.uint8).ravel().copy()).cuda()
    plan = plfft.make_plan("r2c", n, hm, 1, 2 * h, 1, h, alias=plfft.IoAlias.MAY_ALIAS,
                           data_type=plfft.DataType[name])
    plan.execute(d.data_ptr(), d.data_ptr())
    torch.cuda.synchronize()
    got = d.cpu().numpy().view(lane).reshape(hm, h, 2)
    ref = oracle.q15_r2c(x[:, :n]) if dtype == "q15" else oracle.q7_r2c(x[:, :n])
    assert np.array_equal(got, ref), plan.describe()


@pytest.mark.parametrize("name", ["Q15", "Q7"])
def test_fixed_real_unsupported_configs_fail_plan_creation(name):
    """Fixed-point R2C / C2R lengths outside the powers of two 2..4096 fail
    plan creation with the reference's status."""
    import plfft

    dt = plfft.DataType[name]
    for kind, n in (("r2c", 8192), ("r2c", 24), ("c2r", 8192), ("c2r", 24)):
        with pytest.raises(plfft.PlfftError) as e:
            plfft.make_plan(kind, n, 4, data_type=dt)
        assert e.value.status == plfft.Status.PLAN_CREATION_FAILED, (kind, n)
