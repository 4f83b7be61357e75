"""Parity at the exact shapes the benchmark times.

Every benchmarked configuration is run here at its full batch through the
C-ABI and every member is compared with the FP64 oracle (the Q0.15 one bit
for bit with the fixed-point restatement).  At these batch sizes the
persistent kernels walk their shared-memory rings past the wrap-around
(the power-of-two ring kernel reuses each slot several times per CTA at
N=1024 x 4096), the last CTA holds a partial group, and the four-step and
convolution schedules run several workspace chunks -- none of which the
small parity cases reach.

Checks: FP32 rel-L2 <= 4*log2(N)*2^-24 over the whole batch and per member;
split-BF16 rel-L2 <= 1e-6; Q0.15 bit-exact.  Where the oracle's direct sums
are too slow for a full batch, the whole batch is checked against the FP64
FFT (itself pinned to the direct sums in tests/test_oracle.py) and a spread
sample of members against the direct sums.

Shapes follow the benchmark configurations: C2C N=1024 x 4096; R2C and
C2R(1/N) N=4096 x 8192; DCT-II / DST-II N=1024 x 4096; Q0.15 N=256 x 16384;
FP32 and split-BF16 N=2^20 x 64 and N=2^16 x 1024; the 4000-transform
grouped mix.
"""
import numpy as np
import pytest

import oracle
import plfft

pytestmark = pytest.mark.gpu


def _per_member_ok(got, ref, tol):
    """rel-L2 of every member (rows) within tol; returns the worst."""
    num = np.linalg.norm(got - ref, axis=-1)
    den = np.linalg.norm(ref, axis=-1)
    rel = num / np.maximum(den, 1e-300)
    return float(rel.max()), bool(np.all(rel <= tol))


def _spread(howmany, count=64, seed=0):
    """Member indices spread over the batch, always including the first and
    the last few (the final partial group of the last CTAs)."""
    rng = np.random.default_rng(seed)
    pick = set(rng.choice(howmany, min(count, howmany), replace=False).tolist())
    pick.update(range(min(4, howmany)))
    pick.update(range(max(0, howmany - 8), howmany))
    return np.array(sorted(pick))


def _dev_complex(shape, seed):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    n = int(np.prod(shape))
    return torch.complex(torch.rand(n, device="cuda", generator=g) * 2 - 1,
                         torch.rand(n, device="cuda", generator=g) * 2 - 1)


@pytest.mark.parametrize("howmany", [4096, 4096 * 4 + 3])
def test_c2c_n1024_full_batch(howmany):
    """Headline shape (and a ragged 4x batch): every member against the FP64 FFT,
    64 spread members against the direct DFT."""
    import torch

    n = 1024
    plan = plfft.make_plan("c2c", n, howmany, direction=plfft.FORWARD)
    x = _dev_complex((howmany, n), seed=howmany)
    y = torch.full_like(x, complex(3.0, 3.0))
    plan.execute(x.data_ptr(), y.data_ptr())
    xs = x.cpu().numpy().reshape(howmany, n).astype(np.complex128)
    got = y.cpu().numpy().reshape(howmany, n)
    ref = oracle.c2c(xs, -1, method="fft")
    tol = oracle.fp32_tol(n)
    assert oracle.rel_l2(got, ref) <= tol, plan.describe()
    worst, ok = _per_member_ok(got, ref, tol)
    assert ok, (worst, plan.describe())
    idx = _spread(howmany)
    assert oracle.rel_l2(got[idx], oracle.c2c(xs[idx], -1, method="dft")) <= tol


def test_c2c_n1024_full_batch_backward_scaled():
    import torch

    n, howmany = 1024, 4096
    plan = plfft.make_plan("c2c", n, howmany, direction=plfft.BACKWARD, scale=1.0 / n)
    x = _dev_complex((howmany, n), seed=5)
    y = torch.empty_like(x)
    plan.execute(x.data_ptr(), y.data_ptr())
    ref = oracle.c2c(x.cpu().numpy().reshape(howmany, n).astype(np.complex128), 1, method="fft") / n
    worst, ok = _per_member_ok(y.cpu().numpy().reshape(howmany, n), ref, oracle.fp32_tol(n))
    assert ok, worst


def test_c2c_n1024_async_rotating_buffers():
    """The benchmark's step: execute_async over rotating buffer sets on one
    stream, many times in a row; the last result of each set is checked."""
    import torch

    n, howmany, sets = 1024, 4096, 3
    plan = plfft.make_plan("c2c", n, howmany)
    xs = [_dev_complex((howmany, n), seed=100 + s) for s in range(sets)]
    ys = [torch.empty_like(xs[0]) for _ in range(sets)]
    ws = torch.empty(max(1, plan.workspace_size()), dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    for i in range(30):
        plan.execute_async(xs[i % sets].data_ptr(), ys[i % sets].data_ptr(), ws.data_ptr(), st)
    torch.cuda.synchronize()
    for s in range(sets):
        ref = oracle.c2c(xs[s].cpu().numpy().reshape(howmany, n).astype(np.complex128), -1, method="fft")
        worst, ok = _per_member_ok(ys[s].cpu().numpy().reshape(howmany, n), ref, oracle.fp32_tol(n))
        assert ok, (s, worst)


def test_r2c_c2r_n4096_full_batch():
    """R2C then C2R(1/N), N=4096 x 8192: every member of both against the oracle."""
    import torch

    n, howmany = 4096, 8192
    h = n // 2 + 1
    f = plfft.make_plan("r2c", n, howmany)
    b = plfft.make_plan("c2r", n, howmany, scale=1.0 / n)
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    x = torch.rand(howmany * n, device="cuda", generator=g) * 2 - 1
    X = torch.empty(howmany * h, dtype=torch.complex64, device="cuda")
    z = torch.empty_like(x)
    f.execute(x.data_ptr(), X.data_ptr())
    b.execute(X.data_ptr(), z.data_ptr())
    xs = x.cpu().numpy().reshape(howmany, n).astype(np.float64)
    Xg = X.cpu().numpy().reshape(howmany, h)
    ref = oracle.r2c(xs, method="fft")
    tol = oracle.fp32_tol(n)
    worst, ok = _per_member_ok(Xg, ref, tol)
    assert ok, ("r2c", worst, f.describe())
    # C2R on the device's own spectrum against the oracle's C2R of that spectrum
    refz = oracle.c2r(Xg.astype(np.complex128), n, method="fft") / n
    worst, ok = _per_member_ok(z.cpu().numpy().reshape(howmany, n), refz, tol)
    assert ok, ("c2r", worst, b.describe())
    idx = _spread(howmany, 16)
    assert oracle.rel_l2(Xg[idx], oracle.r2c(xs[idx], method="dft")) <= tol


def _r2r_fft_ref(x, kind):
    """DCT-II / DST-II (FFTW REDFT10 / RODFT10) of every row from the FP64
    FFT of the length-2N even / odd extension."""
    n = x.shape[-1]
    k = np.arange(n)
    sign = 1.0 if kind == "DCT_2" else -1.0
    ext = np.concatenate([x, sign * x[:, ::-1]], axis=1).astype(np.complex128)
    F = oracle.c2c(ext, -1, method="fft")
    if kind == "DCT_2":
        return (np.exp(-1j * np.pi * k / (2 * n)) * F[:, :n]).real
    return -(np.exp(-1j * np.pi * (k + 1) / (2 * n)) * F[:, 1:n + 1]).imag


@pytest.mark.parametrize("kind", ["DCT_2", "DST_2"])
def test_r2r_n1024_full_batch(kind):
    import torch

    n, howmany = 1024, 4096
    plan = plfft.make_plan("r2r", n, howmany, r2r_kind=plfft.R2RKind[kind])
    g = torch.Generator(device="cuda")
    g.manual_seed(12)
    x = torch.rand(howmany * n, device="cuda", generator=g) * 2 - 1
    y = torch.full_like(x, 5.0)
    plan.execute(x.data_ptr(), y.data_ptr())
    xs = x.cpu().numpy().reshape(howmany, n).astype(np.float64)
    got = y.cpu().numpy().reshape(howmany, n)
    tol = oracle.fp32_tol(2 * n)
    worst, ok = _per_member_ok(got, _r2r_fft_ref(xs, kind), tol)
    assert ok, (worst, plan.describe())
    idx = _spread(howmany)
    assert oracle.rel_l2(got[idx], oracle.r2r(xs[idx], kind)) <= tol


def test_q15_n256_full_batch_bit_exact():
    """Q0.15 N=256 x 16384, int16 uniform in [-2^14, 2^14): every member bit for bit."""
    import torch

    n, howmany = 256, 16384
    plan = plfft.make_plan("c2c", n, howmany, data_type=plfft.DataType.Q15)
    rng = np.random.default_rng(13)
    xq = rng.integers(-(1 << 14), 1 << 14, (howmany, n, 2)).astype(np.int16)
    d_in = torch.from_numpy(xq.view(np.int32).reshape(-1).copy()).cuda()
    d_out = torch.full_like(d_in, 0x5A5A5A5A)
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    got = d_out.cpu().numpy().view(np.int16).reshape(howmany, n, 2)
    ref = oracle.q15_c2c(xq, -1)
    bad = np.nonzero(np.any(got != ref, axis=(1, 2)))[0]
    assert bad.size == 0, (bad[:10], plan.describe())


def test_q15_r2c_n256_full_batch_bit_exact():
    """Q0.15 R2C N=256 x 16384 (the bench's R2C workload), int16 reals over
    the full range: every member's bins bit for bit, nothing written past
    the output."""
    import torch

    n, howmany = 256, 16384
    h = n // 2 + 1
    plan = plfft.make_plan("r2c", n, howmany, data_type=plfft.DataType.Q15)
    rng = np.random.default_rng(17)
    x = rng.integers(-(1 << 15), 1 << 15, (howmany, n)).astype(np.int16)
    d_in = torch.from_numpy(x.reshape(-1).copy()).cuda()
    d_out = torch.full((howmany * h + 64,), 0x5A5A5A5A, dtype=torch.int32, device="cuda")
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    out = d_out.cpu().numpy()
    assert np.all(out[howmany * h:] == 0x5A5A5A5A)
    got = out[:howmany * h].view(np.int16).reshape(howmany, h, 2)
    ref = oracle.q15_r2c(x)
    bad = np.nonzero(np.any(got != ref, axis=(1, 2)))[0]
    assert bad.size == 0, (bad[:10], plan.describe())


def _impulse_input(howmany, n, seed):
    """U[-1,1) re/im plus a +-1e3 impulse at a seeded bin per member."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (howmany, n)) + 1j * rng.uniform(-1, 1, (howmany, n))
    x[np.arange(howmany), rng.integers(0, n, howmany)] += 1e3 * rng.choice([-1, 1], howmany)
    return x.astype(np.complex64)


@pytest.mark.parametrize("n,howmany", [(1 << 16, 1024), (1 << 20, 64)])
@pytest.mark.parametrize("precision", ["fp32", "split_bf16"])
def test_long_c2c_full_batch(n, howmany, precision):
    """The precision configurations at their benchmark batch: plain FP32 at the
    FP32 gate, split-BF16 at rel-L2 <= 1e-6, every member."""
    import torch

    prec = plfft.Precision.SPLIT_BF16 if precision == "split_bf16" else plfft.Precision.FP32
    plan = plfft.make_plan("c2c", n, howmany, precision=prec)
    x = _impulse_input(howmany, n, seed=n + howmany)
    d = torch.from_numpy(x.ravel()).cuda()
    y = torch.empty_like(d)
    plan.execute(d.data_ptr(), y.data_ptr())
    got = y.cpu().numpy().reshape(howmany, n)
    del d, y
    ref = oracle.c2c(x.astype(np.complex128), -1, method="fft")
    tol = 1e-6 if precision == "split_bf16" else oracle.fp32_tol(n)
    worst, ok = _per_member_ok(got, ref, tol)
    err = oracle.rel_l2(got, ref)
    print(f"{precision} n={n} x{howmany}: rel-L2 {err:.3e}, worst member {worst:.3e}, "
          f"max-abs {np.abs(got - ref).max():.3e}")
    assert ok, (worst, plan.describe())
    # direct-sum spot check of a few bins of a few members (O(N) per bin)
    rng = np.random.default_rng(1)
    for m in (0, howmany // 2, howmany - 1):
        bins = rng.integers(0, n, 8)
        j = np.arange(n)
        for kbin in bins:
            w = np.exp(-2j * np.pi * ((j * int(kbin)) % n) / n)
            exact = np.sum(x[m].astype(np.complex128) * w)
            assert abs(got[m, kbin] - exact) <= 8 * tol * np.linalg.norm(ref[m]) / np.sqrt(n) + 1e-3


def test_grouped_4000_full_mix():
    """The 4000-transform grouped benchmark mix: every transform against the oracle."""
    import torch

    from helpers import grouped_lengths

    L = np.array(sorted(grouped_lengths(4000, seed=2026)), np.int64)
    offs = np.concatenate([[0], np.cumsum(L)[:-1]]).astype(np.int64)
    total = int(L.sum())
    group = plfft.Group(L, offs, offs, plfft.FORWARD)
    x = _dev_complex((total,), seed=77)
    y = torch.full_like(x, complex(9.0, 9.0))
    group.execute_async(x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    xs = x.cpu().numpy()
    ys = y.cpu().numpy()
    bad = []
    for n in np.unique(L):
        sel = np.nonzero(L == n)[0]
        rows = offs[sel][:, None] + np.arange(n)[None, :]
        ref = oracle.c2c(xs[rows].astype(np.complex128), -1, method="fft")
        worst, ok = _per_member_ok(ys[rows], ref, oracle.fp32_tol(int(n)))
        if not ok:
            bad.append((int(n), worst))
    assert not bad, (bad[:10], group.describe())
