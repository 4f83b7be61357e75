"""Split-BF16 tensor-core precision mode (PLFFT_CUDA_PRECISION_SPLIT_BF16).

Gate: rel-L2 <= 1e-6 against the FP64 oracle, with the max-abs error stated
per N (printed), for the precision configurations N = 2^16 and 2^20 and the
one-pass lengths 256 and 4096.  Inputs: U[-1, 1) plus a +-1e3 impulse at a
seeded bin, the precision workload's distribution.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _case(n, howmany, direction, seed, istride=1, idist=None, ostride=1, odist=None):
    import plfft
    import torch

    rng = np.random.default_rng(seed)
    x = (rng.uniform(-1, 1, (howmany, n)) + 1j * rng.uniform(-1, 1, (howmany, n)))
    x[np.arange(howmany), rng.integers(0, n, howmany)] += 1e3 * rng.choice([-1, 1], howmany)
    x = x.astype(np.complex64)
    idist = n if idist is None else idist
    odist = n if odist is None else odist
    plan = plfft.make_plan("c2c", n, howmany, istride, idist, ostride, odist, direction=direction,
                           precision=plfft.Precision.SPLIT_BF16)
    assert "split-bf16" in plan.describe()
    span_i = (howmany - 1) * idist + (n - 1) * istride + 1
    span_o = (howmany - 1) * odist + (n - 1) * ostride + 1
    buf = np.zeros(span_i, np.complex64)
    idx_i = np.arange(howmany)[:, None] * idist + np.arange(n)[None, :] * istride
    buf[idx_i] = x
    d_in = torch.from_numpy(buf).cuda()
    d_out = torch.zeros(span_o, dtype=torch.complex64, device="cuda")
    plan.execute(d_in.data_ptr(), d_out.data_ptr())
    idx_o = np.arange(howmany)[:, None] * odist + np.arange(n)[None, :] * ostride
    got = d_out.cpu().numpy()[idx_o]
    ref = oracle.c2c(x.astype(np.complex128), direction, method="fft")
    return got, ref


@pytest.mark.parametrize("n,howmany", [(256, 37), (4096, 5), (65536, 3), (1 << 20, 2)])
@pytest.mark.parametrize("direction", [-1, 1])
def test_split_bf16_accuracy(n, howmany, direction):
    got, ref = _case(n, howmany, direction, seed=n + direction)
    err = oracle.rel_l2(got, ref)
    maxabs = float(np.abs(got - ref).max())
    print(f"split-bf16 n={n} dir={direction}: rel-L2 {err:.3e}, max-abs {maxabs:.3e} "
          f"(max |X| {np.abs(ref).max():.3e})")
    assert err <= 1e-6, (n, err)


def test_split_bf16_strided():
    got, ref = _case(4096, 3, -1, seed=2, istride=3, idist=1, ostride=4, odist=1)
    assert oracle.rel_l2(got, ref) <= 1e-6


def test_split_bf16_unsupported_lengths_fail():
    import plfft

    for n in (1000, 512, 1 << 18):
        with pytest.raises(plfft.PlfftError) as e:
            plfft.make_plan("c2c", n, 2, precision=plfft.Precision.SPLIT_BF16)
        assert e.value.status == plfft.Status.PLAN_CREATION_FAILED


@pytest.mark.parametrize("n", [4096, 65536])
def test_split_bf16_in_place_host(n):
    """In place on host buffers: the plan stages through the device."""
    import plfft

    rng = np.random.default_rng(n)
    hm = 2
    x = (rng.uniform(-1, 1, (hm, n)) + 1j * rng.uniform(-1, 1, (hm, n))).astype(np.complex64)
    buf = x.copy()
    plan = plfft.make_plan("c2c", n, hm, direction=-1, precision=plfft.Precision.SPLIT_BF16,
                           alias=plfft.IoAlias.MAY_ALIAS)
    plan.execute(buf.ctypes.data, buf.ctypes.data)
    assert oracle.rel_l2(buf, oracle.c2c(x.astype(np.complex128), -1, method="fft")) <= 1e-6
