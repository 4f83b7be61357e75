"""Fixed-point C2R (Q0.15 and Q0.7): the CPU restatement (oracle/fixed.c,
fixed_c2r) against the reference's own kernels' outputs
(tests/golden/q15_c2r_reference.npz, q7_c2r_reference.npz: the reference's
ESTIMATE C2R plans executed from their NEON source by
tests/golden/neon_a64.py), bit for bit; a constant-spectrum known answer
(the reference's constant_to_delta style, scaled by 1/n); and agreement with
a float inverse FFT within the reference's fixed-point tolerance of
6 log2(n) LSB (test/test_utils.hpp:131-152).
"""
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
SIZES = [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]


def _fn(dtype):
    return oracle.q15_c2r if dtype == "q15" else oracle.q7_c2r


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", SIZES)
def test_fixed_c2r_oracle_matches_reference_kernels(dtype, n):
    g = np.load(os.path.join(HERE, "golden", f"{dtype}_c2r_reference.npz"))
    y = _fn(dtype)(g[f"x_{n}"], n)
    assert np.array_equal(y, g[f"y_{n}"]), str(g[f"plan_{n}"])
    if n <= 256:  # the batched plans of members laid out adjacent
        assert np.array_equal(y, g[f"yu_{n}"]), str(g[f"plan_u_{n}"])


@pytest.mark.parametrize("dtype,bits", [("q15", 16), ("q7", 8)])
@pytest.mark.parametrize("n", [8, 64, 1024])
def test_fixed_c2r_constant_spectrum(dtype, bits, n):
    """X_0 = A, all other bins 0: x_t = A / n for every t (within the
    pre-shift rounding)."""
    it = np.int16 if bits == 16 else np.int8
    a = (1 << (bits - 1)) - 1
    X = np.zeros((1, n // 2 + 1, 2), it)
    X[0, 0, 0] = a
    x = _fn(dtype)(X, n)[0].astype(np.int64)
    assert np.all(np.abs(x - a / n) <= 1), x


@pytest.mark.parametrize("dtype,bits", [("q15", 16), ("q7", 8)])
@pytest.mark.parametrize("n", [4, 16, 128, 2048])
def test_fixed_c2r_within_float_tolerance(dtype, bits, n):
    """Against numpy's irfft (1/n scaled, imaginary parts of bins 0 and n/2
    ignored) of the same bins, within 6 log2(n) LSB."""
    it = np.int16 if bits == 16 else np.int8
    q = 1 << (bits - 1)
    rng = np.random.default_rng(n + bits)
    X = rng.integers(-q // 2, q // 2, (20, n // 2 + 1, 2)).astype(it)
    x = _fn(dtype)(X, n).astype(np.float64)
    ref = np.fft.irfft(X[..., 0] + 1j * X[..., 1], n, axis=-1)
    assert np.max(np.abs(x - ref)) <= 6 * np.log2(n), np.max(np.abs(x - ref))


@pytest.mark.parametrize("bits", [16, 8])
@pytest.mark.parametrize("n", [8, 256, 512])
def test_fixed_c2r_strided_entry(bits, n):
    """The strided entry point in a gapped layout agrees member by member
    with the contiguous one."""
    it = np.int16 if bits == 16 else np.int8
    lim = 1 << (bits - 1)
    hm, h = 7, n // 2 + 1
    rng = np.random.default_rng(n + bits)
    X = rng.integers(-lim, lim, (hm, h, 2)).astype(it)
    ref = (oracle.q15_c2r if bits == 16 else oracle.q7_c2r)(X, n)
    idist, odist = 2 * h + 3, 3 * n + 1
    buf = np.zeros(((hm - 1) * idist + 2 * (h - 1) + 1, 2), it)
    for b in range(hm):
        buf[b * idist:b * idist + 2 * h:2] = X[b]
    out = oracle.fixed_c2r_strided(bits, buf, n, hm, 2, idist, 3, odist, (hm - 1) * odist + 3 * (n - 1) + 1)
    got = np.stack([out[b * odist:b * odist + 3 * n:3] for b in range(hm)])
    assert np.array_equal(got, ref)
