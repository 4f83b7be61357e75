"""Q0.15 oracle pins (CPU, no GPU needed).

tests/golden/q15_reference.npz holds outputs of the reference's own NEON
Q0.15 kernels (src/providers/aot/asm/neon/plfft_*q15*.S), executed from
their source text by tests/golden/neon_q15.py and composed as the
reference's ESTIMATE plan by tests/golden/make_q15_golden.py.  The C
restatement oracle/q15.c must reproduce them bit for bit.  It must also
meet the reference's own fixed-point accuracy bound: 6 * log2(n) LSB
against the exact DFT scaled by 1/n (test/test_utils.hpp:131-152).
"""
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "q15_reference.npz")
SIZES = [2, 4, 8, 16, 32, 64, 128, 256]


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("d", ["f", "b"])
def test_q15_oracle_matches_reference_kernels(golden, n, d):
    x = golden[f"x_{n}"]
    got = oracle.q15_c2c(x, -1 if d == "f" else 1)
    assert np.array_equal(got, golden[f"y_{n}_{d}"])
    # single-member fixture (the reference's howmany == 1 code path)
    got1 = oracle.q15_c2c(x[:1], -1 if d == "f" else 1)
    assert np.array_equal(got1, golden[f"y1_{n}_{d}"])


def _exact(x, direction):
    xc = x[..., 0].astype(float) + 1j * x[..., 1].astype(float)
    y = np.fft.fft(xc, axis=-1) if direction < 0 else np.fft.ifft(xc, axis=-1) * x.shape[1]
    return y / x.shape[1]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("direction", [-1, 1])
def test_q15_oracle_within_reference_tolerance(n, direction):
    rng = np.random.default_rng(n)
    # no saturation: the reference's tolerance assumes none occurs
    x = rng.integers(-2 ** 14, 2 ** 14, (64, n, 2)).astype(np.int16)
    y = oracle.q15_c2c(x, direction)
    err = np.abs(y[..., 0] + 1j * y[..., 1] - _exact(x, direction))
    tol = 6 * np.log2(n)
    assert err.max() <= tol, (n, err.max(), tol)


def test_q15_oracle_known_pairs():
    """Delta -> constant x/n and constant -> delta (test/delta_constant_test.hpp:38-63)."""
    n = 256
    x = np.zeros((2, n, 2), np.int16)
    x[0, 0] = (32767, 0)
    x[1, :] = (16384, -16384)
    y = oracle.q15_c2c(x, -1)
    # 32767 / 256 = 127.996: every bin within the tolerance of 127.996
    assert np.abs(y[0, :, 0] - 32767 / n).max() <= 6 * 8 and np.abs(y[0, :, 1]).max() <= 6 * 8
    assert tuple(y[1, 0]) == (16384, -16384)
    assert np.abs(y[1, 1:]).max() <= 6 * 8


def test_q15_twiddle_table_conversion():
    """cvt(x) = sat16(trunc(float(x) 2^15)): cos 0 -> 32767, sin pi/2 -> 32767, -sin -> -32768."""
    w = oracle.q15_twiddles(64, -1).reshape(3, 15, 4)
    # row j = 2, input i = 8: angle -2 pi * 16 / 64 = -pi/2 -> (0, -32768, 32767, 0)
    c, s, ms, c2 = w[1, 7]
    assert c == 0 and s == -32768 and ms == 32767 and c2 == 0
    assert np.all(w[..., 0] == w[..., 3])
