"""Q0.7 oracle pins (CPU, no GPU needed).

tests/golden/q7_reference.npz holds outputs of the reference's own NEON
Q0.7 kernels (src/providers/aot/asm/neon/plfft_q7_pppn_*.S,
plfft_ab_q7_pppt_dit_*.S, plfft_ac_q7_pppt_dit_uu.S) executed from their
source text by tests/golden/neon_a64.py and composed as the reference's
ESTIMATE plans (tests/golden/ref_plan.py).  The C restatement
oracle/fixed.c must reproduce them bit for bit for every power-of-two N up
to 4096, both directions, including saturating inputs.  It must also meet
the reference's own fixed-point accuracy bound: 6 * log2(n) LSB against the
exact DFT scaled by 1/n (test/test_utils.hpp:131-152).
"""
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "q7_reference.npz")
SIZES = [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("d", ["f", "b"])
def test_q7_oracle_matches_reference_kernels(golden, n, d):
    x = golden[f"x_{n}"]
    assert x.dtype == np.int8
    got = oracle.q7_c2c(x, -1 if d == "f" else 1)
    assert np.array_equal(got, golden[f"y_{n}_{d}"]), str(golden[f"plan_{n}_{d}"])
    got1 = oracle.q7_c2c(x[:1], -1 if d == "f" else 1)
    assert np.array_equal(got1, golden[f"y1_{n}_{d}"])


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("direction", [-1, 1])
def test_q7_oracle_within_reference_tolerance(n, direction):
    rng = np.random.default_rng(n)
    # no saturation: the reference's tolerance assumes none occurs
    x = rng.integers(-2 ** 6, 2 ** 6, (64, n, 2)).astype(np.int8)
    y = oracle.q7_c2c(x, direction)
    xc = x[..., 0].astype(float) + 1j * x[..., 1].astype(float)
    ex = (np.fft.fft(xc, axis=-1) if direction < 0 else np.fft.ifft(xc, axis=-1) * n) / n
    err = np.abs(y[..., 0] + 1j * y[..., 1] - ex)
    assert err.max() <= 6 * np.log2(n), (n, err.max())


def test_q7_oracle_delta_to_constant():
    """delta -> constant x/n (test/delta_to_constant_q0_7.cpp via
    test/delta_constant_test.hpp:38-63)."""
    n = 64
    x = np.zeros((1, n, 2), np.int8)
    x[0, 0] = (127, 0)
    y = oracle.q7_c2c(x, -1)
    assert np.abs(y[0, :, 0] - 127 / n).max() <= 6 * 6 and np.abs(y[0, :, 1]).max() <= 6 * 6
