"""Fixed-point R2C (Q0.15 and Q0.7): the CPU restatement (oracle/fixed.c)
against the reference's own kernels' outputs (tests/golden/q15_r2c_reference
.npz, q7_r2c_reference.npz: the reference's ESTIMATE R2C plans executed from
their NEON source by tests/golden/neon_a64.py), bit for bit; and its known
pairs (reference test/delta_to_constant_q0_15.cpp, pure_tone_fwd_q0_15.cpp
style: an impulse gives a constant spectrum scaled by 1/n).
"""
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
SIZES = [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", SIZES)
def test_fixed_r2c_oracle_matches_reference_kernels(dtype, n):
    g = np.load(os.path.join(HERE, "golden", f"{dtype}_r2c_reference.npz"))
    fn = oracle.q15_r2c if dtype == "q15" else oracle.q7_r2c
    y = fn(g[f"x_{n}"])
    assert np.array_equal(y, g[f"y_{n}"]), str(g[f"plan_{n}"])


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", [2, 4, 8, 16])
def test_fixed_r2c_oracle_odist_unit_variant(dtype, n):
    """Members adjacent in the output (the reference's gu kernel variant)."""
    g = np.load(os.path.join(HERE, "golden", f"{dtype}_r2c_reference.npz"))
    fn = oracle.q15_r2c if dtype == "q15" else oracle.q7_r2c
    y = fn(g[f"xu_{n}"], odist_unit=True)
    assert np.array_equal(y, g[f"yu_{n}"]), str(g[f"plan_u_{n}"])


@pytest.mark.parametrize("dtype", ["q15", "q7"])
@pytest.mark.parametrize("n", [4, 8])
def test_fixed_r2c_variants_differ(dtype, n):
    """The two variant families are distinct on these fixtures (so the test
    above pins the unit-output-distance forms, not the other ones)."""
    g = np.load(os.path.join(HERE, "golden", f"{dtype}_r2c_reference.npz"))
    fn = oracle.q15_r2c if dtype == "q15" else oracle.q7_r2c
    assert not np.array_equal(fn(g[f"xu_{n}"]), g[f"yu_{n}"])


@pytest.mark.parametrize("dtype,bits", [("q15", 16), ("q7", 8)])
@pytest.mark.parametrize("n", [8, 64, 1024])
def test_fixed_r2c_delta_to_constant(dtype, bits, n):
    """x = A at 0: X_k = A / n for every bin (within the pre-shift rounding)."""
    it = np.int16 if bits == 16 else np.int8
    a = (1 << (bits - 1)) - 1
    x = np.zeros((1, n), it)
    x[0, 0] = a
    fn = oracle.q15_r2c if dtype == "q15" else oracle.q7_r2c
    y = fn(x)[0].astype(np.int64)
    assert np.all(y[:, 1] == 0)
    assert np.all(np.abs(y[:, 0] - a / n) <= 1), y[:, 0]


@pytest.mark.parametrize("dtype,bits", [("q15", 16), ("q7", 8)])
@pytest.mark.parametrize("n", [16, 256, 4096])
def test_fixed_r2c_within_float_tolerance(dtype, bits, n):
    """Against the FP64 R2C scaled by 1/n: the fixed-point error stays within
    a few LSB per level."""
    it = np.int16 if bits == 16 else np.int8
    lim = 1 << (bits - 1)
    rng = np.random.default_rng(n + bits)
    x = rng.integers(-lim // 2, lim // 2, (4, n)).astype(it)
    fn = oracle.q15_r2c if dtype == "q15" else oracle.q7_r2c
    y = fn(x).astype(np.float64)
    ref = oracle.r2c(x.astype(np.float64)) / n
    err = np.abs((y[..., 0] + 1j * y[..., 1]) - ref).max()
    assert err <= 2 + np.log2(n), err


@pytest.mark.parametrize("bits", [16, 8])
@pytest.mark.parametrize("n", [4, 8, 64, 512])
def test_fixed_r2c_strided_entry_matches_layout_forms(bits, n):
    """The strided entry point agrees with the two layout forms the
    fixtures pin: gs (contiguous members) and gu (members adjacent in the
    output), and a gapped layout agrees with the contiguous one member by
    member (the variant depends only on howmany and odist)."""
    it = np.int16 if bits == 16 else np.int8
    lim = 1 << (bits - 1)
    hm, h = 9, n // 2 + 1
    rng = np.random.default_rng(n + bits)
    x = rng.integers(-lim, lim, (hm, n)).astype(it)
    fn = oracle.q15_r2c if bits == 16 else oracle.q7_r2c
    gs = oracle.fixed_r2c_strided(bits, x.ravel(), n, hm, 1, n, 1, h, hm * h).reshape(hm, h, 2)
    assert np.array_equal(gs, fn(x))
    gu = oracle.fixed_r2c_strided(bits, x.ravel(), n, hm, 1, n, hm, 1, hm * h).reshape(h, hm, 2)
    assert np.array_equal(gu.transpose(1, 0, 2), fn(x, odist_unit=True))
    buf = np.zeros((hm - 1) * (2 * n + 3) + 2 * (n - 1) + 1, it)
    for b in range(hm):
        buf[b * (2 * n + 3):b * (2 * n + 3) + 2 * n:2] = x[b]
    od = 3 * h + 1
    out = oracle.fixed_r2c_strided(bits, buf, n, hm, 2, 2 * n + 3, 3, od, (hm - 1) * od + 3 * (h - 1) + 1)
    got = np.stack([out[b * od:b * od + 3 * h:3] for b in range(hm)])
    assert np.array_equal(got, fn(x))
