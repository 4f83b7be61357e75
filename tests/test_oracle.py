"""Pins the FP64 oracle (CPU, no GPU needed).

The reference ships no golden vectors; its tests derive expected values
analytically.  The oracle is pinned here against those same families
(delta<->constant test/delta_constant_test.hpp:38-63, pure tone
test/pure_tone_test.hpp:36-62, sum checks test/simple_test.hpp:16-95, round
trips test/advanced_test_utils.hpp:49-124, R2R round-trip scales
test/r2r_test.hpp:60-80) and against the committed fixtures in
tests/golden/ (FFTW-convention values produced by make_golden.py with
numpy/scipy, independent implementations of the same definitions).
"""
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_delta_to_constant():
    for n in [1, 2, 3, 8, 23, 64, 1058]:
        x = np.zeros(n, complex)
        x[0] = 1
        y = oracle.c2c(x[None], -1)[0]
        assert np.allclose(y, 1.0, atol=1e-12)
        # constant -> delta
        y = oracle.c2c(np.ones((1, n), complex), -1)[0]
        ref = np.zeros(n, complex)
        ref[0] = n
        assert np.allclose(y, ref, atol=1e-9)


def test_pure_tone():
    for n in [4, 16, 23, 100, 1024]:
        for k0 in [0, 1, n // 3]:
            x = np.zeros(n, complex)
            x[k0] = 2.5
            for direction in (-1, 1):
                y = oracle.c2c(x[None], direction)[0]
                k = np.arange(n)
                ref = 2.5 * np.exp(direction * 2j * np.pi * k * k0 / n)
                assert np.abs(y - ref).max() < 1e-11


def test_sum_check_and_round_trip():
    rng = np.random.default_rng(0)
    for n in [2, 5, 16, 97, 360, 1031]:
        x = rng.uniform(-1, 1, (3, n)) + 1j * rng.uniform(-1, 1, (3, n))
        y = oracle.c2c(x, -1)
        assert np.allclose(y[:, 0], x.sum(axis=1), atol=1e-10)
        z = oracle.c2c(y, 1) / n
        assert np.abs(z - x).max() < 1e-11


@pytest.mark.parametrize("n", [1, 7, 64, 97, 360, 1000, 1031, 4096])
def test_fft_matches_direct(n):
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, (2, n)) + 1j * rng.uniform(-1, 1, (2, n))
    a = oracle.c2c(x, -1, method="dft")
    b = oracle.c2c(x, -1, method="fft")
    assert oracle.rel_l2(b, a) < 1e-13


def test_r2c_c2r():
    rng = np.random.default_rng(2)
    for n in [1, 2, 5, 8, 17, 64, 4096]:
        x = rng.uniform(-1, 1, (2, n))
        y = oracle.r2c(x)
        full = oracle.c2c(x.astype(complex), -1)
        assert np.allclose(y, full[:, : n // 2 + 1], atol=1e-10)
        z = oracle.c2r(y, n)
        assert np.abs(z - n * x).max() < 1e-9


R2R_SCALE = {  # docs/plfft.md round-trip factors
    "DCT_1": lambda n: 2 * (n - 1), "DCT_2": lambda n: 2 * n, "DCT_3": lambda n: 2 * n,
    "DCT_4": lambda n: 2 * n, "DST_1": lambda n: 2 * (n + 1), "DST_2": lambda n: 2 * n,
    "DST_3": lambda n: 2 * n, "DST_4": lambda n: 2 * n, "DHT": lambda n: n,
    "R2HC": lambda n: n, "HC2R": lambda n: n,
}
R2R_INVERSE = {"DCT_1": "DCT_1", "DCT_2": "DCT_3", "DCT_3": "DCT_2", "DCT_4": "DCT_4", "DST_1": "DST_1",
               "DST_2": "DST_3", "DST_3": "DST_2", "DST_4": "DST_4", "DHT": "DHT", "R2HC": "HC2R",
               "HC2R": "R2HC"}


@pytest.mark.parametrize("kind", list(R2R_SCALE))
def test_r2r_round_trip(kind):
    rng = np.random.default_rng(3)
    for n in [2, 3, 8, 17, 128]:
        x = rng.uniform(-1, 1, (2, n))
        y = oracle.r2r(oracle.r2r(x, kind), R2R_INVERSE[kind])
        assert np.abs(y - R2R_SCALE[kind](n) * x).max() < 1e-9


def test_r2r_first_element_sums():
    """reference test/r2r_test.hpp: DCT-II y0 = 2*sum, DHT and R2HC y0 = sum."""
    x = np.random.default_rng(4).uniform(-1, 1, (1, 33))
    assert np.isclose(oracle.r2r(x, "DCT_2")[0, 0], 2 * x.sum())
    assert np.isclose(oracle.r2r(x, "DHT")[0, 0], x.sum())
    assert np.isclose(oracle.r2r(x, "R2HC")[0, 0], x.sum())


def test_golden_fixtures():
    path = os.path.join(GOLDEN, "fftw_conventions.npz")
    g = np.load(path)
    for key in g.files:
        if not key.endswith("_in"):
            continue
        name = key[:-3]
        x = g[key]
        ref = g[name + "_out"]
        kind = name.split("_n")[0]
        if kind == "c2c_fwd":
            got = oracle.c2c(x, -1)
        elif kind == "c2c_bwd":
            got = oracle.c2c(x, 1)
        elif kind == "r2c":
            got = oracle.r2c(x)
        else:
            got = oracle.r2r(x, kind)
        assert oracle.rel_l2(got, ref) < 1e-12, name
