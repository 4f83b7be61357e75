"""Q0.15 oracle pins (CPU, no GPU needed).

tests/golden/q15_reference.npz holds outputs of the reference's own NEON
Q0.15 kernels (src/providers/aot/asm/neon/plfft_*q15*.S), executed from
their source text by tests/golden/neon_a64.py and composed as the
reference's ESTIMATE plan by tests/golden/ref_plan.py
(tests/golden/make_ref_golden.py).  The C
restatement oracle/fixed.c must reproduce them bit for bit.  It must also
meet the reference's own fixed-point accuracy bound: 6 * log2(n) LSB
against the exact DFT scaled by 1/n (test/test_utils.hpp:131-152).
"""
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "q15_reference.npz")
SIZES = [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]


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


# ---------------------------------------------------------------------------
# Interval analysis behind the device kernels' choice to clamp only codelet
# outputs (perf-libs-fft_b200/csrc/q15.cu): with every codelet input
# pre-shifted by log2(r), no intermediate value of the radix 2/4/8/16
# codelets (sums, sqrdmulh constants, 32-bit MACs) and no twiddled row input
# can leave int16; only the outputs y_k can saturate.
# ---------------------------------------------------------------------------
def _saturating_ops(bits=16):
    class I:
        def __init__(s, lo, hi): s.lo, s.hi = lo, hi
        def __add__(s, o): return I(s.lo + o.lo, s.hi + o.hi)
        def __sub__(s, o): return I(s.lo - o.hi, s.hi - o.lo)
        def __repr__(s): return f"[{s.lo},{s.hi}]"
    LO, HI = -(1 << (bits - 1)), (1 << (bits - 1)) - 1
    def sat(x): return I(max(LO, min(HI, x.lo)), max(LO, min(HI, x.hi)))
    need = {}
    def chk(tag, x):
        if x.lo < LO or x.hi > HI: need[tag] = need.get(tag, 0) + 1
        else: need.setdefault(tag, 0)
        return sat(x)
    def add(tag, a, b): return (chk(tag + '.re', a[0] + b[0]), chk(tag + '.im', a[1] + b[1]))
    def sub(tag, a, b): return (chk(tag + '.re', a[0] - b[0]), chk(tag + '.im', a[1] - b[1]))
    def mulk(x, k):  # exact product interval
        c = [x.lo * k, x.hi * k]; return I(min(c), max(c))
    def rdm(x, k): p = mulk(x, k); return I((p.lo + (1 << (bits - 2))) >> (bits - 1), (p.hi + (1 << (bits - 2))) >> (bits - 1))
    def rdmt(tag, x, k): return chk(tag, rdm(x, k))
    def mac(tag, a, ka, b, kb):
        s = mulk(a, ka) + mulk(b, kb)
        assert -(1 << (2 * bits - 1)) <= s.lo and s.hi < (1 << (2 * bits - 1)), tag  # no lane wrap
        return chk(tag, I((s.lo + (1 << (bits - 2))) >> (bits - 1), (s.hi + (1 << (bits - 2))) >> (bits - 1)))
    def mul_pi(t, z): return (rdmt(t + '.pr', z[1], LO), rdmt(t + '.pi', z[0], HI))
    def mul_mi(t, z): return (rdmt(t + '.mr', z[1], HI), rdmt(t + '.mi', z[0], LO))
    C8, C16, S16 = (23170, 30273, 12539) if bits == 16 else (90, 118, 48)
    def w8(t, z): return (mac(t + '.w8r', z[0], C8, rdm(z[1], C8), HI), mac(t + '.w8i', z[1], C8, rdm(z[0], C8), LO))
    def w83(t, z): return (mac(t + '.w83r', z[0], -C8, rdm(z[1], -C8), LO), mac(t + '.w83i', z[1], -C8, rdm(z[0], -C8), HI))
    def mw(t, z, wr, wi): return (mac(t + '.r', z[0], wr, z[1], -wi), mac(t + '.i', z[1], wr, z[0], wi))
    def dft16(a):
        p = [add(f'p{k}', a[k], a[k + 8]) for k in range(8)]; m = [sub(f'm{k}', a[k], a[k + 8]) for k in range(8)]
        s04 = add('s04', p[0], p[4]); s26 = add('s26', p[2], p[6]); s15 = add('s15', p[1], p[5]); s37 = add('s37', p[3], p[7])
        e0 = add('e0', s04, s26); e1 = add('e1', s15, s37); y = {}
        y[0] = add('y0', e0, e1); y[8] = sub('y8', e0, e1)
        A = sub('A', s04, s26); jB = mul_pi('jB', sub('B', s15, s37)); y[4] = sub('y4', A, jB); y[12] = add('y12', A, jB)
        C = sub('C', p[0], p[4]); jD = mul_pi('jD', sub('D', p[2], p[6]))
        kE = w8('kE', sub('E', p[1], p[5])); kF = w83('kF', sub('F', p[3], p[7]))
        g1 = sub('g1', C, jD); g2 = add('g2', C, jD); h = add('h', kE, kF); h2 = mul_mi('h2', sub('h2s', kF, kE))
        y[2] = add('y2', g1, h); y[10] = sub('y10', g1, h); y[6] = sub('y6', g2, h2); y[14] = add('y14', g2, h2)
        j4 = mul_pi('j4', m[4]); q = sub('q', m[0], j4); q2 = add('q2', m[0], j4)
        k2 = w8('k2', m[2]); k6 = w83('k6', m[6]); r = add('r', k2, k6); r2 = mul_mi('r2', sub('r2s', k6, k2))
        j5 = mul_pi('j5', m[5]); j7 = mul_pi('j7', m[7])
        u = sub('u', m[1], j5); u2 = add('u2', m[1], j5); v = sub('v', m[3], j7); v2 = add('v2', m[3], j7)
        l1 = mw('l1', u, C16, -S16); l3 = mw('l3', v, S16, -C16); l3b = mw('l3b', u2, S16, -C16); l9 = mw('l9', v2, -C16, S16)
        qr = add('qr', q, r); qmr = sub('qmr', q, r); ls = add('ls', l1, l3); ld = mul_mi('ld', sub('lds', l3, l1))
        y[1] = add('y1', qr, ls); y[9] = sub('y9', qr, ls); y[5] = sub('y5', qmr, ld); y[13] = add('y13', qmr, ld)
        qa = sub('qa', q2, r2); qb = add('qb', q2, r2); ls2 = add('ls2', l3b, l9); ld2 = mul_mi('ld2', sub('ld2s', l9, l3b))
        y[3] = add('y3', qa, ls2); y[11] = sub('y11', qa, ls2); y[7] = sub('y7', qb, ld2); y[15] = add('y15', qb, ld2)
    def dft8(a):
        p = [add(f'8p{k}', a[k], a[k + 4]) for k in range(4)]; m = [sub(f'8m{k}', a[k], a[k + 4]) for k in range(4)]
        e0 = add('8e0', p[0], p[2]); e1 = add('8e1', p[1], p[3]); add('8y0', e0, e1); sub('8y4', e0, e1)
        d = sub('8d', p[0], p[2]); jd = mul_pi('8jd', sub('8ds', p[1], p[3])); sub('8y2', d, jd); add('8y6', d, jd)
        z = add('8z', m[1], m[3]); w = sub('8w', m[1], m[3]); rd = (rdmt('8rdr', w[0], C8), rdmt('8rdi', w[1], C8))
        x = (mac('8xr', m[2][1], LO, z[1], -C8), mac('8xi', m[2][0], HI, z[0], C8))
        x2 = (mac('8x2r', m[2][1], LO, z[1], C8), mac('8x2i', m[2][0], HI, z[0], -C8))
        u = add('8u', m[0], rd); v = sub('8v', m[0], rd)
        sub('8y1', u, x); add('8y7', u, x); add('8y3', v, x2); sub('8y5', v, x2)
    def dft4(a):
        s02 = add('4s02', a[0], a[2]); s13 = add('4s13', a[1], a[3]); d02 = sub('4d02', a[0], a[2]); j13 = mul_pi('4j13', sub('4d13', a[1], a[3]))
        add('4y0', s02, s13); sub('4y2', s02, s13); sub('4y1', d02, j13); add('4y3', d02, j13)
    def dft2(a): add('2y0', a[0], a[1]); sub('2y1', a[0], a[1])
    def pre(s):  # rounding shift of any lane value
        return I((LO + (1 << (s - 1))) >> s, (HI + (1 << (s - 1))) >> s)
    for r, f in ((2, dft2), (4, dft4), (8, dft8), (16, dft16)):
        s = r.bit_length() - 1
        a = [(pre(s), pre(s))] * r
        f(a)
    # twiddled row inputs: mac of pre-shifted values with arbitrary int16 twiddles
    t = pre(4)
    mac('tw.re', t, HI, t, LO); mac('tw.re2', t, LO, t, LO)
    return need


def test_q15_codelet_intermediates_never_saturate():
    need = _saturating_ops()
    can = sorted(k for k, v in need.items() if v)
    assert len(need) > 200
    # every op that can saturate is a codelet output (named y*, 2y*, 4y*, 8y*)
    assert can and all(k.lstrip("248").startswith("y") for k in can), can


def test_q7_codelet_intermediates_never_saturate():
    """The same interval analysis for Q0.7 lanes (8-bit values, 16-bit MAC
    lanes that must not wrap): only codelet outputs can saturate."""
    need = _saturating_ops(8)
    can = sorted(k for k, v in need.items() if v)
    assert len(need) > 200
    assert can and all(k.lstrip("248").startswith("y") for k in can), can
