"""FP64 CPU oracle -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package, and only to check the CUDA path's results.  It wraps
``oracle/lib/liboracle.so`` (built from ``oracle/oracle.c`` by ``make -C
oracle``), which restates the reference's transform definitions
(arm/perf-libs-fft docs/plfft.md:100-212, include/plfft.h:98-134) as FP64
direct sums and an FP64 mixed-radix FFT.

Parity pins: the reference ships no golden vector files (its tests generate
references analytically: test/delta_constant_test.hpp:38-63,
test/pure_tone_test.hpp:36-62, test/simple_test.hpp:16-95,
test/advanced_test_utils.hpp:49-124).  ``tests/test_oracle.py`` pins this
oracle against those same analytic families and against
``tests/golden/*.npz`` fixtures (see ``tests/golden/make_golden.py``).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "lib", "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle)")
        L = ctypes.CDLL(path)
        i64 = ctypes.c_int64
        dp = ctypes.c_void_p
        for name in ("oracle_dft_c2c", "oracle_fft_c2c"):
            f = getattr(L, name)
            f.argtypes = [dp, dp, i64, i64, i64, i64, i64, i64, ctypes.c_int, ctypes.c_int]
            f.restype = None
        for name in ("oracle_r2c", "oracle_c2r", "oracle_r2r"):
            f = getattr(L, name)
            f.argtypes = [dp, dp, i64, i64, i64, i64, i64, i64, ctypes.c_int, ctypes.c_int]
            f.restype = None
        L.oracle_max_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def max_threads():
    return lib().oracle_max_threads()


def c2c(x, direction=-1, method="auto", threads=0):
    """Batched C2C along the last axis; x complex (..., n). Returns complex128."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    n = x.shape[-1]
    hm = int(np.prod(x.shape[:-1])) if x.ndim > 1 else 1
    out = np.empty_like(x)
    use_fft = method == "fft" or (method == "auto" and n > 4096)
    f = lib().oracle_fft_c2c if use_fft else lib().oracle_dft_c2c
    f(_ptr(x), _ptr(out), n, hm, 1, n, 1, n, int(direction), int(threads))
    return out


def r2c(x, method="auto", threads=0):
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[-1]
    hm = int(np.prod(x.shape[:-1])) if x.ndim > 1 else 1
    h = n // 2 + 1
    out = np.empty(x.shape[:-1] + (h,), dtype=np.complex128)
    use_fft = method == "fft" or (method == "auto" and n > 4096)
    lib().oracle_r2c(_ptr(x), _ptr(out), n, hm, 1, n, 1, h, int(use_fft), int(threads))
    return out


def c2r(x, n, method="auto", threads=0):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    h = n // 2 + 1
    assert x.shape[-1] == h
    hm = int(np.prod(x.shape[:-1])) if x.ndim > 1 else 1
    out = np.empty(x.shape[:-1] + (n,), dtype=np.float64)
    use_fft = method == "fft" or (method == "auto" and n > 4096)
    lib().oracle_c2r(_ptr(x), _ptr(out), n, hm, 1, h, 1, n, int(use_fft), int(threads))
    return out


R2R_KINDS = {
    "DCT_1": 0, "DCT_2": 1, "DCT_3": 2, "DCT_4": 3,
    "DST_1": 4, "DST_2": 5, "DST_3": 6, "DST_4": 7,
    "DHT": 8, "R2HC": 9, "HC2R": 10,
}


def r2r(x, kind, threads=0):
    """kind: plfft_r2r_kind_t value or name (FFTW conventions)."""
    k = R2R_KINDS[kind] if isinstance(kind, str) else int(kind)
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[-1]
    hm = int(np.prod(x.shape[:-1])) if x.ndim > 1 else 1
    out = np.empty_like(x)
    lib().oracle_r2r(_ptr(x), _ptr(out), n, hm, 1, n, 1, n, k, int(threads))
    return out


def c2c_strided(buf_in, buf_out, n, howmany, istride, idist, ostride, odist, direction, method="dft"):
    """C2C with explicit element strides on flat complex128 buffers (in place on buf_out)."""
    assert buf_in.dtype == np.complex128 and buf_out.dtype == np.complex128
    f = lib().oracle_fft_c2c if method == "fft" else lib().oracle_dft_c2c
    f(_ptr(buf_in), _ptr(buf_out), n, howmany, istride, idist, ostride, odist, int(direction), 0)
    return buf_out


def rel_l2(got, ref):
    got = np.asarray(got, dtype=np.complex128 if np.iscomplexobj(got) else np.float64)
    ref = np.asarray(ref)
    num = np.linalg.norm((got - ref).ravel())
    den = np.linalg.norm(ref.ravel())
    return float(num / den) if den > 0 else float(num)


def fp32_tol(n):
    """FP32 gate: rel-L2 <= 4 * log2(N) * 2^-24."""
    return 4.0 * max(1.0, np.log2(max(n, 2))) * 2.0 ** -24


# ---------------------------------------------------------------------------
# fixed point (oracle/fixed.c): bit-exact restatement of the Q0.15 and Q0.7
# paths, n a power of two <= 4096
# ---------------------------------------------------------------------------
_LIBQ = None
FIXED_MAX_N = 4096


def _libq():
    global _LIBQ
    if _LIBQ is None:
        path = os.path.join(_HERE, "lib", "liboracle_fixed.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle)")
        L = ctypes.CDLL(path)
        i64 = ctypes.c_int64
        dp = ctypes.c_void_p
        for name in ("oracle_q15_c2c", "oracle_q7_c2c"):
            getattr(L, name).argtypes = [dp, dp, i64, i64, i64, i64, ctypes.c_int]
            getattr(L, name).restype = ctypes.c_int
        for name in ("oracle_q15_r2c", "oracle_q7_r2c", "oracle_q15_c2r", "oracle_q7_c2r"):
            getattr(L, name).argtypes = [dp, dp, i64, i64, i64, i64, i64, i64]
            getattr(L, name).restype = ctypes.c_int
        L.oracle_q15_twiddles.argtypes = [i64, ctypes.c_int, dp]
        L.oracle_q15_twiddles.restype = None
        _LIBQ = L
    return _LIBQ


def _fixed_c2c(x, direction, dtype, fn):
    x = np.ascontiguousarray(x, dtype=dtype)
    hm, n = x.shape[0], x.shape[1]
    y = np.empty_like(x)
    rc = fn(_ptr(x), _ptr(y), n, hm, n, n, int(direction))
    if rc != 0:
        raise ValueError(f"fixed-point oracle: unsupported length {n}")
    return y


def q15_c2c(x, direction=-1):
    """x: int16 [howmany, n, 2] (re, im) -> int16 [howmany, n, 2], scaled by 1/n."""
    return _fixed_c2c(x, direction, np.int16, _libq().oracle_q15_c2c)


def q7_c2c(x, direction=-1):
    """x: int8 [howmany, n, 2] (re, im) -> int8 [howmany, n, 2], scaled by 1/n."""
    return _fixed_c2c(x, direction, np.int8, _libq().oracle_q7_c2c)


def _fixed_r2c(x, dtype, fn, odist_unit):
    x = np.ascontiguousarray(x, dtype=dtype)
    hm, n = x.shape[0], x.shape[1]
    h = n // 2 + 1
    if odist_unit and hm > 1:
        # members adjacent in the output (ostride hm, odist 1): the reference's
        # uu / gu kernel variants for n <= 16
        y = np.empty((h, hm, 2), dtype)
        rc = fn(_ptr(x), _ptr(y), n, hm, 1, n, hm, 1)
        y = np.ascontiguousarray(y.transpose(1, 0, 2))
    else:
        y = np.empty((hm, h, 2), dtype)
        rc = fn(_ptr(x), _ptr(y), n, hm, 1, n, 1, h)
    if rc != 0:
        raise ValueError(f"fixed-point oracle: unsupported length {n}")
    return y


def fixed_r2c_strided(bits, buf, n, howmany, istride, idist, ostride, odist, out_elems):
    """R2C of the members of the flat real buffer buf (int16 for bits 16, int8
    for 8) in the given layout; returns a flat complex buffer [out_elems, 2]
    (zero where no output lands)."""
    dtype = np.int16 if bits == 16 else np.int8
    buf = np.ascontiguousarray(buf, dtype=dtype)
    y = np.zeros((out_elems, 2), dtype)
    fn = _libq().oracle_q15_r2c if bits == 16 else _libq().oracle_q7_r2c
    if fn(_ptr(buf), _ptr(y), n, howmany, istride, idist, ostride, odist) != 0:
        raise ValueError(f"fixed-point oracle: unsupported length {n}")
    return y


def q15_r2c(x, odist_unit=False):
    """x: int16 [howmany, n] reals -> int16 [howmany, n/2+1, 2], scaled by 1/n.
    odist_unit: compute as a batch laid out with output distance 1."""
    return _fixed_r2c(x, np.int16, _libq().oracle_q15_r2c, odist_unit)


def q7_r2c(x, odist_unit=False):
    """x: int8 [howmany, n] reals -> int8 [howmany, n/2+1, 2], scaled by 1/n.
    odist_unit: compute as a batch laid out with output distance 1."""
    return _fixed_r2c(x, np.int8, _libq().oracle_q7_r2c, odist_unit)


def fixed_c2r_strided(bits, buf, n, howmany, istride, idist, ostride, odist, out_elems):
    """C2R of the members of the flat buffer buf of complex lanes ([elements,
    2], int16 for bits 16, int8 for 8) in the given layout; returns the flat
    real output [out_elems] (zero where no output lands)."""
    dtype = np.int16 if bits == 16 else np.int8
    buf = np.ascontiguousarray(buf, dtype=dtype)
    y = np.zeros(out_elems, dtype)
    fn = _libq().oracle_q15_c2r if bits == 16 else _libq().oracle_q7_c2r
    if fn(_ptr(buf), _ptr(y), n, howmany, istride, idist, ostride, odist) != 0:
        raise ValueError(f"fixed-point oracle: unsupported length {n}")
    return y


def q15_c2r(X, n):
    """X: int16 [howmany, n/2+1, 2] bins -> int16 [howmany, n] reals, scaled by 1/n."""
    X = np.ascontiguousarray(X, dtype=np.int16)
    hm = X.shape[0]
    return fixed_c2r_strided(16, X, n, hm, 1, n // 2 + 1, 1, n, hm * n).reshape(hm, n)


def q7_c2r(X, n):
    """X: int8 [howmany, n/2+1, 2] bins -> int8 [howmany, n] reals, scaled by 1/n."""
    X = np.ascontiguousarray(X, dtype=np.int8)
    hm = X.shape[0]
    return fixed_c2r_strided(8, X, n, hm, 1, n // 2 + 1, 1, n, hm * n).reshape(hm, n)


def q15_twiddles(n, direction=-1):
    w = np.empty(max(0, n // 16 - 1) * 15 * 4, np.int16)
    _libq().oracle_q15_twiddles(n, int(direction), _ptr(w))
    return w
