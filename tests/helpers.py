"""Shared helpers for the parity tests (device buffers via torch, oracle checks)."""
import numpy as np

import oracle
import plfft


def span(howmany, dist, n, stride):
    return (howmany - 1) * (dist if howmany > 1 else 0) + (n - 1) * stride + 1


def seeded_complex(count, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    re = rng.uniform(-1, 1, count)
    im = rng.uniform(-1, 1, count)
    return ((re + 1j * im) * scale).astype(np.complex64)


def seeded_real(count, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, count).astype(np.float32)


def to_dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def from_dev(t):
    return t.cpu().numpy()


def gather(buf, howmany, dist, n, stride):
    """Logical (howmany, n) view of a strided flat buffer."""
    idx = np.arange(howmany)[:, None] * dist + np.arange(n)[None, :] * stride
    return buf[idx]


def c2c_case(n, howmany=1, istride=1, idist=None, ostride=1, odist=None, direction=-1, seed=0,
             alias=False, scale=1.0, host=False, method="auto", rigor=None):
    """Run a C2C plan on seeded data; return (got, ref) logical arrays."""
    import torch

    idist = n if idist is None else idist
    odist = n if odist is None else odist
    nin = span(howmany, idist, n, istride)
    nout = span(howmany, odist, n, ostride)
    x = seeded_complex(nin, seed)
    xin = x.copy()
    plan = plfft.make_plan("c2c", n, howmany, istride, idist, ostride, odist, direction=direction,
                           alias=plfft.IoAlias.MAY_ALIAS if alias else plfft.IoAlias.NO_ALIAS, scale=scale,
                           rigor=plfft.Rigor.ESTIMATE if rigor is None else rigor)
    if host:
        out = np.zeros(nout, np.complex64) if not alias else x
        plan.execute(x.ctypes.data, out.ctypes.data)
        got_buf = out
    else:
        d_in = to_dev(x)
        d_out = d_in if alias else torch.zeros(nout, dtype=torch.complex64, device="cuda")
        plan.execute(d_in.data_ptr(), d_out.data_ptr())
        got_buf = from_dev(d_out)
    xl = gather(xin, howmany, idist, n, istride)
    ref = oracle.c2c(xl.astype(np.complex128), direction, method=method) * scale
    got = gather(got_buf, howmany, odist, n, ostride)
    return got, ref, plan


def _is_prime(n):
    if n < 2:
        return False
    d = 2
    while d * d <= n:
        if n % d == 0:
            return False
        d += 1
    return True


def _smooth7(n):
    for p in (2, 3, 5, 7):
        while n % p == 0:
            n //= p
    return n == 1


def grouped_lengths(count, seed=0, min_len=16, max_len=65536):
    """Seeded lengths for the grouped workload: log-uniform in [min_len, max_len],
    60% powers of two, 20% 2^a 3^b 5^c 7^d, 10% primes with smooth p-1 (Rader),
    10% lengths with a large prime factor (Bluestein)."""
    rng = np.random.default_rng(seed)
    out = []
    lo, hi = np.log(min_len), np.log(max_len)
    while len(out) < count:
        cls = rng.choice(4, p=[0.6, 0.2, 0.1, 0.1])
        target = int(np.exp(rng.uniform(lo, hi)))
        if cls == 0:
            n = 1 << int(round(np.log2(max(target, 1))))
        elif cls == 1:
            n = target
            while not _smooth7(n):
                n += 1
        elif cls == 2:
            n = target | 1
            while not (_is_prime(n) and _smooth7_13(n - 1)):
                n += 2
        else:
            n = target
            while _smooth7_13(n) or _is_prime(n):
                n += 1
        if min_len <= n <= max_len:
            out.append(int(n))
    return out


def _smooth7_13(n):
    for p in (2, 3, 5, 7, 11, 13):
        while n % p == 0:
            n //= p
    return n == 1
