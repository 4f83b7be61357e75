"""Generates tests/golden/fftw_conventions.npz.

The reference (arm/perf-libs-fft) cannot be built on this x86_64 host (it
needs <arm_neon.h>, __fp16 and AArch64 .S kernels) and ships no golden
vectors, so the fixtures here come from independent implementations of the
same published definitions: numpy.fft for the DFT sign/bin conventions
(docs/plfft.md:100-116) and scipy.fft dct/dst (type 1-4, norm=None, which are
FFTW's REDFT/RODFT definitions, include/plfft.h:98-134).  DHT / R2HC are
built from numpy.fft.fft by their FFTW definitions.

Run: python tests/golden/make_golden.py   (seeded; output is deterministic)
"""
import os

import numpy as np
import scipy.fft as sf

rng = np.random.default_rng(20261203)
out = {}


def add(name, x, y):
    out[name + "_in"] = x
    out[name + "_out"] = y


for n in [1, 2, 3, 8, 23, 100, 1024]:
    x = rng.uniform(-1, 1, (2, n)) + 1j * rng.uniform(-1, 1, (2, n))
    add(f"c2c_fwd_n{n}", x, np.fft.fft(x, axis=-1))
    add(f"c2c_bwd_n{n}", x, np.fft.ifft(x, axis=-1) * n)
for n in [1, 2, 5, 16, 97]:
    x = rng.uniform(-1, 1, (2, n))
    add(f"r2c_n{n}", x, np.fft.rfft(x, axis=-1))

for n in [2, 3, 8, 17, 64]:
    x = rng.uniform(-1, 1, (2, n))
    for t in (1, 2, 3, 4):
        add(f"DCT_{t}_n{n}", x, sf.dct(x, type=t, axis=-1))
        add(f"DST_{t}_n{n}", x, sf.dst(x, type=t, axis=-1))
    F = np.fft.fft(x, axis=-1)
    add(f"DHT_n{n}", x, F.real - F.imag)
    hc = np.empty_like(x)
    for k in range(n // 2 + 1):
        hc[:, k] = F[:, k].real
    for k in range(1, (n + 1) // 2):
        hc[:, n - k] = F[:, k].imag
    add(f"R2HC_n{n}", x, hc)

path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fftw_conventions.npz")
np.savez_compressed(path, **out)
print("wrote", path, len(out) // 2, "cases")
