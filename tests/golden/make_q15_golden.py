"""Generate tests/golden/q15_reference.npz: outputs of the reference's own
Q0.15 NEON kernels, executed by the interpreter in neon_q15.py.

Run once, in a container that holds the reference sources:
    python tests/golden/make_q15_golden.py /root/reference
Nothing at test time reads the reference; the tests read the .npz only.

Composition (the reference's ESTIMATE plan for Q0.15 C2C of power-of-two
N <= 256, src/providers/aot/kernels.hpp:2394-2440 for the kernel table):
  N <= 16 : one radix-N codelet over the batch (plfft_N_q15_jjjn{f,b}_gs).
  N = 16 m: per member, stage 1 = m-point codelets over the 16 columns
            (plfft_m_q15_jjjn{f,b}_uu, stride 16); stage 2 = 16-point
            codelets on the m rows, row 0 untwiddled (..._uun), rows 1..m-1
            twiddled (plfft_ab_16_q15_jjjt{f,b}_dit_gu), output stride m.
Stage-2 twiddles follow src/generate_twiddles.hpp:72-132 with n1 = m,
n2 = 16, premultiplied pairs: for j = 1..m-1, i = 1..15,
(cvt(cos t), cvt(sin t)), (cvt(-sin t), cvt(cos t)), t = dir*2*pi*i*j/N,
cvt(x) = sat16(trunc(float(x) * 2^15)) (src/plfft_convert.hpp:48-54).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import neon_q15  # noqa: E402

SOURCES = ["plfft_q15_jjjn_uu.S", "plfft_q15_jjjn_uun.S", "plfft_q15_jjjn_gs.S",
           "plfft_ab_q15_jjjt_dit_gu.S"]


def cvt(x):
    v = np.float32(x) * np.float32(32768.0)
    return int(np.clip(np.trunc(np.float64(v)), -32768, 32767))


def twiddles(m, dirn):
    n = 16 * m
    base = dirn * 2.0 * np.pi / n
    out = []
    for j in range(1, m):
        for i in range(1, 16):
            a, b = np.cos(base * i * j), np.sin(base * i * j)
            out += [cvt(a), cvt(b), cvt(-b), cvt(a)]
    return np.array(out, np.int16)


def run(machine, n, dirn, x):
    """x: int16 [howmany, n, 2] -> int16 [howmany, n, 2]"""
    hm = x.shape[0]
    d = "f" if dirn < 0 else "b"
    ax = machine.alloc(x.nbytes)
    ay = machine.alloc(x.nbytes)
    machine.write(ax, np.ascontiguousarray(x))
    if n <= 16:
        if hm == 1:
            machine.call(f"plfft_{n}_q15_jjjn{d}_uun_neon", [ax, ay, 1, 1, 1, 0, 0])
        else:
            machine.call(f"plfft_{n}_q15_jjjn{d}_gs_neon", [ax, ay, 1, 1, hm, n, n])
    else:
        m = n // 16
        w = twiddles(m, dirn)
        aw = machine.alloc(w.nbytes)
        machine.write(aw, w)
        tmp = machine.alloc(4 * n)
        for b in range(hm):
            xb, yb = ax + 4 * n * b, ay + 4 * n * b
            machine.call(f"plfft_{m}_q15_jjjn{d}_uu_neon", [xb, tmp, 16, 16, 16, 1, 1])
            machine.call(f"plfft_16_q15_jjjn{d}_uun_neon", [tmp, yb, 1, m, 1, 0, 0])
            machine.call(f"plfft_ab_16_q15_jjjt{d}_dit_gu_neon",
                         [tmp + 64, yb + 4, 1, m, aw, m - 1, 16, 1])
    return machine.read(ay, np.int16, x.size).reshape(x.shape)


def inputs(n, seed):
    rng = np.random.default_rng(seed)
    hm = 8
    x = rng.integers(-32768, 32768, (hm, n, 2)).astype(np.int16)
    x[1] = 32767                      # saturating constant
    x[2] = -32768
    x[3] = 0
    x[3, 0] = (32767, -32768)         # impulse
    x[4] = (rng.standard_normal((n, 2)) * 3000).astype(np.int16)  # small signal
    x[6] = np.where(rng.random((n, 2)) < 0.5, -32768, 32767)       # full-scale extremes
    x[7, :, 0] = np.where(np.arange(n) % 2 == 0, 32767, -32768)    # alternating, all energy at n/2
    x[7, :, 1] = -32768
    return x


def main():
    ref = sys.argv[1]
    kdir = os.path.join(ref, "src", "providers", "aot", "asm", "neon")
    kern = neon_q15.Kernels([os.path.join(kdir, s) for s in SOURCES])
    out = {}
    for n in [2, 4, 8, 16, 32, 64, 128, 256]:
        for dirn in (-1, 1):
            machine = neon_q15.Machine(kern)
            x = inputs(n, 1000 + n)
            out[f"x_{n}"] = x
            out[f"y_{n}_{'f' if dirn < 0 else 'b'}"] = run(machine, n, dirn, x)
            y1 = run(machine, n, dirn, x[:1])  # single-member code path
            out[f"y1_{n}_{'f' if dirn < 0 else 'b'}"] = y1
    np.savez_compressed(os.path.join(HERE, "q15_reference.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
