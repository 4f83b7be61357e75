"""Generate reference-output fixtures by executing the reference's own NEON
kernels (interpreter: neon_a64.py) composed as its ESTIMATE plans
(ref_c2c_plan.py).

Run once, in a container that holds the reference sources:
    python tests/golden/make_ref_golden.py <path to the reference checkout> [q15 q7 f32]
Nothing at test time reads the reference; the tests read the .npz files.

Writes:
  q15_reference.npz      Q0.15 C2C, N = 2 .. 4096 (powers of two), both
                         directions, 8 members per N (random, saturating,
                         impulse, small-signal, full-scale and alternating
                         inputs) plus a single-member run (the howmany = 1
                         code path)
  q7_reference.npz       the same for Q0.7
  f32_c2c_reference.npz  FP32 C2C for a spread of lengths (single-radix,
                         two-level and three-level plans), both directions,
                         4 members of U[-1, 1) data
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import neon_a64  # noqa: E402
import ref_c2c_plan  # noqa: E402

FIXED_SOURCES = {
    "q15": ["plfft_q15_jjjn_uu.S", "plfft_q15_jjjn_uun.S", "plfft_q15_jjjn_gs.S", "plfft_q15_jjjn_gu.S",
            "plfft_q15_jjjn_us.S", "plfft_ab_q15_jjjt_dit_gu.S", "plfft_ab_q15_jjjt_dit_gs.S",
            "plfft_ac_q15_jjjt_dit_uu.S"],
    "q7": ["plfft_q7_pppn_uu.S", "plfft_q7_pppn_uun.S", "plfft_q7_pppn_gs.S", "plfft_q7_pppn_gu.S",
           "plfft_q7_pppn_us.S", "plfft_ab_q7_pppt_dit_gu.S", "plfft_ab_q7_pppt_dit_gs.S",
           "plfft_ac_q7_pppt_dit_uu.S"],
}
F32_SOURCES = ["plfft_cccn_uu.S", "plfft_cccn_uun.S", "plfft_cccn_gs.S", "plfft_cccn_gu.S", "plfft_cccn_us.S",
               "plfft_ab_ccct_dit_gu.S", "plfft_ab_ccct_dit_gs.S", "plfft_ac_ccct_dit_uu.S"]

FIXED_SIZES = [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]
F32_SIZES = [2, 3, 5, 7, 8, 12, 16, 20, 32, 64, 100, 128, 360, 1000, 1024, 4096]


def fixed_inputs(n, seed, bits):
    """8 members: random full range, saturating constants, impulse, small
    signal, random full-scale extremes, alternating sign (all energy at n/2)."""
    lo, hi = -(1 << (bits - 1)), (1 << (bits - 1)) - 1
    dt = np.int16 if bits == 16 else np.int8
    rng = np.random.default_rng(seed)
    x = rng.integers(lo, hi + 1, (8, n, 2)).astype(dt)
    x[1] = hi
    x[2] = lo
    x[3] = 0
    x[3, 0] = (hi, lo)
    x[4] = np.clip(rng.standard_normal((n, 2)) * (3000 if bits == 16 else 12), lo, hi).astype(dt)
    x[6] = np.where(rng.random((n, 2)) < 0.5, lo, hi)
    x[7, :, 0] = np.where(np.arange(n) % 2 == 0, hi, lo)
    x[7, :, 1] = lo
    return x


def run(kern, dtype, n, dirn, x):
    machine = neon_a64.Machine(kern)
    hm = x.shape[0]
    flat = x.reshape(-1) if dtype == "f32" else x.reshape(-1, 2)
    y, desc = ref_c2c_plan.run_c2c(machine, dtype, dirn, flat, n, hm)
    return y.reshape(x.shape), desc


def make_fixed(kdir, dtype, bits):
    kern = neon_a64.Kernels([os.path.join(kdir, s) for s in FIXED_SOURCES[dtype]])
    out = {}
    for n in FIXED_SIZES:
        x = fixed_inputs(n, 1000 + n if dtype == "q15" else 7000 + n, bits)
        out[f"x_{n}"] = x
        for dirn in (-1, 1):
            d = "f" if dirn < 0 else "b"
            out[f"y_{n}_{d}"], desc = run(kern, dtype, n, dirn, x)
            out[f"y1_{n}_{d}"], _ = run(kern, dtype, n, dirn, x[:1])
            out[f"plan_{n}_{d}"] = np.array(desc)
            print(dtype, n, d, desc, flush=True)
    np.savez_compressed(os.path.join(HERE, f"{dtype}_reference.npz"), **out)


def make_f32(kdir):
    kern = neon_a64.Kernels([os.path.join(kdir, s) for s in F32_SOURCES])
    out = {}
    for n in F32_SIZES:
        rng = np.random.default_rng(5000 + n)
        x = (rng.uniform(-1, 1, (4, n)) + 1j * rng.uniform(-1, 1, (4, n))).astype(np.complex64)
        out[f"x_{n}"] = x
        for dirn in (-1, 1):
            d = "f" if dirn < 0 else "b"
            out[f"y_{n}_{d}"], desc = run(kern, "f32", n, dirn, x)
            out[f"plan_{n}_{d}"] = np.array(desc)
            print("f32", n, d, desc, flush=True)
    np.savez_compressed(os.path.join(HERE, "f32_c2c_reference.npz"), **out)


def main():
    kdir = os.path.join(sys.argv[1], "src", "providers", "aot", "asm", "neon")
    which = sys.argv[2:] or ["q15", "q7", "f32"]
    if "q15" in which:
        make_fixed(kdir, "q15", 16)
    if "q7" in which:
        make_fixed(kdir, "q7", 8)
    if "f32" in which:
        make_f32(kdir)


if __name__ == "__main__":
    main()
