"""Generate reference-output fixtures by executing the reference's own NEON
kernels (interpreter: neon_a64.py) composed as its ESTIMATE plans
(ref_plan.py).

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
  q15_c2r_reference.npz  Q0.15 / Q0.7 C2R (backward), N = 2 .. 4096: 32
  q7_c2r_reference.npz   members (N <= 256) or 6, Hermitian half spectra
                         with random, extreme, zero and constant bins; for
                         N <= 256 also the same members laid out adjacent
                         (the batched plans: yu_N)
  q15_r2c_reference.npz  Q0.15 R2C (forward), N = 2 .. 4096: 6 members
  q7_r2c_reference.npz   (random, constants at both extremes, an impulse,
                         alternating extremes, random extremes) per N; for
                         N <= 256 also 32 random members; for N <= 16 also
                         64 extreme-heavy members laid out with output
                         distance 1 (the gu kernel variant: xu_N, yu_N)
  f32_c2c_reference.npz  FP32 C2C for a spread of lengths (single-radix,
                         two-level and three-level plans), both directions,
                         4 members of U[-1, 1) data
  f32_real_reference.npz FP32 R2C and C2R for the same kind of spread, and
                         DCT-II / DST-II: the reference's R2R plan is, per
                         member, an input permutation, its ESTIMATE R2C plan
                         of length n, and a post-rotation
                         (r2r_plan.cpp:56-77, r2r_buffer_helper.hpp:316-335,
                         455-469, 686-701, 828-854); the permutation and
                         rotation are restated here in single precision
"""
import glob
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import neon_a64  # noqa: E402
import ref_plan  # noqa: E402

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
FIXED_REAL_SOURCES = {
    "q15": FIXED_SOURCES["q15"] + ["plfft_q15_jjjnoh_uu.S", "plfft_q15_jjjnoh_uun.S",
                                   "plfft_q15_hjjnoh_uu.S", "plfft_q15_hjjnoh_uun.S", "plfft_q15_hjjnoh_gs.S",
                                   "plfft_q15_hjjnoh_gu.S", "plfft_q15_hjjnoh_us.S", "plfft_ab_q15_jjjtj_dit_gu.S",
                                   "plfft_ab_q15_jjjtj_dit_gs.S", "plfft_ab_q15_jjjtol_dit_uun.S",
                                   "plfft_ac_q15_jjjtj_dit_uu.S", "plfft_ac_q15_jjjtol_dit_uu.S"],
    "q7": FIXED_SOURCES["q7"] + ["plfft_q7_pppnoh_uu.S", "plfft_q7_pppnoh_uun.S",
                                 "plfft_q7_rppnoh_uu.S", "plfft_q7_rppnoh_uun.S", "plfft_q7_rppnoh_gs.S",
                                 "plfft_q7_rppnoh_gu.S", "plfft_q7_rppnoh_us.S", "plfft_ab_q7_ppptj_dit_gu.S",
                                 "plfft_ab_q7_ppptj_dit_gs.S", "plfft_ab_q7_ppptol_dit_uun.S",
                                 "plfft_ac_q7_ppptj_dit_uu.S", "plfft_ac_q7_ppptol_dit_uu.S"],
}
F32_SIZES = [2, 3, 5, 7, 8, 12, 16, 20, 32, 64, 100, 128, 360, 1000, 1024, 4096]
REAL_SIZES = [2, 3, 8, 16, 20, 64, 100, 256, 1000, 1024, 4096]
R2R_SIZES = [16, 100, 1024]
REAL_SOURCES = F32_SOURCES + ["plfft_sccnoh_uu.S", "plfft_sccnoh_uun.S", "plfft_sccnoh_gs.S", "plfft_sccnoh_gu.S",
                              "plfft_sccnoh_us.S", "plfft_ccsn_uu.S", "plfft_ccsn_uun.S", "plfft_ccsn_gs.S",
                              "plfft_ccsn_gu.S", "plfft_ccsn_us.S", "plfft_cccnoh_uu.S", "plfft_cccnoh_uun.S",
                              "plfft_cccnih_uu.S", "plfft_cccnih_uun.S", "plfft_ab_ccctj_dit_gu.S",
                              "plfft_ab_ccctj_dit_gs.S", "plfft_ab_ccctol_dit_uun.S", "plfft_ab_ccctil_dif_us.S",
                              "plfft_ab_ccctil_dif_gs.S", "plfft_ab_ccctih_dif_us.S", "plfft_ab_ccctih_dif_gs.S",
                              "plfft_ac_ccctj_dit_uu.S", "plfft_ac_ccctol_dit_uu.S", "plfft_ac_ccctil_dif_uu.S",
                              "plfft_ac_ccctih_dif_uu.S"]


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
    y, desc = ref_plan.run_c2c(machine, dtype, dirn, flat, n, hm)
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


def fixed_real_inputs(n, hm, seed, bits):
    lo, hi = -(1 << (bits - 1)), (1 << (bits - 1)) - 1
    dt = np.int16 if bits == 16 else np.int8
    rng = np.random.default_rng(seed)
    x = rng.integers(lo, hi + 1, (hm, n)).astype(dt)
    x[1] = hi
    x[2] = lo
    x[3] = 0
    x[3, 0] = hi
    x[4, ::2] = lo
    x[4, 1::2] = hi
    x[5] = np.where(rng.random(n) < 0.5, lo, hi)
    return x


def make_fixed_real(kdir, dtype, bits):
    kern = neon_a64.Kernels([os.path.join(kdir, s) for s in FIXED_REAL_SOURCES[dtype]])
    out = {}
    for n in FIXED_SIZES:
        hm = 32 if n <= 256 else 6
        x = fixed_real_inputs(n, hm, (3000 if bits == 16 else 9000) + n, bits)
        y, desc = ref_plan.run(neon_a64.Machine(kern), dtype, "r2c", -1, x.ravel(), n, hm)
        out[f"x_{n}"], out[f"y_{n}"], out[f"plan_{n}"] = x, y.reshape(hm, n // 2 + 1, 2), np.array(desc)
        print(dtype, "r2c", n, desc, flush=True)
        if n <= 16:
            # members adjacent in the output (ostride hm, odist 1): the
            # reference's gu kernel variant, whose length-4 and length-8
            # codelets round differently from the gs one above
            hm = 64
            rng = np.random.default_rng((3100 if bits == 16 else 9100) + n)
            lo, hi = -(1 << (bits - 1)), (1 << (bits - 1)) - 1
            ext = np.array([lo, lo + 1, hi - 1, hi])
            xu = np.where(rng.random((hm, n)) < 0.85, rng.choice(ext, (hm, n)),
                          rng.integers(lo, hi + 1, (hm, n))).astype(x.dtype)
            y, desc = ref_plan.run(neon_a64.Machine(kern), dtype, "r2c", -1, xu.ravel(), n, hm,
                                   1, n, hm, 1)
            out[f"xu_{n}"], out[f"plan_u_{n}"] = xu, np.array(desc)
            out[f"yu_{n}"] = np.ascontiguousarray(y.reshape(n // 2 + 1, hm, 2).transpose(1, 0, 2))
            print(dtype, "r2c odist 1", n, desc, flush=True)
    np.savez_compressed(os.path.join(HERE, f"{dtype}_r2c_reference.npz"), **out)


def make_fixed_c2r(kdir, dtype, bits):
    """Fixed-point C2R (backward): the reference's real-output plans on
    Hermitian half spectra (random, extremes, zero and constant bins), for
    N = 2..4096; for N <= 256 also a batch laid out with members adjacent
    (istride = howmany, idist = 1: the batched AC plans)."""
    kern = neon_a64.Kernels(sorted(glob.glob(os.path.join(kdir, f"*{dtype}*.S"))))
    lo, hi = -(1 << (bits - 1)), (1 << (bits - 1)) - 1
    it = np.int16 if bits == 16 else np.int8
    out = {}
    for n in FIXED_SIZES:
        h = n // 2 + 1
        hm = 32 if n <= 256 else 6
        rng = np.random.default_rng((5000 if bits == 16 else 7000) + n)
        X = np.where(rng.random((hm, h, 2)) < 0.6, rng.choice([lo, hi, lo + 1, hi - 1, 0], (hm, h, 2)),
                     rng.integers(lo, hi + 1, (hm, h, 2))).astype(it)
        X[1] = 0
        X[1, 0, 0] = hi  # a constant signal
        X[2] = hi
        X[3] = lo
        y, desc = ref_plan.run(neon_a64.Machine(kern), dtype, "c2r", 1, X.ravel(), n, hm)
        out[f"x_{n}"], out[f"y_{n}"], out[f"plan_{n}"] = X, y.reshape(hm, n), np.array(desc)
        print(dtype, "c2r", n, desc, flush=True)
        if n <= 256:
            buf = np.ascontiguousarray(X.transpose(1, 0, 2))  # element k of member b at k * hm + b
            y, desc = ref_plan.run(neon_a64.Machine(kern), dtype, "c2r", 1, buf.ravel(), n, hm, hm, 1, hm, 1)
            out[f"yu_{n}"], out[f"plan_u_{n}"] = np.ascontiguousarray(y.reshape(n, hm).T), np.array(desc)
            print(dtype, "c2r members adjacent", n, desc, flush=True)
    np.savez_compressed(os.path.join(HERE, f"{dtype}_c2r_reference.npz"), **out)


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


def dct2_input(x):
    """r2r_buffer_helper<DCT_2>::prepare_fft_input: even elements to the
    first half, odd elements reversed into the second half."""
    n = x.shape[-1]
    i = np.arange(n)
    src = np.where(i < (n + 1) // 2, 2 * i, 2 * (n - i) - 1)
    return x[..., src]


def dst2_input(x):
    """r2r_buffer_helper<DST_2>::prepare_fft_input: fft_in[j] = +-x[i],
    j = i / 2 (i even), n - (i + 1) / 2 (i odd, negated)."""
    n = x.shape[-1]
    out = np.empty_like(x)
    for i in range(n):
        j = n - (i + 1) // 2 if i % 2 else i // 2
        out[..., j] = -x[..., i] if i % 2 else x[..., i]
    return out


def dct2_output(F, n):
    """r2r_buffer_helper<DCT_2>::extract_output_from_fft with the single-
    precision rotation w_k = (cos m, -sin m), m = pi k / 2n
    (generate_twiddles.hpp:191-194)."""
    y = np.empty(F.shape[:-1] + (n,), np.float32)
    y[..., 0] = F[..., 0].real * np.float32(2)
    for k in range(1, n // 2 + 1):
        m = np.float32(np.pi) * np.float32(k) / np.float32(2 * n)
        w = np.complex64(complex(np.cos(m), -np.sin(m)))
        j = (F[..., k] * w) * np.complex64(2)
        y[..., k] = j.real
        y[..., n - k] = -j.imag
    return y


def dst2_output(F, n):
    """r2r_buffer_helper<DST_2>::extract_output_from_fft: division by
    (sin c, -cos c), c = pi i / 2n, real part times 2."""
    y = np.empty(F.shape[:-1] + (n,), np.float32)
    h = n // 2 + 1
    for i in range(1, n):
        tmp = F[..., i] if i < h else np.conj(F[..., n - i])
        c = np.float32(0.5 * np.pi * i / n)
        d = complex(np.sin(c), -np.cos(c))
        y[..., i - 1] = (tmp.astype(np.complex128) / d).real.astype(np.float32) * np.float32(2)
    y[..., n - 1] = F[..., 0].real * np.float32(2)
    return y


def make_real(kdir):
    kern = neon_a64.Kernels([os.path.join(kdir, s) for s in REAL_SOURCES])
    out = {}
    for n in REAL_SIZES:
        rng = np.random.default_rng(6000 + n)
        h = n // 2 + 1
        x = rng.uniform(-1, 1, (4, n)).astype(np.float32)
        y, desc = ref_plan.run(neon_a64.Machine(kern), "f32", "r2c", -1, x.ravel(), n, 4)
        out[f"r2c_x_{n}"], out[f"r2c_y_{n}"], out[f"r2c_plan_{n}"] = x, y.reshape(4, h), np.array(desc)
        X = (rng.uniform(-1, 1, (4, h)) + 1j * rng.uniform(-1, 1, (4, h))).astype(np.complex64)
        y, desc = ref_plan.run(neon_a64.Machine(kern), "f32", "c2r", 1, X.ravel(), n, 4)
        out[f"c2r_x_{n}"], out[f"c2r_y_{n}"], out[f"c2r_plan_{n}"] = X, y.reshape(4, n), np.array(desc)
        print("f32 real", n, desc, flush=True)
    for n in R2R_SIZES:
        rng = np.random.default_rng(6500 + n)
        x = rng.uniform(-1, 1, (4, n)).astype(np.float32)
        for name, pre, post in (("dct2", dct2_input, dct2_output), ("dst2", dst2_input, dst2_output)):
            F = np.stack([ref_plan.run(neon_a64.Machine(kern), "f32", "r2c", -1, pre(x[b]), n, 1)[0]
                          for b in range(4)])
            out[f"{name}_x_{n}"], out[f"{name}_y_{n}"] = x, post(F, n)
        print("f32 r2r", n, flush=True)
    np.savez_compressed(os.path.join(HERE, "f32_real_reference.npz"), **out)


def main():
    kdir = os.path.join(sys.argv[1], "src", "providers", "aot", "asm", "neon")
    which = sys.argv[2:] or ["q15", "q7", "f32", "real", "q15r", "q7r", "q15cr", "q7cr"]
    if "q15" in which:
        make_fixed(kdir, "q15", 16)
    if "q7" in which:
        make_fixed(kdir, "q7", 8)
    if "f32" in which:
        make_f32(kdir)
    if "real" in which:
        make_real(kdir)
    if "q15r" in which:
        make_fixed_real(kdir, "q15", 16)
    if "q7r" in which:
        make_fixed_real(kdir, "q7", 8)
    if "q15cr" in which:
        make_fixed_c2r(kdir, "q15", 16)
    if "q7cr" in which:
        make_fixed_c2r(kdir, "q7", 8)


if __name__ == "__main__":
    main()
