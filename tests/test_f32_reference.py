"""FP32 C2C, R2C, C2R, DCT-II and DST-II pinned to the reference's own outputs.

tests/golden/f32_c2c_reference.npz holds what the reference's NEON FP32
kernels (src/providers/aot/asm/neon/plfft_cccn_*.S, plfft_ab_ccct_dit_*.S,
plfft_ac_ccct_dit_uu.S) return when composed as its ESTIMATE plans --
single-radix kernels, two-level (cooley_tukey_ab) and three-level
(cooley_tukey_ab over cooley_tukey_ac) plans -- executed from their source
text by tests/golden/neon_a64.py (tests/golden/make_ref_golden.py).

CPU: the FP64 oracle agrees with the reference's outputs within the FP32
gate rel-L2 <= 4*log2(N)*2^-24, so the oracle's sign, ordering and scaling
conventions are the reference's.  GPU: the device path agrees with them
within the same gate.
"""
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "f32_c2c_reference.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _sizes():
    g = np.load(GOLDEN)
    return sorted({int(k.split("_")[1]) for k in g.files if k.startswith("x_")})


@pytest.mark.parametrize("n", _sizes())
@pytest.mark.parametrize("d", ["f", "b"])
def test_oracle_matches_reference_fp32_kernels(golden, n, d):
    x = golden[f"x_{n}"]
    ref = golden[f"y_{n}_{d}"]
    got = oracle.c2c(x.astype(np.complex128), -1 if d == "f" else 1)
    assert oracle.rel_l2(ref, got) <= oracle.fp32_tol(n), str(golden[f"plan_{n}_{d}"])


def test_fixture_covers_three_level_plans(golden):
    plans = [str(golden[k]) for k in golden.files if k.startswith("plan_")]
    assert any("ct-ac" in p for p in plans) and any("ct-ab" in p for p in plans)


@pytest.mark.gpu
@pytest.mark.parametrize("n", _sizes())
@pytest.mark.parametrize("d", ["f", "b"])
def test_device_matches_reference_fp32_kernels(golden, n, d):
    import plfft
    import torch

    x = golden[f"x_{n}"]
    hm = x.shape[0]
    plan = plfft.make_plan("c2c", n, hm, direction=-1 if d == "f" else 1)
    dx = torch.from_numpy(np.ascontiguousarray(x).ravel()).cuda()
    dy = torch.empty_like(dx)
    plan.execute(dx.data_ptr(), dy.data_ptr())
    got = dy.cpu().numpy().reshape(hm, n)
    assert oracle.rel_l2(got, golden[f"y_{n}_{d}"]) <= oracle.fp32_tol(n), plan.describe()


# ---------------------------------------------------------------------------
# R2C, C2R, DCT-II and DST-II (tests/golden/f32_real_reference.npz): the
# reference's R2C / C2R kernel compositions (plfft_sccnoh_*, plfft_ccsn_*,
# the half-spectrum ab / ac levels) and, for DCT-II / DST-II, its R2R
# input permutation and post-rotation around its R2C plan.
# ---------------------------------------------------------------------------
REAL = os.path.join(os.path.dirname(__file__), "golden", "f32_real_reference.npz")


@pytest.fixture(scope="module")
def real():
    return np.load(REAL)


def _real_sizes(prefix):
    g = np.load(REAL)
    return sorted({int(k.split("_")[-1]) for k in g.files if k.startswith(prefix + "_x_")})


@pytest.mark.parametrize("n", _real_sizes("r2c"))
def test_oracle_matches_reference_r2c_c2r(real, n):
    got = oracle.r2c(real[f"r2c_x_{n}"].astype(np.float64))
    assert oracle.rel_l2(real[f"r2c_y_{n}"], got) <= oracle.fp32_tol(n), str(real[f"r2c_plan_{n}"])
    got = oracle.c2r(real[f"c2r_x_{n}"].astype(np.complex128), n)
    assert oracle.rel_l2(real[f"c2r_y_{n}"], got) <= oracle.fp32_tol(n), str(real[f"c2r_plan_{n}"])


@pytest.mark.parametrize("n", _real_sizes("dct2"))
@pytest.mark.parametrize("kind", ["DCT_2", "DST_2"])
def test_oracle_matches_reference_r2r(real, n, kind):
    key = kind.lower().replace("_", "")
    got = oracle.r2r(real[f"{key}_x_{n}"].astype(np.float64), kind)
    assert oracle.rel_l2(real[f"{key}_y_{n}"], got) <= oracle.fp32_tol(2 * n)


@pytest.mark.gpu
@pytest.mark.parametrize("n", _real_sizes("r2c"))
def test_device_matches_reference_r2c_c2r(real, n):
    import plfft
    import torch

    x = real[f"r2c_x_{n}"]
    hm, h = x.shape[0], n // 2 + 1
    plan = plfft.make_plan("r2c", n, hm)
    dx = torch.from_numpy(np.ascontiguousarray(x).ravel()).cuda()
    dy = torch.empty(hm * h, dtype=torch.complex64, device="cuda")
    plan.execute(dx.data_ptr(), dy.data_ptr())
    assert oracle.rel_l2(dy.cpu().numpy().reshape(hm, h), real[f"r2c_y_{n}"]) <= oracle.fp32_tol(n), plan.describe()
    X = real[f"c2r_x_{n}"]
    plan = plfft.make_plan("c2r", n, hm)
    dX = torch.from_numpy(np.ascontiguousarray(X).ravel()).cuda()
    dz = torch.empty(hm * n, dtype=torch.float32, device="cuda")
    plan.execute(dX.data_ptr(), dz.data_ptr())
    assert oracle.rel_l2(dz.cpu().numpy().reshape(hm, n), real[f"c2r_y_{n}"]) <= oracle.fp32_tol(n), plan.describe()


@pytest.mark.gpu
@pytest.mark.parametrize("n", _real_sizes("dct2"))
@pytest.mark.parametrize("kind", ["DCT_2", "DST_2"])
def test_device_matches_reference_r2r(real, n, kind):
    import plfft
    import torch

    key = kind.lower().replace("_", "")
    x = real[f"{key}_x_{n}"]
    hm = x.shape[0]
    plan = plfft.make_plan("r2r", n, hm, r2r_kind=plfft.R2RKind[kind])
    dx = torch.from_numpy(np.ascontiguousarray(x).ravel()).cuda()
    dy = torch.empty_like(dx)
    plan.execute(dx.data_ptr(), dy.data_ptr())
    assert oracle.rel_l2(dy.cpu().numpy().reshape(hm, n), real[f"{key}_y_{n}"]) <= oracle.fp32_tol(2 * n), \
        plan.describe()
