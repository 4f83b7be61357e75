"""Adjoint kernels: dot-product identity, gradcheck, analytic reference gradient.

The adjoint of every transform is exposed through
plfft_cuda_execute_adjoint_async and wrapped (test-only) by
tests/autograd_fft.PlanFunction.  Checks:
  * <A x, y> == <x, A^T y> for every kind (FP64 accumulation of FP32 outputs);
  * torch.autograd.gradcheck with FP64 tensors at N=64, 97 (Rader),
    1031 (Bluestein) and DCT-II N=128.  The kernels compute in FP32; the maps
    are linear, so central differences are exact for any step and the step is
    chosen so FP32 rounding stays below the tolerance;
  * loss = sum W |R2C(x)|^2 (N=8192): gradient vs the FP64 oracle gradient on
    a subset, and x . grad == 2 L (quadratic form) at the full 1024-row batch.
"""
import numpy as np
import pytest

import oracle
import plfft
from autograd_fft import apply

pytestmark = pytest.mark.gpu

KIND_SPECS = {
    # name: (plan kind, r2r kind, in complex, out complex, n_in(n), n_out(n))
    "c2c": ("c2c", None, True, True),
    "r2c": ("r2c", None, False, True),
    "c2r": ("c2r", None, True, False),
}
R2R = ["DCT_1", "DCT_2", "DCT_3", "DCT_4", "DST_1", "DST_2", "DST_3", "DST_4", "DHT", "R2HC", "HC2R"]


def _sizes(kind, n):
    h = n // 2 + 1
    if kind == "r2c":
        return n, h
    if kind == "c2r":
        return h, n
    return n, n


def _rand(shape_n, cplx, rng):
    if cplx:
        return (rng.uniform(-1, 1, shape_n) + 1j * rng.uniform(-1, 1, shape_n)).astype(np.complex64)
    return rng.uniform(-1, 1, shape_n).astype(np.float32)


def _dot(a, b):
    return np.vdot(a.astype(np.complex128), b.astype(np.complex128)).real


@pytest.mark.parametrize("kind", ["c2c", "r2c", "c2r"] + R2R)
@pytest.mark.parametrize("n", [8, 17, 64, 97, 1000])
def test_adjoint_dot_product(kind, n):
    import torch

    hm = 3
    rng = np.random.default_rng(n)
    if kind in R2R:
        plan = plfft.make_plan("r2r", n, hm, r2r_kind=plfft.R2RKind[kind])
        ci = co = False
        ni = no = n
    else:
        plan = plfft.make_plan(kind, n, hm)
        ci, co = KIND_SPECS[kind][2], KIND_SPECS[kind][3]
        ni, no = _sizes(kind, n)
    x = _rand(hm * ni, ci, rng)
    y = _rand(hm * no, co, rng)
    if kind == "c2r":  # a Hermitian half-spectrum: DC and Nyquist real
        x = x.reshape(hm, ni)
        x[:, 0] = x[:, 0].real
        if n % 2 == 0:
            x[:, -1] = x[:, -1].real
        x = x.ravel()
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y).cuda()
    ax = torch.empty(hm * no, dtype=torch.complex64 if co else torch.float32, device="cuda")
    aty = torch.empty(hm * ni, dtype=torch.complex64 if ci else torch.float32, device="cuda")
    plan.execute(dx.data_ptr(), ax.data_ptr())
    plan.execute_adjoint(dy.data_ptr(), aty.data_ptr())
    torch.cuda.synchronize()
    lhs = _dot(ax.cpu().numpy(), y)
    rhs = _dot(x, aty.cpu().numpy())
    scale = np.linalg.norm(ax.cpu().numpy()) * np.linalg.norm(y) + 1e-30
    assert abs(lhs - rhs) <= 1e-5 * scale, (kind, n, lhs, rhs)


def _gradcheck(plan, n_in, n_out, in_cplx, out_cplx, fast):
    import torch

    torch.manual_seed(0)
    dt = torch.complex128 if in_cplx else torch.float64
    x = torch.randn(n_in, dtype=dt, device="cuda", requires_grad=True)
    f = lambda t: apply(plan, t, n_out, out_cplx)  # noqa: E731
    return torch.autograd.gradcheck(f, (x,), eps=5e-2, atol=2e-3, rtol=2e-3, fast_mode=fast)


@pytest.mark.parametrize("n", [64, 97, 1031])
def test_gradcheck_c2c(n):
    plan = plfft.make_plan("c2c", n, 1)
    assert _gradcheck(plan, n, n, True, True, fast=n > 64)


@pytest.mark.parametrize("n", [64, 97, 1031])
def test_gradcheck_r2c(n):
    plan = plfft.make_plan("r2c", n, 1)
    assert _gradcheck(plan, n, n // 2 + 1, False, True, fast=n > 64)


def test_gradcheck_dct2_128():
    plan = plfft.make_plan("r2r", 128, 1, r2r_kind=plfft.R2RKind.DCT_2)
    assert _gradcheck(plan, 128, 128, False, False, fast=False)


def _ref_grad(x, w):
    """FP64 gradient of sum w |rfft(x)|^2: 2 Re sum_{k<=n/2} w_k y_k e^{+2 pi i jk/n}."""
    n = x.shape[-1]
    y = oracle.r2c(x)
    g = np.zeros(x.shape, np.complex128)
    g[:, : n // 2 + 1] = w * y
    return 2.0 * oracle.c2c(g, +1).real


def test_weighted_power_loss_gradient():
    """Differentiation workload: loss = sum W |R2C(x)|^2, x FP32 1024 x 8192."""
    import torch

    n, hm = 8192, 1024
    h = n // 2 + 1
    rng = np.random.default_rng(11)
    w = rng.uniform(0.5, 1.5, h)
    plan = plfft.make_plan("r2c", n, hm)
    x = torch.from_numpy(rng.uniform(-1, 1, (hm, n)).astype(np.float32)).cuda().requires_grad_(True)
    W = torch.from_numpy(w.astype(np.float32)).cuda()
    y = apply(plan, x, hm * h, True).reshape(hm, h)
    loss = (W * (y.real ** 2 + y.imag ** 2)).sum()
    loss.backward()
    grad = x.grad.double()
    # size-independent: x . grad = 2 L for a quadratic form
    lhs = float((x.detach().double() * grad).sum())
    assert abs(lhs - 2 * float(loss)) <= 1e-4 * abs(2 * float(loss))
    # analytic FP64 reference on a subset of rows
    rows = [0, 511, 1023]
    ref = _ref_grad(x.detach().cpu().numpy()[rows].astype(np.float64), w)
    assert oracle.rel_l2(grad.cpu().numpy()[rows], ref) <= oracle.fp32_tol(n)
