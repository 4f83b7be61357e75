"""Test-only torch.autograd.Function around a plfft_b200 plan.

forward: plfft_cuda_execute_async on the plan; backward: the plan's adjoint
kernels (plfft_cuda_execute_adjoint_async).  Tensors may be FP64 at the
interface (for gradcheck); the device kernels compute in FP32.
"""
import torch

import plfft

_CPLX = {torch.complex64, torch.complex128}


def _to_kernel(t, complex_data):
    t = t.detach()
    if complex_data:
        return t.to(torch.complex64).contiguous()
    return t.to(torch.float32).contiguous()


class PlanFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, plan, out_numel, out_complex):
        in_complex = x.dtype in _CPLX
        xi = _to_kernel(x, in_complex)
        y = torch.empty(out_numel, dtype=torch.complex64 if out_complex else torch.float32, device=x.device)
        plan.execute_async(xi.data_ptr(), y.data_ptr(), 0, torch.cuda.current_stream().cuda_stream)
        ctx.plan = plan
        ctx.in_meta = (x.shape, x.dtype, in_complex)
        ctx.out_complex = out_complex
        wide = torch.complex128 if out_complex else torch.float64
        return y.to(wide) if x.dtype in (torch.float64, torch.complex128) else y

    @staticmethod
    def backward(ctx, gy):
        shape, dtype, in_complex = ctx.in_meta
        g = _to_kernel(gy, ctx.out_complex)
        gx = torch.empty(shape.numel(), dtype=torch.complex64 if in_complex else torch.float32, device=gy.device)
        ctx.plan.execute_adjoint(g.data_ptr(), gx.data_ptr(), 0, torch.cuda.current_stream().cuda_stream)
        return gx.to(dtype).reshape(shape), None, None, None


def apply(plan, x, out_numel, out_complex):
    return PlanFunction.apply(x, plan, out_numel, out_complex)
