"""torch.autograd wrapper of the SpMM and its adjoints -- a gradient harness.

    Y = spmm(plan, vals, B)

computes Y = A B with A the plan's sparsity pattern carrying `vals` (one
value per nonzero, in the CSR order the plan was built from). Backward:
    d vals = SDDMM(dY, B) on A's pattern   (tca_sddmm)
    d B    = A^T dY                         (tca_spmm_t)
Both accumulate in FP32; dY is rounded to FP16 (the kernels' input type)."""
from __future__ import annotations

import torch

from . import Plan


class SpMMFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, B, plan: Plan, out_dtype):
        v16 = vals.detach().to(torch.float16).contiguous()
        B16 = B.detach().to(torch.float16).contiguous()
        plan.update_values(v16)
        Y = plan.spmm(B16, out_dtype=out_dtype)
        ctx.plan = plan
        ctx.save_for_backward(v16, B16)
        ctx.vals_dtype, ctx.B_dtype = vals.dtype, B.dtype
        return Y

    @staticmethod
    def backward(ctx, dY):
        v16, B16 = ctx.saved_tensors
        plan = ctx.plan
        dY16 = dY.to(torch.float16).contiguous()
        d_vals = d_B = None
        if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
            plan.update_values(v16)  # the pattern's values as they were in forward
        if ctx.needs_input_grad[0]:
            d_vals = plan.sddmm(dY16, B16, out_dtype=torch.float32).to(ctx.vals_dtype)
        if ctx.needs_input_grad[1]:
            d_B = plan.spmm_t(dY16, out_dtype=torch.float32).to(ctx.B_dtype)
        return d_vals, d_B, None, None


def spmm(plan: Plan, vals, B, out_dtype=torch.float32):
    """Differentiable Y = A(vals) @ B on the plan's pattern."""
    return SpMMFunction.apply(vals, B, plan, out_dtype)
