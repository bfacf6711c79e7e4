"""``torch.autograd.Function`` over the CB-SpMV C ABI (a test harness).

Y = A(vals) X where ``vals`` are the matrix's input nonzero values (the
caller's COO order) and X is (n,) or (n, k).  Backward:

* dL/dX    = A^T dL/dY, on the plan's transposed CB layout (build the plan
  with ``want_transpose=1``);
* dL/dvals = for each input nonzero k, dL/dY[row_k, :] . X[col_k, :],
  computed per stored value of A (``adjoint``: the value-gradient kernel on
  a second stream beside A^T dL/dY, the faster of the library's two adjoint
  forms on the stream layouts) and gathered back to input order through
  ``input_slots`` -- every input is summed into exactly one stored value, so
  that value's gradient is the input's gradient.  ``adjoint_fused`` (one
  launch, gradient gathered through ``grad_positions_t``) computes the same.

Build the plan with ``keep_values=1`` when its initial values may all be 1:
a unit-valued plan stores no values and cannot take new ones.
"""
from __future__ import annotations

import torch


class CBSpMVFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, x, plan):
        plan.set_values(vals.detach().contiguous())
        y = plan.spmv(x.detach().contiguous())
        ctx.plan = plan
        ctx.save_for_backward(x)
        return y

    @staticmethod
    def backward(ctx, gy):
        plan = ctx.plan
        (x,) = ctx.saved_tensors
        gy = gy.contiguous()
        want_gx, want_v = ctx.needs_input_grad[1], ctx.needs_input_grad[0]
        if not (want_gx or want_v):
            return None, None, None
        # both in one call: the value gradient overlaps A^T g on a second
        # stream
        gx, gslots = plan.adjoint(gy, x.contiguous(), want_gx=want_gx, want_gvals=want_v)
        gvals = None
        if want_v:
            slots = getattr(plan, "_slots_dev", None)
            if slots is None or slots.device != gy.device:
                slots = torch.from_numpy(plan.input_slots()).to(gy.device)
                plan._slots_dev = slots
            gvals = gslots[slots]
        return gvals, gx, None


def cbspmv_apply(plan, vals, x):
    """Differentiable Y = A(vals) X through the plan."""
    return CBSpMVFunction.apply(vals, x, plan)
