"""torch.autograd.Function wrapper around the hand-written leapfrog adjoint.

The forward computes L = mean_i |x_T,i - target_i|^2 after `nsteps`
kick-drift-kick steps from (x0, v0, m) with the CUDA kernels; the backward
returns the gradients the adjoint sweep already produced (one C call does
both, so the forward keeps them). Tensors are FP64 on the host or any device
(they are copied through host memory at the C boundary: the wrapper exists
to test the adjoint against torch's autograd machinery, not as a fast path).
"""
from __future__ import annotations

import numpy as np
import torch

from .api import MIXED, Context, Params


class LeapfrogLoss(torch.autograd.Function):
    @staticmethod
    def forward(fctx, x0, v0, m, target, params: Params, nsteps: int, precision: int = MIXED,
                checkpoint_every: int = 32, context: Context | None = None):
        ctx_ = context or Context(0)
        ctx_.upload(x0.detach().cpu().numpy(), v0.detach().cpu().numpy(), m.detach().cpu().numpy())
        loss, gx, gv, gm = ctx_.adjoint(params, nsteps, target.detach().cpu().numpy(), precision, checkpoint_every)
        dev, dt = x0.device, x0.dtype
        fctx.save_for_backward(torch.as_tensor(gx, dtype=dt, device=dev), torch.as_tensor(gv, dtype=dt, device=dev),
                               torch.as_tensor(gm, dtype=dt, device=dev))
        return torch.tensor(loss, dtype=dt, device=dev)

    @staticmethod
    def backward(fctx, grad_out):
        gx, gv, gm = fctx.saved_tensors
        return grad_out * gx, grad_out * gv, grad_out * gm, None, None, None, None, None, None


def leapfrog_loss(x0, v0, m, target, params: Params, nsteps: int, precision: int = MIXED,
                  checkpoint_every: int = 32, context: Context | None = None):
    """Differentiable trajectory loss (see module docstring)."""
    return LeapfrogLoss.apply(x0, v0, m, target, params, nsteps, precision, checkpoint_every, context)
