"""The Blatter-Pattyn energy as a differentiable torch operation.

``IceflowEnergy.apply(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, phys)``
returns COST = sum of the per-term means (solve.py:57-59) computed by the
fused stencil kernel; its backward is the hand-written adjoint kernel (the
forward is re-run with the gradient enabled), so a loss built on it
differentiates with respect to U and V without autograd tracing the stencil.
The FP64 energy sum is cast to the dtype of U.
"""

from __future__ import annotations

import torch

from . import kernels as K


class IceflowEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, phys=None):
        U = U.contiguous()
        V = V.contiguous()
        terms, _, _ = K.energy(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, phys)
        B = U.shape[0] if U.dim() == 4 else 1
        ny, nx = U.shape[-2:]
        count = B * (ny - 1) * (nx - 1)
        ctx.save_for_backward(U, V, thk, usurf, arrhenius, slidingco)
        ctx.args = (dx, dzeta, phys, count)
        return (terms.sum() / count).to(U.dtype)

    @staticmethod
    def backward(ctx, gout):
        U, V, thk, usurf, arrhenius, slidingco = ctx.saved_tensors
        dx, dzeta, phys, count = ctx.args
        scale = float(gout) / count
        _, dU, dV = K.energy(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, phys, grad=True, grad_scale=scale)
        return dU, dV, None, None, None, None, None, None, None


def iceflow_energy(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, phys=None):
    return IceflowEnergy.apply(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, phys)
