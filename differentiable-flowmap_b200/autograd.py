"""torch.autograd integration of the flow-map adjoint.

``FlowmapLoss.apply(sim, rho0, rho_target, *u0)`` runs the forward leapfrog
simulation and the hand-written adjoint (LFM_Diff_Simulator.gradient) and
returns the scalar loss L = sum (rho(T) - rho*)^2; ``backward`` returns
dL/du0 (one tensor per MAC face grid) scaled by the incoming gradient.  The
adjoint is the reference's discretised continuous adjoint
(3D/lfm_midpoint_diff_simulator.py), not a tape of the forward kernels, so it
is computed eagerly in forward() and only scaled in backward().
"""
from __future__ import annotations

import torch


class FlowmapLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sim, rho0, rho_target, *u0):
        loss, grad = sim.gradient(list(u0), rho0, rho_target)
        ctx.save_for_backward(*grad)
        return torch.tensor(loss, dtype=torch.float64, device=u0[0].device)

    @staticmethod
    def backward(ctx, grad_out):
        grads = ctx.saved_tensors
        scale = grad_out.to(grads[0].dtype)
        return (None, None, None) + tuple(g * scale for g in grads)


def flowmap_loss(sim, u0, rho0, rho_target):
    """Differentiable L(u0) for a list of MAC face tensors u0 (requires_grad allowed)."""
    return FlowmapLoss.apply(sim, rho0, rho_target, *u0)
