"""torch.autograd integration of the flow-map adjoint.

``FlowmapLoss.apply(sim, rho0, rho_target, *u0)`` returns the scalar loss
L = sum (rho(T) - rho*)^2 of the forward leapfrog simulation started from the
MAC velocity u0.  ``forward`` runs only the forward pass
(LFM_Diff_Simulator.run_forward), which leaves the trajectory the adjoint needs
in the simulator's stores; ``backward`` runs the hand-written adjoint on that
trajectory (run_adjoint, the reference's backtrack_step_midpoint loop,
3D/lfm_midpoint_diff_simulator.py:390-594) and returns dL/du0 scaled by the
incoming gradient.  A loss evaluated without gradients (torch.no_grad, or
inputs that do not require grad) therefore costs one forward pass.  If the
simulator ran another forward pass between the two, backward first re-runs
this one's forward pass from the saved inputs.
"""
from __future__ import annotations

import torch

from ._lib import FlowmapError


class FlowmapLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sim, rho0, rho_target, *u0):
        if sim.cfg.add_control_force:
            raise FlowmapError(2, "FlowmapLoss: control forces need gradient(..., control_forces=...)")
        sim.run_forward(list(u0), rho0)
        target = torch.empty(sim.grid.shape, dtype=sim.cfg.dtype, device=sim.device)
        target.copy_(torch.as_tensor(rho_target), non_blocking=True)
        diff = sim.passive - target
        loss = torch.sum(diff.double() ** 2)  # the init_gradient formula: the same bits
        ctx.sim = sim
        ctx.serial = sim.forward_serial
        ctx.rho0 = rho0
        ctx.target = target
        ctx.save_for_backward(*u0)
        return loss

    @staticmethod
    def backward(ctx, grad_out):
        sim = ctx.sim
        if sim.forward_serial != ctx.serial:  # the trajectory was overwritten: rebuild it
            sim.run_forward(list(ctx.saved_tensors), ctx.rho0)
        _, grads = sim.run_adjoint(target_passive=ctx.target)
        scale = grad_out.to(grads[0].dtype)
        return (None, None, None) + tuple(g * scale for g in grads)


def flowmap_loss(sim, u0, rho0, rho_target):
    """Differentiable L(u0) for a list of MAC face tensors u0 (requires_grad allowed)."""
    return FlowmapLoss.apply(sim, rho0, rho_target, *u0)
