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

Per-kernel Functions (each forward kernel with its hand-written adjoint kernel
as the backward pass, for composing custom losses and solvers with torch):

* ``AdvectScalarGrid`` / ``advect_scalar_grid``: s1 sampled at the RK
  backtrace foot through u0 (fm_advect_scalar_grid); backward
  fm_advect_scalar_grid_adj (dL/ds1 and dL/du0 through the backtrace).
* ``AdvectUGrid`` / ``advect_u_grid``: u1 sampled at the backtrace feet of the
  face nodes (fm_advect_u_grid; u1 = u0 for self-advection); backward
  fm_advect_u_grid_adj.
* ``PullbackU`` / ``pullback_u``: alpha (T_c . u0(psi_c) + beta base_c), the
  impulse pullback of advect_u and the BFECC epilogues (fm_pullback_u);
  backward fm_pullback_u_adj (dL/du0, dL/dT, dL/dpsi, dL/dbase).
* ``PullbackScalar`` / ``pullback_scalar``: alpha (s0(psi) + beta base)
  (fm_pullback_scalar); backward fm_pullback_scalar_adj.
* ``Project`` / ``project``: the MGPCG pressure projection P (Poisson).  P is
  symmetric (u - G A^-1 D u with D = -G^T on the interior faces, wall faces
  zeroed), so the backward pass is the same projection of the incoming
  gradient -- the reference's Poisson_adj (3D/fast_mgpcg.py:283-323) -- exact
  to the solver's tolerance.

The adjoint kernels accumulate field gradients with atomic adds, so repeated
backward passes agree to rounding, not bit for bit.
"""
from __future__ import annotations

import torch

from . import kernels as K
from ._lib import FlowmapError
from .kernels import GridSpec


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


def _zeros(ts, want):
    return [torch.zeros_like(t) for t in ts] if want else None


def _c(ts):
    return [t.contiguous() for t in ts]


class AdvectScalarGrid(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rk, dx, dt, s1, *u0):
        g = GridSpec(tuple(s1.shape))
        s1 = s1.contiguous()
        u0 = _c(u0)
        s2 = torch.empty_like(s1)
        K.advect_scalar_grid(g, rk, dx, dt, u0, s1, s2)
        ctx.args = (g, rk, dx, dt)
        ctx.save_for_backward(s1, *u0)
        return s2

    @staticmethod
    def backward(ctx, g_s2):
        g, rk, dx, dt = ctx.args
        s1, *u0 = ctx.saved_tensors
        want_s1, want_u0 = ctx.needs_input_grad[3], any(ctx.needs_input_grad[4:])
        g_s1 = torch.zeros_like(s1) if want_s1 else None
        g_u0 = _zeros(u0, want_u0)
        if want_s1 or want_u0:
            K.advect_scalar_grid_adj(g, rk, dx, dt, u0, s1, g_s2.contiguous(), g_u0, g_s1)
        return (None, None, None, g_s1) + (tuple(g_u0) if want_u0 else (None,) * len(u0))


class AdvectUGrid(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rk, dx, dt, *u01):
        d = len(u01) // 2
        u0, u1 = _c(u01[:d]), _c(u01[d:])
        g = GridSpec.from_mac(u0)
        u2 = [torch.empty_like(x) for x in u1]
        K.advect_u_grid(g, rk, dx, dt, u0, u1, u2)
        ctx.args = (g, rk, dx, dt, d)
        ctx.save_for_backward(*u0, *u1)
        return tuple(u2)

    @staticmethod
    def backward(ctx, *g_u2):
        g, rk, dx, dt, d = ctx.args
        saved = ctx.saved_tensors
        u0, u1 = list(saved[:d]), list(saved[d:])
        want_u0, want_u1 = any(ctx.needs_input_grad[3:3 + d]), any(ctx.needs_input_grad[3 + d:])
        g_u0, g_u1 = _zeros(u0, want_u0), _zeros(u1, want_u1)
        if want_u0 or want_u1:
            K.advect_u_grid_adj(g, rk, dx, dt, u0, u1, _c(g_u2), g_u0, g_u1)
        return ((None, None, None) + (tuple(g_u0) if want_u0 else (None,) * d)
                + (tuple(g_u1) if want_u1 else (None,) * d))


class PullbackU(torch.autograd.Function):
    @staticmethod
    def forward(ctx, dx, alpha, beta, d, *fields):
        u0, T_f, psi_f = _c(fields[:d]), _c(fields[d:2 * d]), _c(fields[2 * d:3 * d])
        base = _c(fields[3 * d:]) if len(fields) > 3 * d else None
        g = GridSpec.from_mac(u0)
        out = [torch.empty_like(x) for x in u0]
        K.pullback_u(g, dx, u0, out, T_f, psi_f, alpha, beta, base)
        ctx.args = (g, dx, alpha, beta, d, base is not None)
        ctx.save_for_backward(*u0, *T_f, *psi_f)
        return tuple(out)

    @staticmethod
    def backward(ctx, *g_out):
        g, dx, alpha, beta, d, has_base = ctx.args
        saved = ctx.saved_tensors
        u0, T_f, psi_f = list(saved[:d]), list(saved[d:2 * d]), list(saved[2 * d:])
        need = ctx.needs_input_grad[4:]
        w_u0, w_T, w_psi = any(need[:d]), any(need[d:2 * d]), any(need[2 * d:3 * d])
        w_base = has_base and any(need[3 * d:])
        g_u0, g_T, g_psi = _zeros(u0, w_u0), _zeros(T_f, w_T), _zeros(psi_f, w_psi)
        g_base = [torch.zeros_like(x) for x in u0] if w_base else None
        if w_u0 or w_T or w_psi or w_base:
            K.pullback_u_adj(g, dx, u0, T_f, psi_f, _c(g_out), alpha, beta, g_u0, g_T, g_psi, g_base)
        res = [None, None, None, None]
        for want, gr in ((w_u0, g_u0), (w_T, g_T), (w_psi, g_psi)):
            res += list(gr) if want else [None] * d
        if has_base:
            res += list(g_base) if w_base else [None] * d
        return tuple(res)


class PullbackScalar(torch.autograd.Function):
    @staticmethod
    def forward(ctx, dx, alpha, beta, s0, psi, base=None):
        s0, psi = s0.contiguous(), psi.contiguous()
        base = base.contiguous() if base is not None else None
        g = GridSpec(tuple(s0.shape))
        out = torch.empty_like(s0)
        K.pullback_scalar(g, dx, s0, out, psi, alpha, beta, base)
        ctx.args = (g, dx, alpha, beta, base is not None)
        ctx.save_for_backward(s0, psi)
        return out

    @staticmethod
    def backward(ctx, g_out):
        g, dx, alpha, beta, has_base = ctx.args
        s0, psi = ctx.saved_tensors
        w_s0, w_psi = ctx.needs_input_grad[3], ctx.needs_input_grad[4]
        w_base = has_base and ctx.needs_input_grad[5]
        g_s0 = torch.zeros_like(s0) if w_s0 else None
        g_psi = torch.zeros_like(psi) if w_psi else None
        g_base = torch.zeros_like(s0) if w_base else None
        if w_s0 or w_psi or w_base:
            K.pullback_scalar_adj(g, dx, s0, psi, g_out.contiguous(), alpha, beta, g_s0, g_psi, g_base)
        return None, None, None, g_s0, g_psi, g_base


class Project(torch.autograd.Function):
    @staticmethod
    def forward(ctx, solver, *u):
        out = [x.detach().clone(memory_format=torch.contiguous_format) for x in u]
        solver.project(out)
        ctx.solver = solver
        return tuple(out)

    @staticmethod
    def backward(ctx, *g_out):
        g = [x.clone(memory_format=torch.contiguous_format) for x in g_out]
        ctx.solver.project(g)  # P^T = P
        return (None,) + tuple(g)


def advect_scalar_grid(u0, s1, dx: float, dt: float, rk: int = 4):
    """Differentiable advect_scalar_grid (3D/flowmap.py:284-320)."""
    return AdvectScalarGrid.apply(rk, dx, dt, s1, *u0)


def advect_u_grid(u0, u1, dx: float, dt: float, rk: int = 4):
    """Differentiable advect_u_grid (3D/flowmap.py:202-282); pass u1 = u0 for self-advection."""
    return list(AdvectUGrid.apply(rk, dx, dt, *u0, *u1))


def pullback_u(u0, T_f, psi_f, dx: float, alpha: float = 1.0, beta: float = 0.0, base=None):
    """Differentiable advect_u / BFECC pullback (3D/flowmap.py:51-69, 405-434)."""
    extra = list(base) if base is not None else []
    return list(PullbackU.apply(dx, alpha, beta, len(u0), *u0, *T_f, *psi_f, *extra))


def pullback_scalar(s0, psi, dx: float, alpha: float = 1.0, beta: float = 0.0, base=None):
    """Differentiable advect_scalar / BFECC_scalar pullback (3D/flowmap.py:71-79, 436-452)."""
    return PullbackScalar.apply(dx, alpha, beta, s0, psi, base)


def project(solver, u):
    """Differentiable pressure projection (solver.Poisson; 3D/mgpcg.py:207-289)."""
    return list(Project.apply(solver, *u))
