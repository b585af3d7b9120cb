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
* ``RkGrid`` / ``rk_grid``: one RK2/RK4 march of a flow map psi and its
  Jacobian row T through u (fm_rk_grid, RK_grid / RK_grid_only_psi);
  backward fm_rk_grid_adj (dL/dpsi, dL/dT, dL/du, the Jacobian update
  differentiated through the B-spline's second derivative).
* ``AccumulateInit`` / ``accumulate_init``: init_c += dt F_c . f(phi_c), with
  the Adams-Bashforth-3 history of accumulate_init_new (fm_accumulate_init);
  backward through fm_pullback_u_adj and the AB3 coefficients.
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


class RkGrid(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rk, dx, dt, face, psi, T, *u):
        u = _c(u)
        g = GridSpec.from_mac(u)
        psi0 = psi.contiguous()
        T0 = T.contiguous() if T is not None else None
        psi1 = psi0.clone()
        T1 = T0.clone() if T0 is not None else None
        K.rk_grid(g, rk, dx, dt, face, psi1, T1, u)
        ctx.args = (g, rk, dx, dt, face, T0 is not None)
        ctx.save_for_backward(psi0, T0, *u)
        return (psi1, T1) if T1 is not None else psi1

    @staticmethod
    def backward(ctx, *grads):
        g, rk, dx, dt, face, has_T = ctx.args
        psi0, T0, *u = ctx.saved_tensors
        g_psi_out = grads[0].contiguous() if grads[0] is not None else torch.zeros_like(psi0)
        g_T_out = None
        if has_T:
            g_T_out = grads[1].contiguous() if grads[1] is not None else torch.zeros_like(T0)
        w_psi, w_T, w_u = ctx.needs_input_grad[4], ctx.needs_input_grad[5], any(ctx.needs_input_grad[6:])
        g_psi = torch.zeros_like(psi0) if w_psi else None
        g_T = torch.zeros_like(T0) if (w_T and has_T) else None
        g_u = _zeros(u, w_u)
        if w_psi or w_T or w_u:
            K.rk_grid_adj(g, rk, dx, dt, face, psi0, T0, u, g_psi_out, g_T_out, g_psi, g_T, g_u)
        return (None, None, None, None, g_psi, g_T) + (tuple(g_u) if w_u else (None,) * len(u))


def _ab3_coefs(ab3: bool, ind: int, dt: float):
    """d init' / d (F.f), d init' / d Hp, d init' / d Hpp of accumulate_init(_new)."""
    if not ab3 or ind == 0:
        return dt, 0.0, 0.0
    if ind == 1:
        return 7.0 / 12.0 * dt, 5.0 / 12.0 * dt, 0.0
    return 23.0 / 12.0 * dt, -16.0 / 12.0 * dt, 5.0 / 12.0 * dt


class AccumulateInit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, dx, dt, ab3, ind, d, *fields):
        f, init, F, phi = (_c(fields[i * d:(i + 1) * d]) for i in range(4))
        Hp = [x.clone(memory_format=torch.contiguous_format) for x in fields[4 * d:5 * d]] if ab3 else None
        Hpp = [x.clone(memory_format=torch.contiguous_format) for x in fields[5 * d:6 * d]] if ab3 else None
        g = GridSpec.from_mac(f)
        out = [x.clone() for x in init]
        K.accumulate_init(g, dx, dt, f, out, F, phi, Hp, Hpp, ind)
        ctx.args = (g, dx, dt, ab3, ind, d)
        ctx.save_for_backward(*f, *F, *phi)
        return tuple(out + (Hp + Hpp if ab3 else []))

    @staticmethod
    def backward(ctx, *grads):
        g, dx, dt, ab3, ind, d = ctx.args
        saved = ctx.saved_tensors
        f, F, phi = list(saved[:d]), list(saved[d:2 * d]), list(saved[2 * d:])

        def grad_or_zero(i, c):
            return grads[i] if grads[i] is not None else torch.zeros_like(f[c])

        G_init = [grad_or_zero(c, c) for c in range(d)]
        c_fv, c_hp, c_hpp = _ab3_coefs(ab3, ind, dt)
        fv_bar = [c_fv * x for x in G_init]  # dL/d(F_c . f(phi_c)) per node
        g_hist = []
        if ab3:  # Hp' = F . f(phi), Hpp' = Hp
            G_hp = [grad_or_zero(d + c, c) for c in range(d)]
            G_hpp = [grad_or_zero(2 * d + c, c) for c in range(d)]
            fv_bar = [a + b for a, b in zip(fv_bar, G_hp)]
            g_hist = [c_hp * a + b for a, b in zip(G_init, G_hpp)] + [c_hpp * a for a in G_init]
        need = ctx.needs_input_grad[5:]
        w_f, w_F, w_phi = any(need[:d]), any(need[2 * d:3 * d]), any(need[3 * d:4 * d])
        g_f, g_F, g_phi = _zeros(f, w_f), _zeros(F, w_F), _zeros(phi, w_phi)
        if w_f or w_F or w_phi:
            K.pullback_u_adj(g, dx, f, F, phi, _c(fv_bar), 1.0, 0.0, g_f, g_F, g_phi)
        res = [None] * 5
        res += list(g_f) if w_f else [None] * d
        res += G_init
        res += list(g_F) if w_F else [None] * d
        res += list(g_phi) if w_phi else [None] * d
        return tuple(res + g_hist)


def rk_grid(u, psi, T=None, face: int = -1, dx: float = 1.0, dt: float = 0.0, rk: int = 4):
    """Differentiable RK_grid / RK_grid_only_psi (3D/flowmap.py:85-179): returns psi' (and T' when T is given)."""
    return RkGrid.apply(rk, dx, dt, face, psi, T, *u)


def accumulate_init(f, init, F_f, phi_f, dx: float, dt: float, Hp=None, Hpp=None, ind: int = 0):
    """Differentiable accumulate_init (Hp/Hpp None) or accumulate_init_new (3D/flowmap.py:485-545).

    Returns init' (a list), or (init', Hp', Hpp') with the AB3 history."""
    d = len(f)
    ab3 = Hp is not None
    extra = list(Hp) + list(Hpp) if ab3 else []
    out = list(AccumulateInit.apply(dx, dt, ab3, ind, d, *f, *init, *F_f, *phi_f, *extra))
    return (out[:d], out[d:2 * d], out[2 * d:]) if ab3 else out


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
