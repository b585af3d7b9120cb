"""CPU restatement of the reference simulator's control flow (forward leapfrog
step with reinitialisation, adjoint backtrack).  TEST INFRASTRUCTURE ONLY:
the end-to-end parity checker for the CUDA simulator; never used by the product.

Follows, statement by statement (including copy_to / add_fields / scale_field
sequences, which the product fuses):
  forward  3D/lfm_midpoint_simulator.py:648-807   (step_midpoint, step_flow_map,
           backtrack_psi_grid :368-375, march_phi_grid :377-381)
  adjoint  3D/lfm_midpoint_diff_simulator.py:336-594 (init_gradient case 11,
           backtrack_step_midpoint, backtrack_flow_map)
  BFECC    3D/flowmap.py:405-452
with use_short_BFECC, BFECC_clamp, Gaussian control
forces (add_control_force), the 2D viscous term (2D/vortex/
lfm_midpoint_simulator.py:552, 607-609; diff :270-271, 387-401) and an
obstacle mask (solid-aware MGPCG and the mask kernels after every projection,
3D/lfm_midpoint_simulator.py:606-608, 712-714, 769-771, 787-789; diff
:357-361, 534-538, 572-576) as the constructor selects.  The trajectory the reference writes to
.npy files is kept in Python lists.  Two documented extensions match the
product: a run whose last reinit interval is partial stores that interval's
forward map at the last step, and the Adams-Bashforth index counts adjoint
steps from the end of the interval actually simulated (identical to the
reference's reinit_every-1-j for full intervals).
"""
from __future__ import annotations

import numpy as np

import force_oracle
import solid_oracle
from oracle import MGParams, Oracle


def viscous_force(u, nu, dx):
    """calculate_viscous_force (2D/vortex/flowmap.py:4-17) on each face grid:
    nu * (s(i+1,j) + s(i-1,j) + s(i,j+1) + s(i,j-1) - 4 s(i,j)) / dx / dx with
    sample()'s index clamp, evaluated left to right in the field's dtype."""
    out = []
    for x in u:
        t = x.dtype.type
        n0, n1 = x.shape
        ip, im = np.minimum(np.arange(n0) + 1, n0 - 1), np.maximum(np.arange(n0) - 1, 0)
        jp, jm = np.minimum(np.arange(n1) + 1, n1 - 1), np.maximum(np.arange(n1) - 1, 0)
        s = ((x[ip, :] + x[im, :]) + x[:, jp]) + x[:, jm]
        out.append(((t(nu) * (s - t(4) * x)) / t(dx) / t(dx)).astype(x.dtype))
    return out


def clamp_u(u, u1):
    """clamp_u (3D/flowmap.py:324-334, 2D/vortex/flowmap.py:333-341): u clamped to
    the min/max of u1 over the axis neighbours, sampled with sample()'s index clamp."""
    lo = hi = None
    for a in range(u1.ndim):
        n = u1.shape[a]
        for idx in (np.maximum(np.arange(n) - 1, 0), np.minimum(np.arange(n) + 1, n - 1)):
            v = np.take(u1, idx, axis=a)
            lo = v if lo is None else np.minimum(lo, v)
            hi = v if hi is None else np.maximum(hi, v)
    return np.minimum(np.maximum(u, lo), hi).astype(u1.dtype)


class OracleSim:
    def __init__(self, res, dx, dt, reinit_every, total_steps, rk=4, backward_u=True, passive=True,
                 trajectory_loss=False, prec="f64", mg=None, bfecc_clamp=False, short_bfecc=False,
                 control_forces=None, viscosity=0.0, mask=None, bvel=None):
        self.o = Oracle(tuple(res), prec)
        self.dim = len(res)
        self.res = tuple(res)
        self.dx, self.dt, self.R, self.total_steps = dx, dt, reinit_every, total_steps
        self.rk, self.backward_u, self.passive_on, self.trajectory_loss = rk, backward_u, passive, trajectory_loss
        self.bfecc_clamp, self.short = bfecc_clamp, short_bfecc
        # per step n: (center n x dim, inv_radius n, strength n x dim) in the run's dtype
        self.cf = control_forces
        self.cf_grads = {}
        self.nu = viscosity  # 2D only, as in the reference
        self.adj_viscous = 0.0
        # obstacle mask (solid > 0): the solid-aware solver and the mask kernels (solid_oracle.py)
        self.mask = None if mask is None or not np.any(np.asarray(mask) > 0) else np.asarray(mask, np.float32)
        self.bvel = bvel
        if short_bfecc:
            o = self.o
            self.psi_tem, self.phi_tem = o.zeros_cell(self.dim), o.zeros_cell(self.dim)
            self.psi_f_tem = [o.zeros_face(c, self.dim) for c in range(self.dim)]
            self.T_tem = [o.zeros_face(c, self.dim) for c in range(self.dim)]
            self.phi_f_tem = [o.zeros_face(c, self.dim) for c in range(self.dim)]
            self.F_tem = [o.zeros_face(c, self.dim) for c in range(self.dim)]
        self.mg = mg if mg is not None else MGParams(max(2, int(np.log2(min(res))) - 2), 2, 50, 0, 400, 1e-12, 0.0,
                                                    1e-12)
        o = self.o
        mac = o.zeros_mac
        self.u, self.ad_u, self.final_u, self.init_u = mac(), mac(), mac(), mac()
        self.err_u, self.tmp_u = mac(), mac()
        self.psi, self.phi = o.zeros_cell(self.dim), o.zeros_cell(self.dim)
        self.psi_f = [o.zeros_face(c, self.dim) for c in range(self.dim)]
        self.T_f = [o.zeros_face(c, self.dim) for c in range(self.dim)]
        self.phi_f = [o.zeros_face(c, self.dim) for c in range(self.dim)]
        self.F_f = [o.zeros_face(c, self.dim) for c in range(self.dim)]
        self.passive = o.zeros_cell()
        self.final_passive, self.init_passive = o.zeros_cell(), o.zeros_cell()
        self.err_passive, self.tmp_passive = o.zeros_cell(), o.zeros_cell()
        self.velocity_storage = {}
        self.store_mid, self.store_passive, self.store_maps = {}, {}, {}
        self.step_num = -1
        self.iters = []

    # -------------------------------------------------------------- helpers
    def Poisson(self, u):
        if self.mask is not None:
            m = self.mg
            _, it, rtr = solid_oracle.project(u, self.mask, m.levels, max_iters=m.max_iters, abs_tol=m.abs_tol,
                                              rel_tol=m.rel_tol, eps=m.eps, pre_post=m.pre_post, bottom=m.bottom)
            self.iters.append(it)
            return
        it, rtr, conv = self.o.Poisson(self.mg, u)
        self.iters.append(it)

    def _mask(self, adjoint=False):
        if self.mask is None:
            return
        solid_oracle.mask_velocity(self.u, self.mask, self.bvel)
        if adjoint:
            solid_oracle.mask_velocity(self.adj_u, self.mask)
        if self.passive_on:
            solid_oracle.mask_passive(self.passive, self.mask)
            if adjoint:
                solid_oracle.mask_adj_passive(self.adj_passive, self.mask)

    def reset_to_identity(self, psi, psi_f, T_f):
        self.o.reset_to_identity(psi, psi_f, T_f, self.dx)

    def RK_grid_only_psi(self, psi, u, dt):
        self.o.RK_grid(self.rk, -1, psi, None, u, self.dx, dt)

    def RK_grid(self, face, psi, T, u, dt):
        self.o.RK_grid(self.rk, face, psi, T, u, self.dx, dt)

    def BFECC(self, init_u, u, err_u, tmp_u, T_f, psi_f, F_f, phi_f):
        o = self.o
        o.advect_u(init_u, u, T_f, psi_f, self.dx)
        o.advect_u(u, err_u, F_f, phi_f, self.dx)
        for c in range(self.dim):
            err_u[c][...] = err_u[c] + (-1.0) * init_u[c]   # add_fields(err, init, err, -1)
        for c in range(self.dim):
            err_u[c][...] = 0.5 * err_u[c]                  # scale_field(err, 0.5, err)
        o.advect_u(err_u, tmp_u, T_f, psi_f, self.dx)
        for c in range(self.dim):
            err_u[c][...] = u[c] + (-1.0) * tmp_u[c]        # add_fields(u, tmp, err, -1)
        if self.bfecc_clamp:
            for c in range(self.dim):
                tmp_u[c][...] = clamp_u(err_u[c], u[c])     # clamp_u(err, u, tmp)
                u[c][...] = tmp_u[c]                        # copy_to(tmp, u)
            return
        for c in range(self.dim):
            u[c][...] = err_u[c]                            # copy_to(err, u)

    def BFECC_scalar(self, init_s, s, err_s, tmp_s, psi, phi):
        o = self.o
        o.advect_scalar(init_s, s, psi, self.dx)
        o.advect_scalar(s, err_s, phi, self.dx)
        err_s[...] = err_s + (-1.0) * init_s
        err_s[...] = 0.5 * err_s
        o.advect_scalar(err_s, tmp_s, psi, self.dx)
        err_s[...] = s + (-1.0) * tmp_s
        if self.bfecc_clamp:
            tmp_s[...] = clamp_u(err_s, s)
            s[...] = tmp_s
            return
        s[...] = err_s

    def short_maps(self, u, dt, centre):
        """use_short_BFECC's one-step maps: psi_tem with dt, phi_tem with -dt
        (3D/lfm_midpoint_simulator.py:725-739, diff :441-450)."""
        self.reset_to_identity(self.psi_tem, self.psi_f_tem, self.T_tem)
        self.reset_to_identity(self.phi_tem, self.phi_f_tem, self.F_tem)
        if centre:
            self.RK_grid_only_psi(self.psi_tem, u, dt)
            self.RK_grid_only_psi(self.phi_tem, u, -dt)
        for c in range(self.dim):
            self.RK_grid(c, self.psi_f_tem[c], self.T_tem[c], u, dt)
        for c in range(self.dim):
            self.RK_grid(c, self.phi_f_tem[c], self.F_tem[c], u, -dt)

    # -------------------------------------------------------------- forward
    def init(self, u0, passive0):
        for c in range(self.dim):
            self.u[c][...] = u0[c]
        self.Poisson(self.u)
        if self.passive_on:
            self.passive[...] = passive0
            self.init_passive[...] = self.passive
        self._mask()
        self.step_num = -1
        self.reset_to_identity(self.phi, self.phi_f, self.F_f)
        for c in range(self.dim):
            self.init_u[c][...] = self.u[c]

    def march_phi_grid(self):
        self.RK_grid_only_psi(self.phi, self.u, -1 * self.dt)
        for c in range(self.dim):
            self.RK_grid(c, self.phi_f[c], self.F_f[c], self.u, -1 * self.dt)

    def march_no_neural(self, step):
        tmp = [np.array(x) for x in self.velocity_storage[step]]
        for c in range(self.dim):
            self.RK_grid(c, self.psi_f[c], self.T_f[c], tmp, self.dt)
        self.RK_grid_only_psi(self.psi, tmp, self.dt)

    def backtrack_psi_grid(self, curr_step):
        self.reset_to_identity(self.psi, self.psi_f, self.T_f)
        self.RK_grid_only_psi(self.psi, self.u, self.dt)
        for c in range(self.dim):
            self.RK_grid(c, self.psi_f[c], self.T_f[c], self.u, self.dt)
        for step in reversed(range(curr_step)):
            self.march_no_neural(step)

    def control_force(self, n):
        """apply_gausion_force with step n's parameters (force_oracle.py)."""
        cen, inv_r, st = self.cf[n]
        return force_oracle.gaussian_force(self.res, self.dx, cen, inv_r, st)

    def step_midpoint(self):
        self.step_num += 1
        n = self.step_num
        j = n % self.R
        if self.passive_on:
            self.store_passive[n] = self.passive.copy()
        self.step_flow_map(j, self.dt)
        final = n == self.total_steps - 1
        if final and self.passive_on:
            self.store_passive[n + 1] = self.passive.copy()
        return final

    def step_flow_map(self, j, dt):
        o, d = self.o, self.dim
        for c in range(d):
            self.ad_u[c][...] = self.u[c]
        o.advect_u_grid(self.rk, self.ad_u, self.ad_u, self.u, self.dx, 0.5 * dt)
        if self.cf is not None:  # 3D/lfm_midpoint_simulator.py:694-706
            f = self.control_force(self.step_num)
            for c in range(d):
                self.u[c][...] = self.u[c] + (0.5 * dt) * f[c]
        self.Poisson(self.u)
        self._mask()
        if self.nu:  # 2D/vortex/lfm_midpoint_simulator.py:552
            self.vis = viscous_force(self.u, self.nu, self.dx)
        self.velocity_storage[j] = [x.copy() for x in self.u]
        self.march_phi_grid()
        self.store_mid[self.step_num] = [x.copy() for x in self.u]
        if self.short:
            self.short_maps(self.u, dt, self.passive_on)
            if self.passive_on:
                self.BFECC_scalar(self.passive, self.final_passive, self.err_passive, self.tmp_passive,
                                  self.psi_tem, self.phi_tem)
                self.passive[...] = self.final_passive
            self.BFECC(self.ad_u, self.u, self.err_u, self.tmp_u, self.T_tem, self.psi_f_tem, self.F_tem,
                       self.phi_f_tem)
        else:
            if self.passive_on:
                o.advect_scalar_grid(self.rk, self.u, self.passive, self.final_passive, self.dx, dt)
                self.passive[...] = self.final_passive
            o.advect_u_grid(self.rk, self.u, self.ad_u, self.final_u, self.dx, dt)
            for c in range(d):
                self.u[c][...] = self.final_u[c]
        if self.cf is not None:  # 3D/lfm_midpoint_simulator.py:755-760
            f = self.control_force(self.step_num)
            for c in range(d):
                self.u[c][...] = self.u[c] + dt * f[c]
            o.accumulate_init(f, self.init_u, self.F_f, self.phi_f, self.dx, dt)
        if self.nu:  # 2D/vortex/lfm_midpoint_simulator.py:607-609
            for c in range(d):
                self.u[c][...] = self.u[c] + dt * self.vis[c]
            o.accumulate_init(self.vis, self.init_u, self.F_f, self.phi_f, self.dx, dt)
        self.Poisson(self.u)
        self._mask()
        n = self.step_num
        if j == self.R - 1:
            self.backtrack_psi_grid(self.R - 1)
            self.BFECC(self.init_u, self.u, self.err_u, self.tmp_u, self.T_f, self.psi_f, self.F_f, self.phi_f)
            self.Poisson(self.u)
            self._mask()
            if self.passive_on:
                self.BFECC_scalar(self.init_passive, self.passive, self.err_passive, self.tmp_passive, self.psi,
                                  self.phi)
                self.init_passive[...] = self.passive
            self.store_maps[n // self.R] = (self.phi.copy(), [x.copy() for x in self.phi_f],
                                            [x.copy() for x in self.F_f])
            self.reset_to_identity(self.phi, self.phi_f, self.F_f)
            for c in range(d):
                self.init_u[c][...] = self.u[c]
            self.velocity_storage = {}
        elif n == self.total_steps - 1:
            self.store_maps[n // self.R] = (self.phi.copy(), [x.copy() for x in self.phi_f],
                                            [x.copy() for x in self.F_f])

    # -------------------------------------------------------------- adjoint
    def init_gradient(self, target=None, seed=None):
        """Passive loss seed (case 11), or seed = (loss, [adj_u faces]) for a velocity loss."""
        o, d = self.o, self.dim
        self.final_ind = self.step_num + 1
        self.adj_viscous = 0.0
        self.adj_u = o.zeros_mac()
        self.src = o.zeros_mac()
        self.H_prev, self.H_prev_prev = o.zeros_mac(), o.zeros_mac()
        self.mid_u = o.zeros_mac()
        self.adj_passive_f = o.zeros_mac()
        if seed is not None:
            self.loss = float(seed[0])
            for c in range(d):
                self.adj_u[c][...] = seed[1][c]
            self.adj_passive = o.zeros_cell()
        else:
            diff = self.passive - target
            self.adj_passive = (2 * diff).astype(o.dtype)
            self.loss = float(np.sum(diff.astype(np.float64) ** 2))
        self._mask(adjoint=True)
        self.init_adj_u = [x.copy() for x in self.adj_u]
        self.init_adj_passive = self.adj_passive.copy()
        self.step_num = self.final_ind
        if self.backward_u:
            for c in range(d):
                self.init_u[c][...] = self.u[c]
            self.init_passive[...] = self.passive
        self.reset_to_identity(self.psi, self.psi_f, self.T_f)

    def march_psi_grid(self, dt):
        self.RK_grid_only_psi(self.psi, self.mid_u, dt)
        for c in range(self.dim):
            self.RK_grid(c, self.psi_f[c], self.T_f[c], self.mid_u, dt)

    def backtrack_step_midpoint(self):
        self.step_num -= 1
        n = self.step_num
        j = n % self.R
        if self.passive_on and not self.backward_u:
            self.passive[...] = self.store_passive[n + 1]
        self.backtrack_flow_map(j, self.dt)
        return n == 0

    def backtrack_flow_map(self, j, dt):
        o, d, dx = self.o, self.dim, self.dx
        n = self.step_num
        if self.cf is not None:  # 3D/lfm_midpoint_diff_simulator.py:423-427
            f_ctrl = self.control_force(n) if self.backward_u else None
            cen, inv_r, st = self.cf[n]
            self.cf_grads[n] = force_oracle.gaussian_force_grad(self.res, dx, cen, inv_r, st, self.adj_u)
        for c in range(d):
            self.mid_u[c][...] = self.store_mid[n][c]
        if self.nu:  # 2D/vortex/lfm_midpoint_diff_simulator.py:270-271
            self.vis = viscous_force(self.mid_u, self.nu, dx)
            self.adj_viscous += sum(float(np.sum((self.adj_u[c] * self.vis[c] / self.nu).astype(np.float64)))
                                    for c in range(d))
        o.calculate_nabla_u_w(self.u if self.backward_u else self.mid_u, self.adj_u, self.src, dx)
        if self.passive_on:
            o.calculate_nabla_scalar_adjoint(self.passive, self.adj_passive, self.adj_passive_f, dx)
        if self.short:  # 3D/lfm_midpoint_diff_simulator.py:440-485
            self.short_maps(self.mid_u, -dt, self.passive_on)
            maps = (self.T_tem, self.psi_f_tem, self.F_tem, self.phi_f_tem)
            self.BFECC(self.adj_u, self.final_u, self.err_u, self.tmp_u, *maps)
            for c in range(d):
                self.adj_u[c][...] = self.final_u[c] + (-2 * dt) * self.src[c]
            if self.passive_on:
                self.BFECC_scalar(self.adj_passive, self.final_passive, self.err_passive, self.tmp_passive,
                                  self.psi_tem, self.phi_tem)
                self.adj_passive[...] = self.final_passive
                for c in range(d):
                    self.adj_u[c][...] = self.adj_u[c] + (-dt) * self.adj_passive_f[c]
            if self.backward_u:
                if self.passive_on:
                    self.BFECC_scalar(self.passive, self.final_passive, self.err_passive, self.tmp_passive,
                                      self.psi_tem, self.phi_tem)
                    self.passive[...] = self.final_passive
                self.BFECC(self.u, self.final_u, self.err_u, self.tmp_u, *maps)
                for c in range(d):
                    self.u[c][...] = self.final_u[c]
        else:
            o.advect_u_grid(self.rk, self.mid_u, self.adj_u, self.final_u, dx, -dt)
            for c in range(d):
                self.adj_u[c][...] = self.final_u[c]
            if self.backward_u:
                if self.passive_on:
                    o.advect_scalar_grid(self.rk, self.mid_u, self.passive, self.final_passive, dx, -dt)
                    self.passive[...] = self.final_passive
                o.advect_u_grid(self.rk, self.mid_u, self.u, self.final_u, dx, -dt)
                for c in range(d):
                    self.u[c][...] = self.final_u[c]
            for c in range(d):
                self.adj_u[c][...] = self.adj_u[c] + (-dt) * self.src[c]
            if self.passive_on:
                o.advect_scalar_grid(self.rk, self.mid_u, self.adj_passive, self.final_passive, dx, -dt)
                self.adj_passive[...] = self.final_passive
                for c in range(d):
                    self.adj_u[c][...] = self.adj_u[c] + (-dt) * self.adj_passive_f[c]
        self.march_psi_grid(dt)
        interval_last = min((n // self.R) * self.R + self.R - 1, self.total_steps - 1)
        ind = interval_last - n
        o.accumulate_init_new(self.src, self.init_adj_u, self.T_f, self.psi_f, self.H_prev, self.H_prev_prev, ind,
                              dx, -2 * dt)
        if self.passive_on:
            o.accumulate_init(self.adj_passive_f, self.init_adj_u, self.T_f, self.psi_f, dx, -dt)
        if self.nu:  # 2D/vortex/lfm_midpoint_diff_simulator.py:387-389
            for c in range(d):
                self.adj_u[c][...] = self.adj_u[c] + (-dt) * self.vis[c]
            o.accumulate_init(self.vis, self.init_adj_u, self.T_f, self.psi_f, dx, -dt)
        self.Poisson(self.adj_u)
        if self.backward_u:
            if self.cf is not None:  # 3D/lfm_midpoint_diff_simulator.py:525-530
                for c in range(d):
                    self.u[c][...] = self.u[c] + (-dt) * f_ctrl[c]
                o.accumulate_init(f_ctrl, self.init_u, self.T_f, self.psi_f, dx, -dt)
            if self.nu:  # 2D/vortex/lfm_midpoint_diff_simulator.py:399-401
                for c in range(d):
                    self.u[c][...] = self.u[c] + (-dt) * self.vis[c]
                o.accumulate_init(self.vis, self.init_u, self.T_f, self.psi_f, dx, -dt)
            self.Poisson(self.u)
        self._mask(adjoint=True)
        if j == 0:
            phi, phi_f, F_f = self.store_maps[n // self.R]
            self.phi[...] = phi
            for c in range(d):
                self.phi_f[c][...] = phi_f[c]
                self.F_f[c][...] = F_f[c]
            self.BFECC(self.init_adj_u, self.adj_u, self.err_u, self.tmp_u, self.F_f, self.phi_f, self.T_f,
                       self.psi_f)
            self.Poisson(self.adj_u)
            for c in range(d):
                self.init_adj_u[c][...] = self.adj_u[c]
            if self.backward_u:
                self.BFECC(self.init_u, self.u, self.err_u, self.tmp_u, self.F_f, self.phi_f, self.T_f, self.psi_f)
                self.Poisson(self.u)
                for c in range(d):
                    self.init_u[c][...] = self.u[c]
            self._mask(adjoint=True)
            if self.passive_on:
                if self.trajectory_loss or not self.backward_u:
                    self.passive[...] = self.store_passive[n]
                else:
                    self.BFECC_scalar(self.init_passive, self.passive, self.err_passive, self.tmp_passive, self.phi,
                                      self.psi)
                self.init_passive[...] = self.passive
                self.BFECC_scalar(self.init_adj_passive, self.adj_passive, self.err_passive, self.tmp_passive,
                                  self.phi, self.psi)
                self.init_adj_passive[...] = self.adj_passive
            self.reset_to_identity(self.psi, self.psi_f, self.T_f)

    def gradient(self, u0, passive0, target):
        self.init(u0, passive0)
        while not self.step_midpoint():
            pass
        self.init_gradient(target)
        while not self.backtrack_step_midpoint():
            pass
        return self.loss, [x.copy() for x in self.adj_u]

    def gradient_vorticity(self, u0, omega_target):
        """2D final-vorticity loss L = sum (omega - omega*)^2 (vortex_oracle.py)."""
        import vortex_oracle as V

        self.init(u0, np.zeros(self.res))
        while not self.step_midpoint():
            pass
        om = V.vorticity(self.u[0], self.u[1], self.dx)
        diff = om.astype(np.float64) - np.asarray(omega_target, np.float64)
        g = (2 * diff).astype(self.o.dtype)
        adj = [x.astype(self.o.dtype) for x in V.vorticity_adjoint(g, self.dx)]
        self.init_gradient(seed=(float(np.sum(diff * diff)), adj))
        while not self.backtrack_step_midpoint():
            pass
        return self.loss, [x.copy() for x in self.adj_u]
