"""2D vortex optimisation gradient: theta -> u0 -> forward -> final-vorticity
loss -> adjoint -> dL/dtheta.

Mirrors the reference's vortex driver (2D/vortex/optimize_vortex.py:16-50,
193-230): the control is a set of K point vortices (strength w_k, centre c_k),
mapped to the initial velocity by sixteen_vortex_vel_func_with_pos_coef /
four_vortex_vel_func_with_coef + split_central_vector + Poisson
(2D/vortex/lfm_midpoint_simulator.py:409-419); dL/dtheta contracts the adjoint
velocity at t = 0 with d u0 / d theta (calculate_dtheta_ind, which the
reference evaluates by forward differences of the init map, epsilon 1e-5; here
the derivative is analytic).  The loss is L = sum (omega - omega*)^2 over the
cells of the final vorticity (the reference's vortex loss is on three passive
scalars; the vorticity loss follows the benchmark definition).
theta = [w_0..w_{K-1}, cx_0..cx_{K-1}, cy_0..cy_{K-1}].
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch

from . import kernels as K
from .simulator import LFM_Diff_Simulator


class VortexProblem:
    """Owns a 2D simulator and evaluates the vortex-parameter gradient."""

    def __init__(self, sim: LFM_Diff_Simulator):
        if sim.dim != 2:
            raise ValueError("VortexProblem needs a 2D simulator")
        self.sim = sim
        self.grid = sim.grid
        self.dx = sim.dx
        self.dtype = sim.cfg.dtype
        self.device = sim.device
        self.loss = None

    def velocity(self, theta: Sequence[float]):
        """Face velocity of theta before projection (split_central_vector of the centre values)."""
        g = self.grid
        u = [torch.empty(g.face_shape(c), dtype=self.dtype, device=self.device) for c in range(2)]
        K.vortex_velocity_2d(g, self.dx, theta, u[0], u[1])
        return u

    def run_forward(self, theta):
        sim = self.sim
        sim.init(theta=self.velocity(theta))
        while not sim.forward_step_midpoint()[1]:
            pass

    def final_vorticity(self, theta) -> torch.Tensor:
        """omega at the final frame of the simulation started from theta (the target builder)."""
        self.run_forward(theta)
        om = torch.empty(self.grid.shape, dtype=self.dtype, device=self.device)
        K.vorticity_2d(self.grid, self.dx, self.sim.u[0], self.sim.u[1], om)
        return om

    def calculate_dtheta(self, theta) -> np.ndarray:
        """dL/dtheta from the simulator's adjoint velocity at t = 0 (after backtracking)."""
        adj = self.sim.adj_u
        return K.vortex_velocity_grad_2d(self.grid, self.dx, theta, adj[0], adj[1]).cpu().numpy()

    def gradient(self, theta, omega_target: torch.Tensor):
        """(L, dL/dtheta) for L = sum (omega(T) - omega*)^2."""
        loss, _ = self.sim.gradient(self.velocity(theta), target_vorticity=omega_target)
        self.loss = loss
        return loss, self.calculate_dtheta(theta)

    # ---- the same gradient replayed from one CUDA graph
    def capture(self, theta, omega_target: torch.Tensor):
        """Record the gradient as one CUDA graph (LFM_Diff_Simulator.capture_gradient)
        with u0(theta) and omega_target as its inputs; graph_gradient then
        evaluates any theta with the same number of vortices in one graph launch."""
        self._u0 = self.velocity(theta)
        self._omega_target = omega_target
        self.graph = self.sim.capture_gradient(self._u0, target_vorticity=omega_target)
        return self.graph

    def prepare_record(self, theta, omega_target: torch.Tensor):
        """First half of recording this gradient into a graph shared with other
        problems (BatchedVortex.capture(single_graph=True)): the graph's input
        tensor and one eager gradient."""
        self._u0 = self.velocity(theta)
        self._omega_target = omega_target
        self.sim.prepare_capture(self._u0, target_vorticity=omega_target)

    def record(self):
        """Second half: record the gradient on the current (capturing) stream;
        returns (roles, loss tensor, kernels) for the shared graph's replay."""
        return self.sim.record_gradient(self._u0, target_vorticity=self._omega_target)

    def launch_gradient(self, theta):
        """The asynchronous part of graph_gradient: u0(theta) into the graph's
        input and one graph launch, on the current stream."""
        if getattr(self, "graph", None) is None:
            raise RuntimeError("launch_gradient: call capture() first")
        K.vortex_velocity_2d(self.grid, self.dx, theta, self._u0[0], self._u0[1])
        self.graph.replay()

    def finish_gradient(self, theta):
        """(L, dL/dtheta) of the last launch_gradient (synchronises the stream)."""
        self.loss = self.graph.loss()
        return self.loss, self.calculate_dtheta(theta)

    def graph_gradient(self, theta):
        self.launch_gradient(theta)
        return self.finish_gradient(theta)
