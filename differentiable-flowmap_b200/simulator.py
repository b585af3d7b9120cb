"""Leapfrog flow-map simulator and its adjoint, driving libflowmap_sm100.so.

``LFM_Simulator`` mirrors 3D/lfm_midpoint_simulator.py:167-807 (and the 2D
copies, 2D/vortex/lfm_midpoint_simulator.py:186-661): ``init``,
``step_midpoint`` -> ``step_flow_map``, ``backtrack_psi_grid``,
``march_phi_grid``.  ``LFM_Diff_Simulator`` mirrors
3D/lfm_midpoint_diff_simulator.py:15-594: ``forward_step_midpoint``,
``init_gradient``, ``backtrack_step_midpoint`` -> ``backtrack_flow_map``.

Differences from the reference, all on the plumbing side:
  * the trajectory the adjoint needs (every step's midpoint velocity, the
    flow maps phi/F at every reinit, optionally every step's passive scalar)
    stays resident in HBM instead of being written to .npy files by RW_Cache;
    the in-interval midpoint velocities that backtrack_psi_grid replays are the
    same device buffers (the reference copies them through a host dict);
  * copy_to/add_fields/scale_field chains are fused into the kernels'
    epilogues (BFECC is three launches) and result buffers are rotated instead
    of copied;
  * calc_max_speed only feeds a print in the reference and is not computed.

Control flow and arithmetic follow the reference step for step; the flags of
3D/hyperparameters.py are fields of ``FlowmapConfig``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from . import kernels as K
from ._lib import FlowmapError
from .kernels import GridSpec
from .mgpcg import MGPCG, SolidMGPCG


@dataclass
class SolverConfig:
    """MGPCG parameters (3D/mgpcg.py:22-35, :429-431)."""

    base_level: int = 3
    levels: Optional[int] = None
    pre_post: int = 2
    bottom: int = 50
    bottom_mode: int = 0
    max_iters: int = 400
    abs_tol: float = 1e-12
    rel_tol: float = 0.0
    eps: float = 1e-12
    check_every: int = 4
    coarse_bf16: bool = False  # FP32 solvers: per-level coarse grids stored in BF16 (arithmetic FP32)
    # FP32 solvers: FP64 outer defect correction in every projection until the FP64
    # residual is below dc_rel_tol |b| (0: off), at most dc_max_outer corrections
    dc_rel_tol: float = 0.0
    dc_max_outer: int = 4


@dataclass
class FlowmapConfig:
    """Simulation flags (names follow 3D/hyperparameters.py)."""

    res: tuple = (128, 128, 128)
    dx: float = 1.0 / 128
    dt: float = 0.0085            # act_dt
    total_steps: int = 150
    reinit_every: int = 8
    RK_number: int = 4
    backward_u: bool = True       # adjoint re-advects u backwards (reference default)
    add_passive_scalar: bool = True
    BFECC_clamp: bool = False
    use_short_BFECC: bool = False
    add_control_force: bool = False  # Gaussian control forces (control_force_para per step)
    control_num: int = 0             # capacity: most Gaussians one step may pass
    store_control_force: bool = True  # adjoint with backward_u reads the forward's force fields from HBM
    viscosity: float = 0.0           # 2D viscous term (2D/vortex/hyperparameters.py:26)
    boundary_mask: Optional[object] = None  # obstacle mask on the cell grid (solid > 0), numpy or tensor
    boundary_vel: Optional[object] = None   # (dim, *grid) velocity of the solid cells (None: 0)
    trajectory_loss: bool = False  # reference's no-force branch: loss over reinit frames
    dtype: torch.dtype = torch.float32
    store_dtype: Optional[torch.dtype] = None  # checkpoint storage dtype (None: dtype)
    # Interval checkpointing: the forward keeps only (u, passive) at the start of
    # each reinit interval, and the adjoint recomputes each interval's forward
    # steps before undoing them (about 7x less trajectory memory at 128^3, one
    # more forward pass of time).  Needs backward_u=False.
    recompute: bool = False
    # storage dtype of the interval checkpoints (None: the working dtype); BF16
    # halves them, and the replay then starts from the rounded state
    ckpt_dtype: Optional[torch.dtype] = None
    # velocity checkpoints in BF16 as differences from the previous checkpoint's
    # reconstruction (the first one in the working dtype): the rounding then applies
    # to one interval's change of u, not to u itself, and never accumulates (each
    # difference is taken against the reconstruction the replay will rebuild).
    # The passive-scalar checkpoints stay in the working dtype.  Needs recompute
    # and an FP32 working dtype.
    ckpt_delta: bool = False
    solver: SolverConfig = field(default_factory=SolverConfig)

    def validate(self):
        """Reject option combinations the simulator does not implement."""
        if self.recompute:
            bad = [name for name, on in (("backward_u", self.backward_u), ("add_control_force", self.add_control_force),
                                         ("viscosity", self.viscosity != 0.0), ("use_short_BFECC", self.use_short_BFECC),
                                         ("trajectory_loss", self.trajectory_loss)) if on]
            if bad:
                raise FlowmapError(2, f"recompute (interval checkpointing) does not support {', '.join(bad)}")
        if self.ckpt_delta and (not self.recompute or self.dtype != torch.float32):
            raise FlowmapError(2, "ckpt_delta needs recompute=True and an FP32 working dtype")

    @property
    def dim(self) -> int:
        return len(self.res)


class _Scalar:
    """0-d holder supporting the reference's ``field[None]`` indexing."""

    def __init__(self, v=0):
        self.v = v

    def __getitem__(self, k):
        return self.v

    def __setitem__(self, k, v):
        self.v = v


class DeviceField:
    """A device tensor read back like a Taichi field (``.to_numpy()``)."""

    def __init__(self, t: torch.Tensor):
        self.tensor = t

    def to_numpy(self):
        return self.tensor.cpu().numpy()


class _GaussianParams:
    """Device copies of one step's Gaussian parameters (center n x dim, inverse
    radius n, strength n x dim), uploaded from host arrays through two pinned
    staging buffers so that an upload never waits for the GPU: a buffer is
    rewritten only after the copy that last read it has completed."""

    def __init__(self, cap: int, dim: int, dtype, device):
        self.cap, self.dim, self.dtype = cap, dim, dtype
        self.per = 2 * dim + 1
        self.dev = torch.empty(max(cap, 1) * self.per, dtype=dtype, device=device)
        self.host = [torch.empty(max(cap, 1) * self.per, dtype=dtype).pin_memory() for _ in range(2)]
        self.events = [None, None]
        self.k = 0

    def load(self, para):
        n = int(para["n"])
        if n < 0 or n > self.cap:
            raise FlowmapError(8, f"{n} Gaussians exceed control_num={self.cap}")
        c, r, st = para["c"], para["r"], para["s"]
        dim = self.dim
        if all(isinstance(x, torch.Tensor) and x.is_cuda for x in (c, r, st)):
            return (c[:n].to(self.dtype).contiguous(), r[:n].to(self.dtype).contiguous(),
                    st[:n].to(self.dtype).contiguous())
        h = self.host[self.k]
        if self.events[self.k] is not None:
            self.events[self.k].synchronize()
        for off, x, cnt in ((0, c, n * dim), (n * dim, r, n), (n * dim + n, st, n * dim)):
            a = x.detach().cpu() if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x))
            h[off:off + cnt].copy_(a.reshape(-1)[:cnt])
        m = n * self.per
        self.dev[:m].copy_(h[:m], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        self.events[self.k] = ev
        self.k ^= 1
        return (self.dev[:n * dim].view(n, dim), self.dev[n * dim:n * dim + n],
                self.dev[n * dim + n:m].view(n, dim))


def _mac(grid: GridSpec, dtype, device, fill=0.0):
    return [torch.full(grid.face_shape(c), fill, dtype=dtype, device=device) for c in range(grid.dim)]


def _vec_face(grid: GridSpec, dtype, device):
    return [torch.zeros((grid.dim,) + grid.face_shape(c), dtype=dtype, device=device) for c in range(grid.dim)]


def _copy_mac(dst, src):
    for d, s in zip(dst, src):
        d.copy_(s)


def _as_tensor(x):
    """numpy array or (pinned host / device) tensor -> tensor for copy_()."""
    return x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x))


class LFM_Simulator:
    """Forward leapfrog flow-map simulator (3D/lfm_midpoint_simulator.py:167)."""

    def __init__(self, res_x=None, res_y=None, res_z=None, dx=None, dt=None, reinit_every=None, log_dir=None,
                 log_target_dir=None, *, config: Optional[FlowmapConfig] = None, device="cuda"):
        cfg = config if config is not None else FlowmapConfig()
        if res_x is not None:
            res = (res_x, res_y) if res_z is None else (res_x, res_y, res_z)
            cfg = replace(cfg, res=tuple(res))
        if dx is not None:
            cfg = replace(cfg, dx=dx)
        if dt is not None:
            cfg = replace(cfg, dt=dt)
        if reinit_every is not None:
            cfg = replace(cfg, reinit_every=reinit_every)
        cfg.validate()
        if not torch.cuda.is_available():
            raise FlowmapError(6, "LFM_Simulator needs a CUDA device (no CPU fallback)")
        self.cfg = cfg
        self.device = torch.device(device)
        self.grid = GridSpec(tuple(cfg.res))
        self.dim = self.grid.dim
        self.dx = cfg.dx
        self.dt = cfg.dt
        self.reinit_every = cfg.reinit_every
        self.res_x, self.res_y = cfg.res[0], cfg.res[1]
        self.res_z = cfg.res[2] if self.dim == 3 else 1
        self.log_dir = log_dir
        self.log_target_dir = log_target_dir
        dt_, dev, g = cfg.dtype, self.device, self.grid
        self.store_dtype = cfg.store_dtype or cfg.dtype

        sc = cfg.solver
        # obstacles: a non-empty mask selects the solid-aware solver and the mask kernels
        self.boundary_mask = self.boundary_vel = None
        if cfg.boundary_mask is not None and bool((torch.as_tensor(cfg.boundary_mask) > 0).any()):
            self.boundary_mask = torch.as_tensor(cfg.boundary_mask).to(dev, torch.float32).contiguous()
            if tuple(self.boundary_mask.shape) != tuple(g.shape):
                raise FlowmapError(1, f"boundary_mask shape {tuple(self.boundary_mask.shape)} != grid {g.shape}")
            if cfg.boundary_vel is not None:
                self.boundary_vel = torch.as_tensor(cfg.boundary_vel).to(dev, dt_).contiguous()
            self.solver = SolidMGPCG(g.shape, self.boundary_mask, dt_, base_level=sc.base_level, levels=sc.levels,
                                     pre_post=sc.pre_post, bottom=sc.bottom, bottom_mode=sc.bottom_mode,
                                     max_iters=sc.max_iters, abs_tol=sc.abs_tol, rel_tol=sc.rel_tol, eps=sc.eps,
                                     check_every=sc.check_every)
        else:
            self.solver = MGPCG(g.shape, dt_, base_level=sc.base_level, levels=sc.levels, pre_post=sc.pre_post,
                                bottom=sc.bottom, bottom_mode=sc.bottom_mode, max_iters=sc.max_iters,
                                abs_tol=sc.abs_tol, rel_tol=sc.rel_tol, eps=sc.eps, check_every=sc.check_every,
                                coarse_bf16=sc.coarse_bf16 and dt_ == torch.float32,
                                dc_rel_tol=sc.dc_rel_tol if dt_ == torch.float32 else 0.0,
                                dc_max_outer=sc.dc_max_outer)

        # flow maps: backward (psi, T) and forward (phi, F); centre maps for scalars
        self.psi = torch.zeros((self.dim,) + g.shape, dtype=dt_, device=dev)
        self.phi = torch.zeros((self.dim,) + g.shape, dtype=dt_, device=dev)
        self.psi_f = _vec_face(g, dt_, dev)
        self.T_f = _vec_face(g, dt_, dev)
        self.phi_f = _vec_face(g, dt_, dev)
        self.F_f = _vec_face(g, dt_, dev)

        self.u = _mac(g, dt_, dev)
        self.ad_u = _mac(g, dt_, dev)
        self.final_u = _mac(g, dt_, dev)
        self.init_u = _mac(g, dt_, dev)
        self.err_u = _mac(g, dt_, dev)

        self.passive = torch.zeros(g.shape, dtype=dt_, device=dev)
        self.final_passive = torch.zeros_like(self.passive)
        self.init_passive = torch.zeros_like(self.passive)
        self.err_passive = torch.zeros_like(self.passive)

        # BFECC clamp (tmp fields) and short BFECC (one-step temporary maps)
        if cfg.BFECC_clamp:
            self.tmp_u = _mac(g, dt_, dev)
            self.tmp_passive = torch.zeros_like(self.passive)
        if cfg.use_short_BFECC:
            self.psi_tem = torch.zeros((self.dim,) + g.shape, dtype=dt_, device=dev)
            self.phi_tem = torch.zeros((self.dim,) + g.shape, dtype=dt_, device=dev)
            self.psi_f_tem, self.T_f_tem = _vec_face(g, dt_, dev), _vec_face(g, dt_, dev)
            self.phi_f_tem, self.F_f_tem = _vec_face(g, dt_, dev), _vec_face(g, dt_, dev)

        # Gaussian control forces: the force field and the parameter staging
        self.control_force = None
        if cfg.add_control_force:
            if cfg.control_num < 0:
                raise FlowmapError(2, "control_num must be >= 0")
            self.control_force = _mac(g, dt_, dev)
            self._gf = _GaussianParams(cfg.control_num, self.dim, dt_, dev)

        # 2D viscous term: the field nu * Laplacian(u) of the step's midpoint velocity
        self.vis = None
        if cfg.viscosity != 0.0:
            if self.dim != 2:
                raise FlowmapError(2, "the viscous term exists in the 2D reference only")
            self.vis = _mac(g, dt_, dev)
            self._vis_part = torch.empty(592, dtype=torch.float64, device=dev)

        self.step_num = _Scalar(-1)
        self.frame_idx = _Scalar(0)
        self.total_steps = cfg.total_steps
        self._recomputing = False
        self._replay_tail = False
        self._replayed = None  # interval whose replay state the last forward pass left in place
        self._alloc_stores()
        self.reset_to_identity(self.phi, self.phi_f, self.F_f)

    # ------------------------------------------------------------ stores
    def _alloc_stores(self):
        """Device-resident trajectory for the adjoint (replaces RW_Cache disk I/O).
        Full form: every step's midpoint velocity, the passive scalar of every
        step and the forward maps at every interval end.  Interval checkpointing
        (recompute): (u, passive) at the start of every interval plus the final
        state, and one interval's midpoint velocities and passives, regenerated
        by the adjoint."""
        g, steps, dev = self.grid, self.total_steps, self.device
        R = self.reinit_every
        n_int = (steps + R - 1) // R
        sd, wd = self.store_dtype, self.cfg.dtype
        self.store_mid = self.store_phi = self.store_phi_f = self.store_F_f = self.store_passive = None
        self.ckpt_u = self.ckpt_passive = self._ring_passive = None
        self._ckpt_u0 = self._ckpt_base = self._ckpt_tmp = None
        if self.cfg.recompute:
            delta = self.cfg.ckpt_delta
            cd = torch.bfloat16 if delta else (self.cfg.ckpt_dtype or wd)
            self.ckpt_u = [torch.zeros((n_int + 1,) + g.face_shape(c), dtype=cd, device=dev) for c in range(self.dim)]
            if delta:  # checkpoint 0 in full, the running reconstruction, a difference buffer
                self._ckpt_u0, self._ckpt_base, self._ckpt_tmp = (
                    [torch.zeros(g.face_shape(c), dtype=wd, device=dev) for c in range(self.dim)] for _ in range(3))
            if self.cfg.add_passive_scalar:
                self.ckpt_passive = torch.zeros((n_int + 1,) + g.shape, dtype=wd if delta else cd, device=dev)
                self._ring_passive = torch.zeros((R + 1,) + g.shape, dtype=wd, device=dev)
            self._ring = [[torch.zeros(g.face_shape(c), dtype=wd, device=dev) for c in range(self.dim)]
                          for _ in range(R)]
            return
        self.store_mid = [torch.zeros((steps,) + g.face_shape(c), dtype=sd, device=dev) for c in range(self.dim)]
        # flow maps (positions and Jacobians) stay in the working dtype: a BF16
        # position would be ~0.5 cells off at 128^3
        self.store_phi = torch.zeros((n_int, self.dim) + g.shape, dtype=wd, device=dev)
        self.store_phi_f = [torch.zeros((n_int, self.dim) + g.face_shape(c), dtype=wd, device=dev)
                            for c in range(self.dim)]
        self.store_F_f = [torch.zeros((n_int, self.dim) + g.face_shape(c), dtype=wd, device=dev)
                          for c in range(self.dim)]
        need_passive = self.cfg.add_passive_scalar and (not self.cfg.backward_u or self.cfg.trajectory_loss)
        # the passive scalar feeds the adjoint source (nabla_scalar_adjoint) directly: stored in BF16 it
        # raised the 64^3 gradient error from 4e-5 to 1.8e-4, so it stays in the working dtype
        self.store_passive = (torch.zeros((steps + 1,) + g.shape, dtype=wd, device=dev) if need_passive else None)
        # in-interval midpoint velocities replayed by backtrack_psi_grid, in the working dtype
        if sd == self.cfg.dtype:
            self._ring = None
        else:
            self._ring = [[torch.zeros(g.face_shape(c), dtype=self.cfg.dtype, device=dev) for c in range(self.dim)]
                          for _ in range(R)]

    def trajectory_bytes(self) -> int:
        """Device bytes held for the adjoint (stores, checkpoints, rings)."""
        ts = []
        for x in (self.store_mid, self.store_phi_f, self.store_F_f, self.ckpt_u, self._ring, self._ckpt_u0,
                  self._ckpt_base, self._ckpt_tmp):
            if x is not None:
                ts += [t for row in x for t in (row if isinstance(row, list) else [row])]
        ts += [x for x in (self.store_phi, self.store_passive, self.ckpt_passive, self._ring_passive)
               if x is not None]
        return sum(t.numel() * t.element_size() for t in ts)

    def _checkpoint(self, k: int):
        """Interval checkpointing: the state at the start of interval k (slot
        n_int: the state after the last step)."""
        if self.cfg.ckpt_delta:
            for c in range(self.dim):
                if k == 0:
                    self._ckpt_u0[c].copy_(self.u[c])
                    self._ckpt_base[c].copy_(self.u[c])
                    continue
                # d = u - base rounded to BF16; base += d as the replay will add it
                K.add_fields(self.u[c], self._ckpt_base[c], self._ckpt_tmp[c], -1.0)
                K.store(self._ckpt_tmp[c], self.ckpt_u[c][k])
                K.store(self.ckpt_u[c][k], self._ckpt_tmp[c])
                K.add_fields(self._ckpt_base[c], self._ckpt_tmp[c], self._ckpt_base[c], 1.0)
        else:
            for c in range(self.dim):
                K.store(self.u[c], self.ckpt_u[c][k])
        if self.ckpt_passive is not None:
            K.store(self.passive, self.ckpt_passive[k])

    def _load_ckpt_u(self, k: int):
        """u = the velocity checkpoint k (rebuilt from the differences in the delta
        form, with the forward's operations in its order)."""
        for c in range(self.dim):
            if not self.cfg.ckpt_delta:
                K.store(self.ckpt_u[c][k], self.u[c])
                continue
            self.u[c].copy_(self._ckpt_u0[c])
            for j in range(1, k + 1):
                K.store(self.ckpt_u[c][j], self._ckpt_tmp[c])
                K.add_fields(self.u[c], self._ckpt_tmp[c], self.u[c], 1.0)

    # ------------------------------------------------------------ kernels
    def reset_to_identity(self, psi, psi_f, T_f):
        K.reset_to_identity(self.grid, self.dx, psi, psi_f, T_f)

    def _advect_u_grid(self, u0, u1, u2, dt):
        K.advect_u_grid(self.grid, self.cfg.RK_number, self.dx, dt, u0, u1, u2)

    def _advect_scalar_grid(self, u0, s1, s2, dt):
        K.advect_scalar_grid(self.grid, self.cfg.RK_number, self.dx, dt, u0, s1, s2)

    def _march(self, psi_c, psi_f, T_f, u, dt):
        K.march_map(self.grid, self.cfg.RK_number, self.dx, dt, psi_c, psi_f, T_f, u)

    def BFECC(self, init_u, u, err_u, T_f, psi_f, F_f, phi_f):
        """BFECC (3D/flowmap.py:405-434) in three fused launches:
        u = T.init(psi); err = 0.5*(F.u(phi) - init); u = u - T.err(psi).
        With BFECC_clamp the last value is clamped to the extrema of the first
        pass's neighbours (clamp_u) before it replaces u."""
        g, dx = self.grid, self.dx
        K.pullback_u(g, dx, init_u, u, T_f, psi_f)
        K.pullback_u(g, dx, u, err_u, F_f, phi_f, alpha=0.5, beta=-1.0, base=init_u)
        if not self.cfg.BFECC_clamp:
            K.pullback_u(g, dx, err_u, u, T_f, psi_f, alpha=-1.0, beta=-1.0, base=u)
            return
        K.pullback_u(g, dx, err_u, self.tmp_u, T_f, psi_f, alpha=-1.0, beta=-1.0, base=u)
        for c in range(self.dim):
            K.clamp_extrema(g, self.tmp_u[c], u[c], err_u[c])
            u[c].copy_(err_u[c])

    def BFECC_scalar(self, init_s, s, err_s, psi, phi):
        """BFECC_scalar (3D/flowmap.py:436-452), clamped like BFECC with BFECC_clamp."""
        g, dx = self.grid, self.dx
        K.pullback_scalar(g, dx, init_s, s, psi)
        K.pullback_scalar(g, dx, s, err_s, phi, alpha=0.5, beta=-1.0, base=init_s)
        if not self.cfg.BFECC_clamp:
            K.pullback_scalar(g, dx, err_s, s, psi, alpha=-1.0, beta=-1.0, base=s)
            return
        K.pullback_scalar(g, dx, err_s, self.tmp_passive, psi, alpha=-1.0, beta=-1.0, base=s)
        K.clamp_extrema(g, self.tmp_passive, s, err_s)
        s.copy_(err_s)

    def _short_maps(self, u, dt, centre: bool):
        """One-step temporary maps of use_short_BFECC: psi_tem with dt, phi_tem
        with -dt, from identity (3D/lfm_midpoint_simulator.py:725-739)."""
        self.reset_to_identity(self.psi_tem, self.psi_f_tem, self.T_f_tem)
        self.reset_to_identity(self.phi_tem, self.phi_f_tem, self.F_f_tem)
        self._march(self.psi_tem if centre else None, self.psi_f_tem, self.T_f_tem, u, dt)
        self._march(self.phi_tem if centre else None, self.phi_f_tem, self.F_f_tem, u, -dt)

    def project(self, u):
        self.solver.project(u)

    def _mask(self, adjoint: bool = False):
        """mask_velocity_by_boundary / mask_passive_by_boundary and, in the adjoint,
        their adjoint forms (3D/init_conditions.py:536-578), after a projection."""
        if self.boundary_mask is None:
            return
        g, m = self.grid, self.boundary_mask
        K.mask_velocity(g, m, self.u, self.boundary_vel)
        if adjoint:
            K.mask_velocity(g, m, self.adj_u)
        if self.cfg.add_passive_scalar:
            K.mask_passive(g, m, self.passive)
            if adjoint:
                K.mask_passive(g, m, self.adj_passive, adjoint=True)

    # ------------------------------------------------------------ API
    @property
    def u_x(self):
        return self.u[0]

    @property
    def u_y(self):
        return self.u[1]

    @property
    def u_z(self):
        return self.u[2] if self.dim == 3 else None

    def init(self, theta=None, forward=True, target=False, init_passive_np=None):
        """Case-11 initialisation (3D/lfm_midpoint_simulator.py:592-615): u from
        ``theta`` (dict with u_x/u_y[/u_z] or a sequence of face arrays; zeros if
        None), projected; passive from ``init_passive_np``; phi, F reset."""
        if not forward:
            return
        for c in range(self.dim):
            self.u[c].zero_()
        if theta is not None:
            comps = ([theta[k] for k in ("u_x", "u_y", "u_z")[: self.dim]] if isinstance(theta, dict) else list(theta))
            for c in range(self.dim):
                self.u[c].copy_(_as_tensor(comps[c]), non_blocking=True)
        self.project(self.u)
        if self.cfg.add_passive_scalar and init_passive_np is not None:
            self.passive.copy_(_as_tensor(init_passive_np), non_blocking=True)
            self.init_passive.copy_(self.passive)
        self._mask()  # 3D/lfm_midpoint_simulator.py:606-608
        self.step_num[None] = -1
        self.frame_idx[None] = 0
        self.reset_to_identity(self.phi, self.phi_f, self.F_f)
        _copy_mac(self.init_u, self.u)

    def final_condition(self):
        return self.step_num[None] == self.total_steps - 1

    def apply_gausion_force(self, f, center, inverse_radius, strength, num):
        """3D/lfm_midpoint_simulator.py:309-314: f = the Gaussians' force field."""
        c, r, st = self._gf.load({"c": center, "r": inverse_radius, "s": strength, "n": num})
        K.gaussian_force(self.grid, self.dx, c, r, st, f)

    def _force_field(self, n):
        """Where step n's control force is written: its slot of the trajectory
        store when the adjoint will read it back, else the scratch field."""
        st = getattr(self, "store_force", None)
        return [x[n] for x in st] if st is not None else self.control_force

    def _control_params(self, control_force_para):
        if control_force_para is None:
            raise FlowmapError(2, "add_control_force needs control_force_para for every step")
        return self._gf.load(control_force_para)

    def step_midpoint(self, write_flow_map=True, write_passive=True, control_force_para=None):
        """One leapfrog step (3D/lfm_midpoint_simulator.py:648-682).  With
        add_control_force, ``control_force_para`` = {"c": centers n x dim,
        "r": inverse radii n, "s": strengths n x dim, "n": n} for this step
        (numpy arrays or tensors); otherwise it is ignored, as in the reference."""
        self.step_num[None] += 1
        n = self.step_num[None]
        if n >= self.total_steps:
            raise FlowmapError(2, f"step {n} beyond total_steps={self.total_steps}")
        j = n % self.reinit_every
        R = self.reinit_every
        self._replayed = None
        # interval checkpointing with a partial last interval: the forward keeps that
        # interval's replay state (midpoint ring, passive ring, maps never reset), so
        # the adjoint's first step need not replay it
        keep_tail = (self.ckpt_u is not None and self.total_steps % R != 0
                     and n // R == (self.total_steps - 1) // R)
        if self.store_passive is not None:
            K.store(self.passive, self.store_passive[n])
        if self.ckpt_u is not None and j == 0:
            self._checkpoint(n // R)
        if keep_tail and self._ring_passive is not None:
            self._ring_passive[j].copy_(self.passive)
        self.step_flow_map(j, self.dt, control_force_para)
        if self.final_condition() and self.store_passive is not None:
            K.store(self.passive, self.store_passive[n + 1])
        if self.final_condition() and self.ckpt_u is not None:
            k_end = (self.total_steps + R - 1) // R
            self._checkpoint(k_end)
            if keep_tail:
                if self._ring_passive is not None:  # as the replay sets it: from the checkpoint
                    K.store(self.ckpt_passive[k_end], self._ring_passive[j + 1])
                self._replayed = n // R
        return False, self.final_condition()

    def march_phi_grid(self, u):
        """3D/lfm_midpoint_simulator.py:377-381 (one launch for centre + faces)."""
        self._march(self.phi, self.phi_f, self.F_f, u, -self.dt)

    def backtrack_psi_grid(self, curr_step: int, interval_start: int):
        """3D/lfm_midpoint_simulator.py:357-375: rebuild psi, T over the
        interval, the last sub-step with the current u (as the reference does)."""
        self.reset_to_identity(self.psi, self.psi_f, self.T_f)
        self._march(self.psi, self.psi_f, self.T_f, self.u, self.dt)
        for s in reversed(range(curr_step)):
            if self._ring is not None:
                um = self._ring[s]
            else:
                um = [m[interval_start + s] for m in self.store_mid]
            self._march(self.psi, self.psi_f, self.T_f, um, self.dt)

    def step_flow_map(self, j: int, curr_dt: float, control_force_para=None):
        """3D/lfm_midpoint_simulator.py:684-807; use_short_BFECC, BFECC_clamp,
        add_control_force and the 2D viscous term (2D/vortex/lfm_midpoint_simulator.py:
        552, 607-609) as configured.  The control force is
        evaluated once per step: the reference evaluates it twice with the same
        parameters, which gives the same field."""
        cfg = self.cfg
        n = self.step_num[None]
        _copy_mac(self.ad_u, self.u)
        self._advect_u_grid(self.ad_u, self.ad_u, self.u, 0.5 * curr_dt)
        if cfg.add_control_force:  # 3D/lfm_midpoint_simulator.py:694-706
            force = self._force_field(n)
            K.gaussian_force(self.grid, self.dx, *self._control_params(control_force_para), force)
            for c in range(self.dim):
                K.add_fields(self.u[c], force[c], self.u[c], 0.5 * curr_dt)
        self.project(self.u)
        self._mask()  # 3D/lfm_midpoint_simulator.py:712-714
        if self.vis is not None:  # 2D/vortex/lfm_midpoint_simulator.py:552
            K.viscous_force_2d(self.grid, cfg.viscosity, self.dx, self.u, self.vis)
        # write_velocity + RW_Cache("u"): the midpoint velocity of step n
        for c in range(self.dim):
            if self.store_mid is not None:
                K.store(self.u[c], self.store_mid[c][n])
            if self._ring is not None:
                self._ring[j][c].copy_(self.u[c])
        self.march_phi_grid(self.u)
        if self._recomputing and self._replay_tail:
            # the last step of a replayed interval: the adjoint needs its midpoint
            # velocity and the interval-end maps, not the end state (the next
            # checkpoint holds it)
            return
        if cfg.use_short_BFECC:
            # BFECC through one-step maps instead of the semi-Lagrangian advection
            # (3D/lfm_midpoint_simulator.py:725-745); the BFECC result replaces u
            self._short_maps(self.u, curr_dt, cfg.add_passive_scalar)
            if cfg.add_passive_scalar:
                self.BFECC_scalar(self.passive, self.final_passive, self.err_passive, self.psi_tem, self.phi_tem)
                self.passive, self.final_passive = self.final_passive, self.passive
            self.BFECC(self.ad_u, self.u, self.err_u, self.T_f_tem, self.psi_f_tem, self.F_f_tem, self.phi_f_tem)
        else:
            if cfg.add_passive_scalar:
                self._advect_scalar_grid(self.u, self.passive, self.final_passive, curr_dt)
                self.passive, self.final_passive = self.final_passive, self.passive
            self._advect_u_grid(self.u, self.ad_u, self.final_u, curr_dt)
            self.u, self.final_u = self.final_u, self.u
        if cfg.add_control_force:  # 3D/lfm_midpoint_simulator.py:755-760
            for c in range(self.dim):
                K.add_fields(self.u[c], force[c], self.u[c], curr_dt)
            K.accumulate_init(self.grid, self.dx, curr_dt, force, self.init_u, self.F_f, self.phi_f)
        if self.vis is not None:  # 2D/vortex/lfm_midpoint_simulator.py:607-609
            for c in range(self.dim):
                K.add_fields(self.u[c], self.vis[c], self.u[c], curr_dt)
            K.accumulate_init(self.grid, self.dx, curr_dt, self.vis, self.init_u, self.F_f, self.phi_f)
        self.project(self.u)
        self._mask()  # 3D/lfm_midpoint_simulator.py:769-771

        if self._recomputing:
            # an interval replayed for the adjoint: it needs the midpoint
            # velocities, passives and end-of-interval maps, not the reinit
            # (the next interval's start state is its checkpoint)
            return
        if j == self.reinit_every - 1:
            self.backtrack_psi_grid(self.reinit_every - 1, n - j)
            self.BFECC(self.init_u, self.u, self.err_u, self.T_f, self.psi_f, self.F_f, self.phi_f)
            self.project(self.u)
            self._mask()  # 3D/lfm_midpoint_simulator.py:787-789
            if cfg.add_passive_scalar:
                self.BFECC_scalar(self.init_passive, self.passive, self.err_passive, self.psi, self.phi)
                self.init_passive.copy_(self.passive)
            self._store_maps(n // self.reinit_every)
            self.reset_to_identity(self.phi, self.phi_f, self.F_f)
            _copy_mac(self.init_u, self.u)
        elif n == self.total_steps - 1:
            # a final partial interval: keep its forward map for the adjoint
            self._store_maps(n // self.reinit_every)

    def _store_maps(self, k: int):
        """The forward maps at the end of interval k (the adjoint's BFECC at j == 0);
        with interval checkpointing the adjoint regenerates them instead."""
        if self.store_phi is None:
            return
        self.store_phi[k].copy_(self.phi)
        for c in range(self.dim):
            self.store_phi_f[c][k].copy_(self.phi_f[c])
            self.store_F_f[c][k].copy_(self.F_f[c])

    def _recompute_interval(self, k: int):
        """Interval checkpointing: replay the forward steps of interval k from its
        checkpoint, keeping their midpoint velocities (ring) and passives
        (passive ring, the interval end from checkpoint k+1), and leaving the
        interval-end forward maps in phi, phi_f, F_f.  The replay runs the same
        kernels on the same inputs as the forward, so every value equals the
        forward's.  Only the forward's buffers are touched (with backward_u=False
        the adjoint keeps none of its state in them)."""
        R = self.reinit_every
        n0 = k * R
        last = min(n0 + R - 1, self.total_steps - 1)
        saved = self.step_num[None]
        self._load_ckpt_u(k)
        if self.ckpt_passive is not None:
            K.store(self.ckpt_passive[k], self.passive)
            self.init_passive.copy_(self.passive)
        _copy_mac(self.init_u, self.u)
        self.reset_to_identity(self.phi, self.phi_f, self.F_f)
        self._recomputing = True
        try:
            for n in range(n0, last + 1):
                self.step_num[None] = n
                if self._ring_passive is not None:
                    self._ring_passive[n - n0].copy_(self.passive)
                self._replay_tail = n == last
                self.step_flow_map(n - n0, self.dt)
        finally:
            self._recomputing = False
            self._replay_tail = False
            self.step_num[None] = saved
        if self._ring_passive is not None:
            K.store(self.ckpt_passive[k + 1], self._ring_passive[last + 1 - n0])


class LFM_Diff_Simulator(LFM_Simulator):
    """Adjoint simulator (3D/lfm_midpoint_diff_simulator.py:15-594)."""

    def __init__(self, *a, **kw):
        super().__init__(*a, **kw)
        g, dt_, dev = self.grid, self.cfg.dtype, self.device
        self.adj_u = _mac(g, dt_, dev)
        self.init_adj_u = _mac(g, dt_, dev)
        self.src = _mac(g, dt_, dev)            # ajd_uw_source
        self.H_prev = _mac(g, dt_, dev)         # adj_u_*_AB_tem
        self.H_prev_prev = _mac(g, dt_, dev)    # adj_u_*_AB_tem2
        self.adj_passive = torch.zeros(g.shape, dtype=dt_, device=dev)
        self.init_adj_passive = torch.zeros_like(self.adj_passive)
        self.adj_passive_f = _mac(g, dt_, dev)
        self.mid_u = _mac(g, dt_, dev)
        if self.cfg.add_control_force:
            # calculate_adj_gausion_force outputs (3D/lfm_midpoint_diff_simulator.py:47-60)
            cap = max(self.cfg.control_num, 1)
            z = [torch.zeros((cap, self.dim), dtype=torch.float64, device=dev) for _ in range(4)]
            self.adj_gaussion_force_center, self.adj_gaussion_force_strength = DeviceField(z[0]), DeviceField(z[1])
            self.penalty_gaussion_force_center = DeviceField(z[2])
            self.penalty_gaussion_force_strength = DeviceField(z[3])
            self._gf_rows = 0
            if self.cfg.backward_u and self.cfg.store_control_force:
                # the forward's force fields, read back by the adjoint instead of re-evaluated
                self.store_force = [torch.empty((self.total_steps,) + g.face_shape(c), dtype=dt_, device=dev)
                                    for c in range(self.dim)]
        self.control_force_grads = {}
        # d loss / d viscosity as the reference accumulates it (adj_viscous), reset by init_gradient
        self.adj_viscous = DeviceField(torch.zeros(1, dtype=torch.float64, device=dev))
        self.target_passive = None
        self.target_trajectory = None
        self.loss = 0.0
        self._loss_dev = None
        self._capturing = False
        self.final_ind = None

    @property
    def adj_u_x(self):
        return self.adj_u[0]

    @property
    def adj_u_y(self):
        return self.adj_u[1]

    @property
    def adj_u_z(self):
        return self.adj_u[2] if self.dim == 3 else None

    def forward_step_midpoint(self, write_flow_map=True, write_passive=True, control_force_para=None):
        return self.step_midpoint(write_flow_map, write_passive, control_force_para)

    def init_gradient(self, theta=None, target_passive=None, target_vorticity=None):
        """Loss and adjoint seed (3D/lfm_midpoint_diff_simulator.py:336-376, case 11):
        L = sum (s - s*)^2, adj_passive = 2 (s - s*), adj_u = 0; psi, T reset.
        With ``target_vorticity`` (2D): L = sum (omega - omega*)^2 over the cells,
        adj_u = (d omega / d u)^T 2 (omega - omega*), adj_passive = 0."""
        if target_vorticity is not None:
            self._seed_vorticity(target_vorticity)
            return
        if target_passive is not None:
            self.target_passive = torch.empty(self.grid.shape, dtype=self.cfg.dtype, device=self.device)
            self.target_passive.copy_(_as_tensor(target_passive), non_blocking=True)
        if self.target_passive is None:
            raise FlowmapError(2, "init_gradient needs target_passive")
        self.final_ind = self.step_num[None] + 1
        for c in range(self.dim):
            self.adj_u[c].zero_()
            self.H_prev[c].zero_()
            self.H_prev_prev[c].zero_()
        diff = self.passive - self.target_passive
        self.adj_passive.copy_(2 * diff)
        self._loss_dev = torch.sum(diff.double() ** 2)
        self.loss = None if self._capturing else float(self._loss_dev)
        self._finish_seed()

    def _seed_vorticity(self, target_vorticity):
        if self.dim != 2:
            raise FlowmapError(1, "a vorticity loss needs a 2D simulator")
        g, dev = self.grid, self.device
        if getattr(self, "_vort_work", None) is None:
            self._vort_target = torch.empty(g.shape, dtype=self.cfg.dtype, device=dev)
            self._vort_work = torch.empty(g.shape, dtype=self.cfg.dtype, device=dev)
            self._vort_part = torch.empty(592, dtype=torch.float64, device=dev)
            self._vort_loss = torch.empty(1, dtype=torch.float64, device=dev)
        self._vort_target.copy_(_as_tensor(target_vorticity), non_blocking=True)
        self.final_ind = self.step_num[None] + 1
        for c in range(self.dim):
            self.H_prev[c].zero_()
            self.H_prev_prev[c].zero_()
        K.vorticity_loss_2d(g, self.dx, self.u[0], self.u[1], self._vort_target, self.adj_u[0], self.adj_u[1],
                            self._vort_work, self._vort_part, self._vort_loss)
        self.adj_passive.zero_()
        self._loss_dev = self._vort_loss
        self.loss = None if self._capturing else float(self._vort_loss.item())
        self._finish_seed()

    def _finish_seed(self):
        self._mask(adjoint=True)  # 3D/lfm_midpoint_diff_simulator.py:357-361
        self.step_num[None] = self.final_ind
        self.adj_viscous.tensor.zero_()
        _copy_mac(self.init_adj_u, self.adj_u)
        self.init_adj_passive.copy_(self.adj_passive)
        if self.cfg.backward_u:
            _copy_mac(self.init_u, self.u)
            self.init_passive.copy_(self.passive)
        self.reset_to_identity(self.psi, self.psi_f, self.T_f)

    def march_psi_grid(self, dt):
        self._march(self.psi, self.psi_f, self.T_f, self.mid_u, dt)

    def _backtrack_short_bfecc(self, curr_dt):
        """use_short_BFECC branch of the adjoint step (3D/lfm_midpoint_diff_simulator.py:440-485):
        adj_u (and adj_passive, and u / passive with backward_u) go back by BFECC
        through one-step maps of the midpoint velocity (psi_tem with -dt, phi_tem
        with +dt).  The reference adds the adjoint source here with -2 dt (the
        semi-Lagrangian branch uses -dt); kept as it is."""
        cfg = self.cfg
        self._short_maps(self.mid_u, -curr_dt, cfg.add_passive_scalar)
        maps = (self.T_f_tem, self.psi_f_tem, self.F_f_tem, self.phi_f_tem)
        self.BFECC(self.adj_u, self.final_u, self.err_u, *maps)
        for c in range(self.dim):
            K.add_fields(self.final_u[c], self.src[c], self.adj_u[c], -2 * curr_dt)
        if cfg.add_passive_scalar:
            self.BFECC_scalar(self.adj_passive, self.final_passive, self.err_passive, self.psi_tem, self.phi_tem)
            self.adj_passive, self.final_passive = self.final_passive, self.adj_passive
            for c in range(self.dim):
                K.add_fields(self.adj_u[c], self.adj_passive_f[c], self.adj_u[c], -curr_dt)
        if cfg.backward_u:
            if cfg.add_passive_scalar:
                self.BFECC_scalar(self.passive, self.final_passive, self.err_passive, self.psi_tem, self.phi_tem)
                self.passive, self.final_passive = self.final_passive, self.passive
            self.BFECC(self.u, self.final_u, self.err_u, *maps)
            self.u, self.final_u = self.final_u, self.u

    def calculate_adj_gausion_force(self, adj_u, center, inverse_radius, strength, num):
        """3D/lfm_midpoint_diff_simulator.py:63-69: the four per-Gaussian sums into
        adj_gaussion_force_center / _strength and penalty_gaussion_force_center /
        _strength (rows past ``num`` zero, as after the reference's fill(0))."""
        self._adj_gaussian(adj_u, self._gf.load({"c": center, "r": inverse_radius, "s": strength, "n": num}))

    def _adj_gaussian(self, adj_u, params):
        n = params[1].shape[0]
        outs = [f.tensor for f in (self.adj_gaussion_force_center, self.adj_gaussion_force_strength,
                                   self.penalty_gaussion_force_center, self.penalty_gaussion_force_strength)]
        if n < self._gf_rows:
            for t in outs:
                t[n:self._gf_rows].zero_()
        self._gf_rows = n
        K.gaussian_force_grad(self.grid, self.dx, *params, adj_u, out=[t[:n] for t in outs])

    def backtrack_step_midpoint(self, write_gradient=False, write_passive=False, control_force_para=None):
        """3D/lfm_midpoint_diff_simulator.py:390-419.  With add_control_force,
        ``control_force_para`` holds the parameters of the step being undone; the
        parameter gradients are left in adj_gaussion_force_* / penalty_gaussion_force_*."""
        self.step_num[None] -= 1
        n = self.step_num[None]
        j = n % self.reinit_every
        n0 = n - j
        if self.ckpt_u is not None and n == min(n0 + self.reinit_every, self.total_steps) - 1:
            if self._replayed == n // self.reinit_every:
                self._replayed = None  # the forward left this interval's replay state in place
            else:
                self._recompute_interval(n // self.reinit_every)  # first adjoint step of this interval
        if self.cfg.add_passive_scalar and not self.cfg.backward_u:
            if self._ring_passive is not None:
                self.passive.copy_(self._ring_passive[n + 1 - n0])
            else:
                K.store(self.store_passive[n + 1], self.passive)
        self.backtrack_flow_map(j, self.dt, control_force_para)
        return False, n == 0

    def backtrack_flow_map(self, j: int, curr_dt: float, control_force_para=None):
        """3D/lfm_midpoint_diff_simulator.py:421-594, with the 2D viscous term of
        2D/vortex/lfm_midpoint_diff_simulator.py:260-401 when viscosity != 0."""
        cfg, g, dx = self.cfg, self.grid, self.dx
        n = self.step_num[None]
        force = None
        if cfg.add_control_force:  # 3D/lfm_midpoint_diff_simulator.py:423-427
            params = self._control_params(control_force_para)
            if cfg.backward_u:
                if getattr(self, "store_force", None) is not None:
                    force = self._force_field(n)  # bitwise the field the forward step evaluated
                else:
                    force = self.control_force
                    K.gaussian_force(g, dx, *params, force)
            self._adj_gaussian(self.adj_u, params)
        for c in range(self.dim):
            if self.store_mid is not None:
                K.store(self.store_mid[c][n], self.mid_u[c])
            else:
                self.mid_u[c].copy_(self._ring[j][c])
        if self.vis is not None:  # 2D/vortex/lfm_midpoint_diff_simulator.py:270-271
            K.viscous_force_2d(g, cfg.viscosity, dx, self.mid_u, self.vis, adj=self.adj_u, part=self._vis_part,
                               dot=self.adj_viscous.tensor)
        K.nabla_u_w(g, dx, self.u if cfg.backward_u else self.mid_u, self.adj_u, self.src)
        if cfg.add_passive_scalar:
            K.nabla_scalar_adjoint(g, dx, self.passive, self.adj_passive, self.adj_passive_f)

        rk = cfg.RK_number
        if cfg.use_short_BFECC:
            self._backtrack_short_bfecc(curr_dt)
        else:
            if cfg.backward_u:
                # adj_u and u go back along the same midpoint velocity: one backtrace
                K.advect_u_grid_pair(g, rk, dx, -curr_dt, self.mid_u, self.adj_u, self.final_u, self.u, self.err_u)
                self.adj_u, self.final_u = self.final_u, self.adj_u
                self.u, self.err_u = self.err_u, self.u
            else:
                self._advect_u_grid(self.mid_u, self.adj_u, self.final_u, -curr_dt)
                self.adj_u, self.final_u = self.final_u, self.adj_u
            for c in range(self.dim):
                K.add_fields(self.adj_u[c], self.src[c], self.adj_u[c], -curr_dt)
            if cfg.add_passive_scalar:
                if cfg.backward_u:  # passive and adj_passive along the same backtrace
                    K.advect_scalar_grid_pair(g, rk, dx, -curr_dt, self.mid_u, self.passive, self.final_passive,
                                              self.adj_passive, self.err_passive)
                    self.passive, self.final_passive = self.final_passive, self.passive
                    self.adj_passive, self.err_passive = self.err_passive, self.adj_passive
                else:
                    self._advect_scalar_grid(self.mid_u, self.adj_passive, self.final_passive, -curr_dt)
                    self.adj_passive, self.final_passive = self.final_passive, self.adj_passive
                for c in range(self.dim):
                    K.add_fields(self.adj_u[c], self.adj_passive_f[c], self.adj_u[c], -curr_dt)

        self.march_psi_grid(curr_dt)
        # Adams-Bashforth index: adjoint steps already taken in this interval
        # (= reinit_every-1-j for a full interval, as the reference computes it)
        interval_last = min((n // self.reinit_every) * self.reinit_every + self.reinit_every - 1,
                            self.total_steps - 1)
        if cfg.add_passive_scalar:  # the two accumulations in one pass (equal to two launches)
            K.accumulate_init_pair(g, dx, -2 * curr_dt, self.src, self.init_adj_u, self.T_f, self.psi_f,
                                   self.adj_passive_f, -curr_dt, self.H_prev, self.H_prev_prev, interval_last - n)
        else:
            K.accumulate_init(g, dx, -2 * curr_dt, self.src, self.init_adj_u, self.T_f, self.psi_f, self.H_prev,
                              self.H_prev_prev, interval_last - n)
        if self.vis is not None:  # 2D/vortex/lfm_midpoint_diff_simulator.py:387-389
            for c in range(self.dim):
                K.add_fields(self.adj_u[c], self.vis[c], self.adj_u[c], -curr_dt)
            K.accumulate_init(g, dx, -curr_dt, self.vis, self.init_adj_u, self.T_f, self.psi_f)
        self.project(self.adj_u)  # Poisson_adj
        if cfg.backward_u:
            if cfg.add_control_force:  # 3D/lfm_midpoint_diff_simulator.py:525-530
                for c in range(self.dim):
                    K.add_fields(self.u[c], force[c], self.u[c], -curr_dt)
                K.accumulate_init(g, dx, -curr_dt, force, self.init_u, self.T_f, self.psi_f)
            if self.vis is not None:  # 2D/vortex/lfm_midpoint_diff_simulator.py:399-401
                for c in range(self.dim):
                    K.add_fields(self.u[c], self.vis[c], self.u[c], -curr_dt)
                K.accumulate_init(g, dx, -curr_dt, self.vis, self.init_u, self.T_f, self.psi_f)
            self.project(self.u)
        self._mask(adjoint=True)  # 3D/lfm_midpoint_diff_simulator.py:534-538

        if j == 0:
            k = n // self.reinit_every
            if self.store_phi is not None:  # with interval checkpointing phi, F hold the replayed interval's maps
                self.phi.copy_(self.store_phi[k])
                for c in range(self.dim):
                    self.phi_f[c].copy_(self.store_phi_f[c][k])
                    self.F_f[c].copy_(self.store_F_f[c][k])
            self.BFECC(self.init_adj_u, self.adj_u, self.err_u, self.F_f, self.phi_f, self.T_f, self.psi_f)
            self.project(self.adj_u)
            _copy_mac(self.init_adj_u, self.adj_u)
            if cfg.backward_u:
                self.BFECC(self.init_u, self.u, self.err_u, self.F_f, self.phi_f, self.T_f, self.psi_f)
                self.project(self.u)
                _copy_mac(self.init_u, self.u)
            self._mask(adjoint=True)  # 3D/lfm_midpoint_diff_simulator.py:572-576
            if cfg.add_passive_scalar:
                if self._ring_passive is not None:
                    self.passive.copy_(self._ring_passive[0])
                elif cfg.trajectory_loss or not cfg.backward_u:
                    K.store(self.store_passive[n], self.passive)
                else:
                    self.BFECC_scalar(self.init_passive, self.passive, self.err_passive, self.phi, self.psi)
                self.init_passive.copy_(self.passive)
                self.BFECC_scalar(self.init_adj_passive, self.adj_passive, self.err_passive, self.phi, self.psi)
                if cfg.trajectory_loss:
                    tgt = self.target_trajectory[n]
                    d = self.passive - tgt
                    self.adj_passive.add_(d)
                    self.loss += float(torch.sum(d.double() ** 2))
                self.init_adj_passive.copy_(self.adj_passive)
            self.reset_to_identity(self.psi, self.psi_f, self.T_f)

    # --------------------------------------------------------- driver
    def gradient(self, u0, passive0=None, target_passive=None, target_vorticity=None, control_forces=None):
        """Full forward + adjoint: returns (loss, dL/du0 as a list of face tensors).
        The loss is the final passive L2 (``target_passive``) or, in 2D, the final
        vorticity L2 (``target_vorticity``).  With add_control_force,
        ``control_forces[n]`` is step n's control_force_para, and the per-step
        parameter gradients are kept in ``control_force_grads[n]`` = (adj_center,
        adj_strength, penalty_center, penalty_strength), device FP64 n x dim."""
        self.run_forward(u0, passive0, control_forces)
        return self.run_adjoint(target_passive, target_vorticity, control_forces)

    def run_forward(self, u0, passive0=None, control_forces=None):
        """The forward half of ``gradient``: init from u0 (and passive0) and every
        leapfrog step, leaving the trajectory the adjoint reads in the stores.
        ``forward_serial`` counts completed forward passes, so that a caller who
        runs the adjoint later can tell whether the trajectory is still its own."""
        cf = self.cfg.add_control_force
        if cf and control_forces is None:
            raise FlowmapError(2, "add_control_force needs control_forces (one control_force_para per step)")
        self.init(theta=u0, init_passive_np=passive0)
        while True:
            para = control_forces[self.step_num[None] + 1] if cf else None
            _, final = self.forward_step_midpoint(control_force_para=para)
            if final:
                break
        self.forward_serial = getattr(self, "forward_serial", 0) + 1

    def run_adjoint(self, target_passive=None, target_vorticity=None, control_forces=None):
        """The adjoint half of ``gradient``, on the trajectory of the last
        ``run_forward``: returns (loss, dL/du0 as a list of face tensors)."""
        cf = self.cfg.add_control_force
        if cf and control_forces is None:
            raise FlowmapError(2, "add_control_force needs control_forces (one control_force_para per step)")
        self.control_force_grads = {}
        self.init_gradient(target_passive=target_passive, target_vorticity=target_vorticity)
        while True:
            n = self.step_num[None] - 1
            _, done = self.backtrack_step_midpoint(control_force_para=control_forces[n] if cf else None)
            if cf:
                rows = self._gf_rows
                self.control_force_grads[n] = tuple(
                    f.tensor[:rows].clone() for f in (self.adj_gaussion_force_center, self.adj_gaussion_force_strength,
                                                      self.penalty_gaussion_force_center,
                                                      self.penalty_gaussion_force_strength))
            if done:
                break
        if self._capturing:
            return None, self.adj_u
        # the solver's device-side counters, read once per gradient (one stream sync)
        self.solver_stats = self.solver.stats(reset=True)
        if self.solver_stats and self.solver_stats["nonfinite"]:
            raise FlowmapError(4, f"{self.solver_stats['nonfinite']} projection(s) hit a non-finite residual")
        return self.loss, [x.clone() for x in self.adj_u]

    def capture_gradient(self, u0, passive0=None, target_passive=None, target_vorticity=None, stream=None):
        """Record ``gradient(u0, ...)`` as one CUDA graph and return its GradientGraph.

        The inputs must be device tensors that stay alive: the graph copies from
        them on every replay, so refill them in place between replays.  One eager
        gradient runs first (it creates every lazily allocated buffer outside the
        capture and leaves the same results).  Not available with control forces (their
        parameters are staged from the host every step), a trajectory loss (read on
        the host) or a host-checked solver (check_every > 0)."""
        self.prepare_capture(u0, passive0, target_passive, target_vorticity)
        s = stream if stream is not None else torch.cuda.Stream(device=self.device)
        torch.cuda.synchronize(self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s, capture_error_mode="thread_local"):
            roles, loss_dev, kernels = self.record_gradient(u0, passive0, target_passive, target_vorticity)
        return GradientGraph(self, graph, roles, loss_dev, kernels)

    def prepare_capture(self, u0, passive0=None, target_passive=None, target_vorticity=None):
        """Checks that a gradient with these inputs can be recorded, and runs it
        once eagerly (every lazily allocated buffer exists afterwards)."""
        cfg = self.cfg
        if cfg.add_control_force or cfg.trajectory_loss:
            raise FlowmapError(2, "capture_gradient: control forces and a trajectory loss are not capturable")
        if not getattr(self.solver, "device_mode", False):
            raise FlowmapError(2, "capture_gradient needs the device-side solver (check_every = 0)")
        for x in list(u0) + [passive0, target_passive, target_vorticity]:
            if x is not None and not (isinstance(x, torch.Tensor) and x.is_cuda):
                raise FlowmapError(2, "capture_gradient: inputs must be device tensors")
        self.gradient(u0, passive0, target_passive, target_vorticity)

    def record_gradient(self, u0, passive0=None, target_passive=None, target_vorticity=None):
        """Record one gradient on the current stream, which must be capturing (after
        prepare_capture).  Returns (roles, loss tensor, kernels recorded outside the
        PCG loop bodies): what a GradientGraph needs to replay it."""
        before = _lib.launch_count()
        self._capturing = True
        try:
            self.gradient(u0, passive0, target_passive, target_vorticity)
        finally:
            self._capturing = False
        kernels = _lib.launch_count() - before
        roles = {k: getattr(self, k) for k in _ROLES if hasattr(self, k)}
        return roles, self._loss_dev, kernels


# fields whose tensors the steps exchange by reference (ping-pong buffers)
_ROLES = ("u", "final_u", "err_u", "adj_u", "passive", "final_passive", "adj_passive", "err_passive")


class GradientGraph:
    """One whole forward + adjoint gradient recorded as a CUDA graph
    (``LFM_Diff_Simulator.capture_gradient``).  ``replay()`` re-runs it on the
    current contents of the input tensors given at capture time, on the current
    stream, with one graph launch; the simulator's fields (adj_u, u, ...) then
    hold that run's results, as after ``gradient()``.  The projections inside
    are device-side PCG loops (conditional WHILE nodes), so the replay needs no
    host decision.  Results are bit-identical to the eager gradient: the graph
    holds the same kernels in the same order."""

    def __init__(self, sim, graph, roles, loss_dev, kernels):
        self.sim = sim
        self.graph = graph
        self.roles = roles
        self.loss_dev = loss_dev
        self.kernels = kernels  # kernel nodes recorded outside the PCG loop bodies

    def replay(self):
        self.graph.replay()
        for k, v in self.roles.items():
            setattr(self.sim, k, v)

    def loss(self) -> float:
        """The last replay's loss (synchronises with the current stream)."""
        return float(self.loss_dev.item())

    def stats(self) -> dict:
        """Solver counters accumulated since the last read (synchronises)."""
        st = self.sim.solver.stats(reset=True)
        if st and st["nonfinite"]:
            raise FlowmapError(4, f"{st['nonfinite']} projection(s) hit a non-finite residual")
        return st
