"""MGPCG pressure projection with the reference's solver interface.

``MGPCG_3`` / ``MGPCG_2`` mirror 3D/mgpcg.py:359-439 and 2D/shape/mgpcg.py:292-368
(plain all-Neumann solver, base_level 3, bottom smoothing 50, absolute
tolerance rTr < 1e-12, max 400 iterations).  ``MGPCG_2_solid`` mirrors
2D/vortex/mgpcg_solid.py:370-458 (base_level 4, 20 bottom sweeps as
10 x (R,B) + 10 x (B,R), tol = max(1e-14, 1e-16 zTr0)); with a non-empty
obstacle mask it is a ``SolidMGPCG`` (libflowmap's fm_solid_*).
``Poisson(u_x, u_y[, u_z])`` projects in place; ``Poisson_adj`` is the same
operation (3D/fast_mgpcg.py:283-323 differs from Poisson only in name).

Every solve runs on the device (libflowmap_sm100.so); there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
import warnings
from typing import Optional, Sequence

import torch

from . import _lib
from .kernels import GridSpec


class MGPCG:
    """Owns the device MG hierarchy for one grid shape and dtype."""

    def __init__(self, N: Sequence[int], dtype=torch.float32, *, base_level: int = 3, levels: Optional[int] = None,
                 pre_post: int = 2, bottom: int = 50, bottom_mode: int = 0, max_iters: int = 400,
                 abs_tol: float = 1e-12, rel_tol: float = 0.0, eps: float = 1e-12, check_every: int = 4,
                 raise_on_nonconvergence: bool = False, coarse_bf16: bool = False, dc_rel_tol: float = 0.0,
                 dc_max_outer: int = 4):
        """coarse_bf16 (FP32 solvers): store the per-level coarse grids between the
        finest level and the shared-memory-resident ones in BF16 (arithmetic stays
        FP32); the preconditioner then no longer equals the FP32 V-cycle bit for bit.
        dc_rel_tol > 0 (FP32 solvers, check_every = 0): every ``project`` runs an FP64
        outer defect correction around the FP32 solves (fm_project_dc) until the FP64
        residual is below dc_rel_tol |b|, at most dc_max_outer corrections."""
        self.N = tuple(int(n) for n in N)
        self.grid = GridSpec(self.N)
        self.dtype = dtype
        if levels is None:
            levels = int(math.log2(min(self.N))) - base_level + 1
        self.params = _lib.MGParams(levels, pre_post, bottom, bottom_mode, max_iters, abs_tol, rel_tol, eps,
                                    check_every, int(coarse_bf16))
        self.raise_on_nonconvergence = raise_on_nonconvergence
        self._h = C.c_void_p()
        _lib.check(_lib.lib().fm_mgpcg_create(C.byref(self.grid.c_grid()), _lib.dtype_code(dtype),
                                              C.byref(self.params), C.byref(self._h)), "fm_mgpcg_create")
        self.last_iters = 0
        self.last_rtr = 0.0
        self.last_converged = True
        self.history = []
        self.dc_rel_tol, self.dc_max_outer = float(dc_rel_tol), int(dc_max_outer)
        self._dc_work = None
        if self.dc_rel_tol > 0:
            if dtype != torch.float32 or check_every != 0:
                raise _lib.FlowmapError(2, "defect correction needs an FP32 solver in device mode (check_every=0)")
            n = self.grid.ncell
            self._dc_work = torch.empty(3 * n, dtype=torch.float64, device="cuda")

    @property
    def n_mg_levels(self) -> int:
        return self.params.levels

    def close(self):
        if self._h:
            _lib.lib().fm_mgpcg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _status(self, st: int, where: str, it: C.c_int, rtr: C.c_double):
        self.last_iters = it.value
        self.last_rtr = rtr.value
        self.last_converged = st == 0
        self.history.append((it.value, rtr.value))
        if st == 3:  # FM_ERR_NOT_CONVERGED: the reference continues silently
            if self.raise_on_nonconvergence:
                _lib.check(st, where)
            return
        _lib.check(st, where)

    def project(self, u: Sequence[torch.Tensor], p_out: Optional[torch.Tensor] = None, stream=None):
        """In-place pressure projection of the MAC velocity ``u``."""
        if len(u) != self.grid.dim:
            raise _lib.FlowmapError(2, "project: wrong number of components")
        for c, x in enumerate(u):
            if tuple(x.shape) != self.grid.face_shape(c) or x.dtype != self.dtype:
                raise _lib.FlowmapError(1, f"project: component {c} shape/dtype mismatch")
        ps = [_lib.ptr(x) for x in u] + [None] * (3 - len(u))
        if self._dc_work is not None:
            if p_out is not None and (p_out.dtype != torch.float64 or tuple(p_out.shape) != self.N):
                raise _lib.FlowmapError(1, "project with defect correction: p_out must be an FP64 cell grid")
            _lib.check(_lib.lib().fm_project_dc(self._h, ps[0], ps[1], ps[2], _lib.ptr(self._dc_work),
                                                self.dc_rel_tol, self.dc_max_outer, _lib.ptr(p_out),
                                                _lib.stream_ptr(stream)), "fm_project_dc")
            return
        if self.device_mode:
            # asynchronous: the outcome is folded into stats()
            st = _lib.lib().fm_project(self._h, ps[0], ps[1], ps[2], _lib.ptr(p_out), _lib.stream_ptr(stream),
                                       None, None)
            _lib.check(st, "fm_project")
            return
        it, rtr = C.c_int(0), C.c_double(0)
        st = _lib.lib().fm_project(self._h, ps[0], ps[1], ps[2], _lib.ptr(p_out), _lib.stream_ptr(stream),
                                   C.byref(it), C.byref(rtr))
        self._status(st, "fm_project", it, rtr)

    @property
    def device_mode(self) -> bool:
        return self.params.check_every == 0

    def stats(self, reset: bool = False, stream=None) -> dict:
        """Cumulative solver outcome (synchronises the stream)."""
        s = _lib.MGStats()
        _lib.check(_lib.lib().fm_mgpcg_stats(self._h, _lib.stream_ptr(stream), int(reset), C.byref(s)),
                   "fm_mgpcg_stats")
        return {"solves": s.solves, "iterations": s.iterations, "not_converged": s.not_converged,
                "nonfinite": s.nonfinite, "last_iters": s.last_iters, "max_iters_seen": s.max_iters_seen,
                "last_rtr": s.last_rtr}

    def solve(self, b: torch.Tensor, x: torch.Tensor, stream=None):
        it, rtr = C.c_int(0), C.c_double(0)
        st = _lib.lib().fm_mgpcg_solve(self._h, _lib.ptr(b), _lib.ptr(x), _lib.stream_ptr(stream), C.byref(it),
                                       C.byref(rtr))
        self._status(st, "fm_mgpcg_solve", it, rtr)
        return it.value, rtr.value

    def apply_preconditioner(self, r: torch.Tensor, z: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        """One V-cycle z = M^-1 r (3D/mgpcg.py:187-205), r not recentred."""
        if tuple(r.shape) != self.N or r.dtype != self.dtype:
            raise _lib.FlowmapError(1, "apply_preconditioner: r shape/dtype mismatch")
        if z is None:
            z = torch.empty_like(r)
        _lib.check(_lib.lib().fm_mg_vcycle(self._h, _lib.ptr(r), _lib.ptr(z), _lib.stream_ptr(stream)),
                   "fm_mg_vcycle")
        return z

    def solve_mixed(self, b: torch.Tensor, x: Optional[torch.Tensor] = None, rel_tol: float = 1e-10,
                    max_outer: int = 10, work: Optional[torch.Tensor] = None, stream=None):
        """Mixed-precision solve: FP32 MGPCG inner solves (this FP32 solver) inside
        an FP64 defect correction, until |b - A x| <= rel_tol |b| in FP64.
        Returns (x FP64, outer corrections, inner PCG iterations, final relative residual)."""
        if self.dtype != torch.float32:
            raise _lib.FlowmapError(7, "solve_mixed needs an FP32 solver")
        if tuple(b.shape) != self.N:
            raise _lib.FlowmapError(1, "solve_mixed: b shape mismatch")
        if x is None:
            x = torch.empty(self.N, dtype=torch.float64, device=b.device)
        if work is None:
            work = torch.empty(self.N, dtype=torch.float64, device=b.device)
        no, ni, rr = C.c_int(0), C.c_int(0), C.c_double(0)
        st = _lib.lib().fm_mgpcg_solve_dc(self._h, _lib.dtype_code(b.dtype), _lib.ptr(b), _lib.ptr(x),
                                          _lib.ptr(work), rel_tol, max_outer, _lib.stream_ptr(stream),
                                          C.byref(no), C.byref(ni), C.byref(rr))
        self.last_converged = st == 0
        if st != 3 or self.raise_on_nonconvergence:
            _lib.check(st, "fm_mgpcg_solve_dc")
        return x, no.value, ni.value, rr.value

    # reference names -------------------------------------------------------
    def Poisson(self, *u, verbose: bool = False):
        self.project(u)
        if verbose:
            print(f"[MGPCG] iters={self.last_iters} |r|={math.sqrt(max(self.last_rtr, 0.0)):.3e} "
                  f"converged={self.last_converged}")

    def Poisson_adj(self, *u, verbose: bool = False):
        self.Poisson(*u, verbose=verbose)


class SolidMGPCG:
    """MGPCG with a boundary mask (2D/vortex/mgpcg_solid.py:14-458, dimension-
    generic): cells with mask > 0 are solid; same interface as MGPCG.  The PCG
    loop polls its device-side convergence flag every ``check_every`` (>= 1)
    iterations."""

    def __init__(self, N: Sequence[int], mask: torch.Tensor, dtype=torch.float32, *, base_level: int = 4,
                 levels: Optional[int] = None, pre_post: int = 2, bottom: int = 20, bottom_mode: int = 1,
                 max_iters: int = 400, abs_tol: float = 1e-14, rel_tol: float = 1e-16, eps: float = 1e-12,
                 check_every: int = 4, raise_on_nonconvergence: bool = False):
        self.N = tuple(int(n) for n in N)
        self.grid = GridSpec(self.N)
        self.dtype = dtype
        if levels is None:
            levels = int(math.log2(min(self.N))) - base_level + 1
        if int(check_every) < 0:
            raise _lib.FlowmapError(2, "check_every must be >= 0")
        self.params = _lib.MGParams(levels, pre_post, bottom, bottom_mode, max_iters, abs_tol, rel_tol, eps,
                                    int(check_every), 0)
        self.raise_on_nonconvergence = raise_on_nonconvergence
        self.mask = self._as_mask(mask)
        self._h = C.c_void_p()
        _lib.check(_lib.lib().fm_solid_create(C.byref(self.grid.c_grid()), _lib.dtype_code(dtype),
                                              C.byref(self.params), _lib.ptr(self.mask), C.byref(self._h)),
                   "fm_solid_create")
        self.last_iters, self.last_rtr, self.last_converged = 0, 0.0, True
        self.history = []
        self._stats = {"solves": 0, "iterations": 0, "not_converged": 0, "nonfinite": 0, "last_iters": 0,
                       "max_iters_seen": 0, "last_rtr": 0.0}

    def _as_mask(self, mask):
        m = torch.as_tensor(mask)
        if tuple(m.shape) != self.N:
            raise _lib.FlowmapError(1, f"mask shape {tuple(m.shape)} != grid {self.N}")
        return m.to(device="cuda", dtype=torch.float32).contiguous()

    @property
    def n_mg_levels(self) -> int:
        return self.params.levels

    @property
    def device_mode(self) -> bool:
        """check_every == 0: the PCG loop runs on the device; project() returns
        at once and the outcome is read by stats()."""
        return self.params.check_every == 0

    def set_mask(self, mask, stream=None):
        self.mask = self._as_mask(mask)
        _lib.check(_lib.lib().fm_solid_set_mask(self._h, _lib.ptr(self.mask), _lib.stream_ptr(stream)),
                   "fm_solid_set_mask")

    def close(self):
        if self._h:
            _lib.lib().fm_solid_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _status(self, st, where, it, rtr):
        self.last_iters, self.last_rtr, self.last_converged = it.value, rtr.value, st == 0
        self.history.append((it.value, rtr.value))
        S = self._stats
        S["solves"] += 1
        S["iterations"] += it.value
        S["last_iters"], S["last_rtr"] = it.value, rtr.value
        S["max_iters_seen"] = max(S["max_iters_seen"], it.value)
        if st == 3:
            S["not_converged"] += 1
            if self.raise_on_nonconvergence:
                _lib.check(st, where)
            return
        if st == 4:
            S["nonfinite"] += 1
            return
        _lib.check(st, where)

    def project(self, u: Sequence[torch.Tensor], p_out: Optional[torch.Tensor] = None, stream=None):
        if len(u) != self.grid.dim:
            raise _lib.FlowmapError(2, "project: wrong number of components")
        for c, x in enumerate(u):
            if tuple(x.shape) != self.grid.face_shape(c) or x.dtype != self.dtype:
                raise _lib.FlowmapError(1, f"project: component {c} shape/dtype mismatch")
        ps = [_lib.ptr(x) for x in u] + [None] * (3 - len(u))
        if self.device_mode:
            st = _lib.lib().fm_solid_project(self._h, ps[0], ps[1], ps[2], _lib.ptr(p_out), _lib.stream_ptr(stream),
                                             None, None)
            _lib.check(st, "fm_solid_project")
            return
        it, rtr = C.c_int(0), C.c_double(0)
        st = _lib.lib().fm_solid_project(self._h, ps[0], ps[1], ps[2], _lib.ptr(p_out), _lib.stream_ptr(stream),
                                         C.byref(it), C.byref(rtr))
        self._status(st, "fm_solid_project", it, rtr)

    def solve(self, b: torch.Tensor, x: torch.Tensor, stream=None):
        it, rtr = C.c_int(0), C.c_double(0)
        st = _lib.lib().fm_solid_solve(self._h, _lib.ptr(b), _lib.ptr(x), _lib.stream_ptr(stream), C.byref(it),
                                       C.byref(rtr))
        self._status(st, "fm_solid_solve", it, rtr)
        return it.value, rtr.value

    def apply_preconditioner(self, r: torch.Tensor, z: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        if tuple(r.shape) != self.N or r.dtype != self.dtype:
            raise _lib.FlowmapError(1, "apply_preconditioner: r shape/dtype mismatch")
        if z is None:
            z = torch.empty_like(r)
        _lib.check(_lib.lib().fm_solid_vcycle(self._h, _lib.ptr(r), _lib.ptr(z), _lib.stream_ptr(stream)),
                   "fm_solid_vcycle")
        return z

    def stats(self, reset: bool = False, stream=None) -> dict:
        """Cumulative solver outcome, counted on the device (synchronises the stream)."""
        s = _lib.MGStats()
        _lib.check(_lib.lib().fm_solid_stats(self._h, _lib.stream_ptr(stream), int(reset), C.byref(s)),
                   "fm_solid_stats")
        if reset:
            for k in self._stats:
                self._stats[k] = 0.0 if k == "last_rtr" else 0
        return {"solves": s.solves, "iterations": s.iterations, "not_converged": s.not_converged,
                "nonfinite": s.nonfinite, "last_iters": s.last_iters, "max_iters_seen": s.max_iters_seen,
                "last_rtr": s.last_rtr}

    def Poisson(self, *u, verbose: bool = False):
        self.project(u)
        if verbose:
            print(f"[MGPCG] iters={self.last_iters} |r|={math.sqrt(max(self.last_rtr, 0.0)):.3e} "
                  f"converged={self.last_converged}")

    def Poisson_adj(self, *u, verbose: bool = False):
        self.Poisson(*u, verbose=verbose)


class MGPCG_3(MGPCG):
    """3D/mgpcg.py:359 MGPCG_3(boundary_types, N, base_level=3)."""

    def __init__(self, boundary_types=None, N=(128, 128, 128), base_level=3, real=None, dtype=torch.float32, **kw):
        kw.setdefault("bottom", 50)
        kw.setdefault("abs_tol", 1e-12)
        super().__init__(N, dtype, base_level=base_level, **kw)


class MGPCG_2(MGPCG):
    """2D/shape/mgpcg.py:292 MGPCG_2(boundary_types, N, base_level=3)."""

    def __init__(self, boundary_types=None, N=(256, 256), base_level=3, real=None, dtype=torch.float32, **kw):
        kw.setdefault("bottom", 50)
        kw.setdefault("abs_tol", 1e-12)
        super().__init__(N, dtype, base_level=base_level, **kw)


class MGPCG_2_solid(MGPCG):
    """2D/vortex/mgpcg_solid.py:370.  With a non-empty boundary_mask the
    constructor returns a SolidMGPCG; with an empty one the all-Neumann solver
    (the same operator) with the solid variant's settings."""

    def __new__(cls, boundary_types=None, boundary_mask=None, boundary_vel=None, N=(256, 256), base_level=4,
                real=None, dtype=torch.float32, **kw):
        if boundary_mask is not None and bool((torch.as_tensor(boundary_mask) > 0).any()):
            return SolidMGPCG(N, boundary_mask, dtype, base_level=4, **kw)
        return super().__new__(cls)

    def __init__(self, boundary_types=None, boundary_mask=None, boundary_vel=None, N=(256, 256), base_level=4,
                 real=None, dtype=torch.float32, **kw):
        kw.setdefault("bottom", 20)
        kw.setdefault("bottom_mode", 1)
        kw.setdefault("abs_tol", 1e-14)
        kw.setdefault("rel_tol", 1e-16)
        super().__init__(N, dtype, base_level=4, **kw)
