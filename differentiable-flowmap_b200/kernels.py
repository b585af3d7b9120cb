"""Thin, typed wrappers over the C ABI (one function per entry point).

Fields are torch CUDA tensors.  A MAC velocity is a tuple of ``dim`` face
tensors; vector fields on a grid (psi, T, phi, F) are ``(dim, *grid)``
tensors (SoA planes), matching include/flowmap_sm100.h.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import torch

from . import _lib
from ._lib import check, dtype_code, ptr, stream_ptr


@dataclass(frozen=True)
class GridSpec:
    """Cell counts of a 2D (nz == 1) or 3D grid."""

    shape: Tuple[int, ...]

    @property
    def dim(self) -> int:
        return len(self.shape)

    def c_grid(self) -> _lib.Grid:
        n = list(self.shape) + [1] * (3 - self.dim)
        return _lib.Grid(self.dim, (C.c_int * 3)(*n))

    def face_shape(self, c: int) -> Tuple[int, ...]:
        s = list(self.shape)
        s[c] += 1
        return tuple(s)

    @property
    def ncell(self) -> int:
        n = 1
        for v in self.shape:
            n *= v
        return n

    @staticmethod
    def from_mac(u: Sequence[torch.Tensor]) -> "GridSpec":
        dim = len(u)
        s = list(u[0].shape[-dim:])
        s[0] -= 1
        return GridSpec(tuple(s))

    def which_grid(self, t: torch.Tensor) -> int:
        """Face index (0..dim-1) of a field, or -1 for the cell grid."""
        sh = tuple(t.shape[-self.dim:])
        if sh == tuple(self.shape):
            return -1
        for c in range(self.dim):
            if sh == self.face_shape(c):
                return c
        raise _lib.FlowmapError(1, f"field shape {tuple(t.shape)} does not match grid {self.shape}")


def _mac3(u):
    u = list(u) if u is not None else []
    return [ptr(x) for x in u] + [None] * (3 - len(u))


def _dt(t: torch.Tensor) -> int:
    return dtype_code(t.dtype)


def _chk_mac(g: GridSpec, u, name):
    if len(u) != g.dim:
        raise _lib.FlowmapError(2, f"{name}: expected {g.dim} components")
    for c, x in enumerate(u):
        if tuple(x.shape) != g.face_shape(c):
            raise _lib.FlowmapError(1, f"{name}[{c}] has shape {tuple(x.shape)}, expected {g.face_shape(c)}")


def _chk_vec(g: GridSpec, t, face, name):
    want = (g.dim,) + (g.face_shape(face) if face >= 0 else tuple(g.shape))
    if tuple(t.shape) != want:
        raise _lib.FlowmapError(1, f"{name} has shape {tuple(t.shape)}, expected {want}")


def advect_u_grid(g: GridSpec, rk: int, dx: float, dt: float, u0, u1, u2, stream=None):
    for n, u in (("u0", u0), ("u1", u1), ("u2", u2)):
        _chk_mac(g, u, n)
    check(_lib.lib().fm_advect_u_grid(C.byref(g.c_grid()), _dt(u0[0]), rk, dx, dt, *_mac3(u0), *_mac3(u1),
                                      *_mac3(u2), stream_ptr(stream)), "fm_advect_u_grid")


def advect_scalar_grid(g: GridSpec, rk: int, dx: float, dt: float, u0, s1, s2, stream=None):
    _chk_mac(g, u0, "u0")
    check(_lib.lib().fm_advect_scalar_grid(C.byref(g.c_grid()), _dt(u0[0]), rk, dx, dt, *_mac3(u0), ptr(s1), ptr(s2),
                                           stream_ptr(stream)), "fm_advect_scalar_grid")


def advect_u_grid_pair(g: GridSpec, rk: int, dx: float, dt: float, u0, u1, u2, v1, v2, stream=None):
    """Two advect_u_grid calls sharing u0/rk/dt, with one backtrace per node."""
    for n, u in (("u0", u0), ("u1", u1), ("u2", u2), ("v1", v1), ("v2", v2)):
        _chk_mac(g, u, n)
    check(_lib.lib().fm_advect_u_grid_pair(C.byref(g.c_grid()), _dt(u0[0]), rk, dx, dt, *_mac3(u0), *_mac3(u1),
                                           *_mac3(u2), *_mac3(v1), *_mac3(v2), stream_ptr(stream)),
          "fm_advect_u_grid_pair")


def advect_scalar_grid_pair(g: GridSpec, rk: int, dx: float, dt: float, u0, s1, s2, t1, t2, stream=None):
    """Two advect_scalar_grid calls sharing u0/rk/dt, with one backtrace per cell."""
    _chk_mac(g, u0, "u0")
    check(_lib.lib().fm_advect_scalar_grid_pair(C.byref(g.c_grid()), _dt(u0[0]), rk, dx, dt, *_mac3(u0), ptr(s1),
                                                ptr(s2), ptr(t1), ptr(t2), stream_ptr(stream)),
          "fm_advect_scalar_grid_pair")


def rk_grid(g: GridSpec, rk: int, dx: float, dt: float, face: int, psi, T, u, stream=None):
    _chk_mac(g, u, "u")
    _chk_vec(g, psi, face, "psi")
    if T is not None:
        _chk_vec(g, T, face, "T")
    check(_lib.lib().fm_rk_grid(C.byref(g.c_grid()), _dt(psi), rk, dx, dt, face, ptr(psi), ptr(T), *_mac3(u),
                                stream_ptr(stream)), "fm_rk_grid")


def march_map(g: GridSpec, rk: int, dx: float, dt: float, psi_c, psi_f, T_f, u, stream=None):
    _chk_mac(g, u, "u")
    ps = list(psi_f) + [None] * (3 - g.dim)
    ts = list(T_f) + [None] * (3 - g.dim)
    check(_lib.lib().fm_march_map(C.byref(g.c_grid()), _dt(u[0]), rk, dx, dt, ptr(psi_c), ptr(ps[0]), ptr(ts[0]),
                                  ptr(ps[1]), ptr(ts[1]), ptr(ps[2]), ptr(ts[2]), *_mac3(u), stream_ptr(stream)),
          "fm_march_map")


def pullback_u(g: GridSpec, dx: float, u0, out, T_f, psi_f, alpha=1.0, beta=0.0, base=None, stream=None):
    _chk_mac(g, u0, "u0")
    _chk_mac(g, out, "out")
    check(_lib.lib().fm_pullback_u(C.byref(g.c_grid()), _dt(u0[0]), dx, *_mac3(u0), *_mac3(out), *_mac3(T_f),
                                   *_mac3(psi_f), alpha, beta, *_mac3(base), stream_ptr(stream)), "fm_pullback_u")


def pullback_scalar(g: GridSpec, dx: float, s0, out, psi, alpha=1.0, beta=0.0, base=None, stream=None):
    check(_lib.lib().fm_pullback_scalar(C.byref(g.c_grid()), _dt(s0), dx, ptr(s0), ptr(out), ptr(psi), alpha, beta,
                                        ptr(base), stream_ptr(stream)), "fm_pullback_scalar")


def _mac_opt(g: GridSpec, u, name):
    if u is not None:
        _chk_mac(g, u, name)
    return _mac3(u)


def advect_scalar_grid_adj(g: GridSpec, rk: int, dx: float, dt: float, u0, s1, g_s2, g_u0=None, g_s1=None,
                           stream=None):
    """g_u0 += dL/du0, g_s1 += dL/ds1 for s2 = advect_scalar_grid(u0, s1), given g_s2 = dL/ds2."""
    _chk_mac(g, u0, "u0")
    check(_lib.lib().fm_advect_scalar_grid_adj(C.byref(g.c_grid()), _dt(u0[0]), rk, dx, dt, *_mac3(u0), ptr(s1),
                                               ptr(g_s2), *_mac_opt(g, g_u0, "g_u0"), ptr(g_s1),
                                               stream_ptr(stream)), "fm_advect_scalar_grid_adj")


def advect_u_grid_adj(g: GridSpec, rk: int, dx: float, dt: float, u0, u1, g_u2, g_u0=None, g_u1=None, stream=None):
    """g_u0 += dL/du0 (backtrace), g_u1 += dL/du1 (sampled field) for u2 = advect_u_grid(u0, u1)."""
    for n, u in (("u0", u0), ("u1", u1), ("g_u2", g_u2)):
        _chk_mac(g, u, n)
    check(_lib.lib().fm_advect_u_grid_adj(C.byref(g.c_grid()), _dt(u0[0]), rk, dx, dt, *_mac3(u0), *_mac3(u1),
                                          *_mac3(g_u2), *_mac_opt(g, g_u0, "g_u0"), *_mac_opt(g, g_u1, "g_u1"),
                                          stream_ptr(stream)), "fm_advect_u_grid_adj")


def pullback_u_adj(g: GridSpec, dx: float, u0, T_f, psi_f, g_out, alpha=1.0, beta=0.0, g_u0=None, g_T=None,
                   g_psi=None, g_base=None, stream=None):
    """Transpose of pullback_u: accumulates into g_u0, g_T, g_psi, g_base (any may be None)."""
    _chk_mac(g, u0, "u0")
    _chk_mac(g, g_out, "g_out")
    check(_lib.lib().fm_pullback_u_adj(C.byref(g.c_grid()), _dt(u0[0]), dx, *_mac3(u0), *_mac3(T_f),
                                       *_mac3(psi_f), alpha, beta, *_mac3(g_out), *_mac_opt(g, g_u0, "g_u0"),
                                       *_mac3(g_T), *_mac3(g_psi), *_mac_opt(g, g_base, "g_base"),
                                       stream_ptr(stream)), "fm_pullback_u_adj")


def pullback_scalar_adj(g: GridSpec, dx: float, s0, psi, g_out, alpha=1.0, beta=0.0, g_s0=None, g_psi=None,
                        g_base=None, stream=None):
    """Transpose of pullback_scalar: accumulates into g_s0, g_psi, g_base (any may be None)."""
    check(_lib.lib().fm_pullback_scalar_adj(C.byref(g.c_grid()), _dt(s0), dx, ptr(s0), ptr(psi), alpha, beta,
                                            ptr(g_out), ptr(g_s0), ptr(g_psi), ptr(g_base), stream_ptr(stream)),
          "fm_pullback_scalar_adj")


def rk_grid_adj(g: GridSpec, rk: int, dx: float, dt: float, face: int, psi, T, u, g_psi_out, g_T_out=None,
                g_psi=None, g_T=None, g_u=None, stream=None):
    """Transpose of rk_grid at its inputs (psi, T, u): accumulates into g_psi, g_T, g_u."""
    _chk_mac(g, u, "u")
    _chk_vec(g, psi, face, "psi")
    check(_lib.lib().fm_rk_grid_adj(C.byref(g.c_grid()), _dt(psi), rk, dx, dt, face, ptr(psi), ptr(T), *_mac3(u),
                                    ptr(g_psi_out), ptr(g_T_out), ptr(g_psi), ptr(g_T), *_mac_opt(g, g_u, "g_u"),
                                    stream_ptr(stream)), "fm_rk_grid_adj")


def accumulate_init(g: GridSpec, dx: float, dt: float, f, init, F_f, phi_f, Hp=None, Hpp=None, ind=0, stream=None):
    ab3 = Hp is not None
    hs = []
    for c in range(3):
        hs += [ptr(Hp[c]) if ab3 and c < g.dim else None, ptr(Hpp[c]) if ab3 and c < g.dim else None]
    check(_lib.lib().fm_accumulate_init(C.byref(g.c_grid()), _dt(f[0]), dx, dt, int(ab3), ind, *_mac3(f),
                                        *_mac3(init), *_mac3(F_f), *_mac3(phi_f), *hs, stream_ptr(stream)),
          "fm_accumulate_init")


def accumulate_init_pair(g: GridSpec, dx: float, dt: float, f, init, F_f, phi_f, f2, dt2: float, Hp=None, Hpp=None,
                         ind=0, stream=None):
    """accumulate_init(f, dt, ...) then a plain accumulate_init(f2, dt2) through the same maps, in one pass."""
    _chk_mac(g, f2, "f2")
    ab3 = Hp is not None
    hs = []
    for c in range(3):
        hs += [ptr(Hp[c]) if ab3 and c < g.dim else None, ptr(Hpp[c]) if ab3 and c < g.dim else None]
    check(_lib.lib().fm_accumulate_init_pair(C.byref(g.c_grid()), _dt(f[0]), dx, dt, int(ab3), ind, *_mac3(f),
                                             *_mac3(init), *_mac3(F_f), *_mac3(phi_f), *hs, *_mac3(f2), dt2,
                                             stream_ptr(stream)), "fm_accumulate_init_pair")


def nabla_u_w(g: GridSpec, dx: float, u, w, r, order: Optional[int] = None, stream=None):
    if order is None:
        order = 3 if g.dim == 3 else 4
    check(_lib.lib().fm_nabla_u_w(C.byref(g.c_grid()), _dt(u[0]), order, dx, *_mac3(u), *_mac3(w), *_mac3(r),
                                  stream_ptr(stream)), "fm_nabla_u_w")


def nabla_scalar_adjoint(g: GridSpec, dx: float, s, adj, r, stream=None):
    check(_lib.lib().fm_nabla_scalar_adjoint(C.byref(g.c_grid()), _dt(s), dx, ptr(s), ptr(adj), *_mac3(r),
                                             stream_ptr(stream)), "fm_nabla_scalar_adjoint")


def reset_to_identity(g: GridSpec, dx: float, psi_c, psi_f, T_f, stream=None):
    t = psi_c if psi_c is not None else (psi_f[0] if psi_f else T_f[0])
    check(_lib.lib().fm_reset_to_identity(C.byref(g.c_grid()), _dt(t), dx, ptr(psi_c), *_mac3(psi_f), *_mac3(T_f),
                                          stream_ptr(stream)), "fm_reset_to_identity")


def add_fields(f1, f2, dest, m: float, stream=None):
    """dest = f1 + m * f2 (elementwise, same shapes)."""
    if f1.shape != f2.shape or f1.shape != dest.shape:
        raise _lib.FlowmapError(1, "add_fields shape mismatch")
    check(_lib.lib().fm_add_fields(_dt(dest), dest.numel(), ptr(f1), ptr(f2), ptr(dest), m, stream_ptr(stream)),
          "fm_add_fields")


def convert(src, dst, stream=None):
    """dst = src with a dtype change (FP32/FP64/BF16), elementwise."""
    if src.numel() != dst.numel():
        raise _lib.FlowmapError(1, "convert size mismatch")
    check(_lib.lib().fm_convert(src.numel(), dtype_code(src.dtype, True), ptr(src), dtype_code(dst.dtype, True),
                                ptr(dst), stream_ptr(stream)), "fm_convert")


def clamp_extrema(g: GridSpec, src, ref, dst, stream=None):
    """dst = clamp(src, extrema of ref over the axis neighbours) (clamp_u); grid inferred from the shape."""
    face = g.which_grid(src)
    if ref.shape != src.shape or dst.shape != src.shape or ref.dtype != src.dtype or dst.dtype != src.dtype:
        raise _lib.FlowmapError(1, "clamp_extrema: src, ref and dst must share shape and dtype")
    if dst.data_ptr() == ref.data_ptr():
        raise _lib.FlowmapError(2, "clamp_extrema: dst may not alias ref")
    check(_lib.lib().fm_clamp_extrema(C.byref(g.c_grid()), _dt(src), face, ptr(src), ptr(ref), ptr(dst),
                                      stream_ptr(stream)), "fm_clamp_extrema")


def store(src, dst, stream=None):
    """Copy into a trajectory store slot: device memcpy when dtypes match, else fm_convert."""
    if src.dtype == dst.dtype:
        dst.copy_(src)
    else:
        convert(src, dst, stream)


def laplacian(g: GridSpec, p, Ap, stream=None):
    check(_lib.lib().fm_laplacian(C.byref(g.c_grid()), _dt(p), ptr(p), ptr(Ap), stream_ptr(stream)), "fm_laplacian")


# ---------------------------------------------------------------------------
# 2D vortex problem
# ---------------------------------------------------------------------------
def _theta_arg(theta):
    import numpy as _np

    th = _np.ascontiguousarray(_np.asarray(theta, dtype=_np.float64))
    if th.ndim != 1 or th.size % 3 != 0:
        raise _lib.FlowmapError(2, "theta must hold 3K values [w.., cx.., cy..]")
    return th, th.size // 3, th.ctypes.data_as(C.POINTER(C.c_double))


def vortex_velocity_2d(g: GridSpec, dx: float, theta, ux, uy, stream=None):
    """Faces of the point-vortex velocity of theta (split_central_vector of the centre values)."""
    _chk_mac(g, (ux, uy), "u")
    th, nv, tp = _theta_arg(theta)
    check(_lib.lib().fm_vortex_velocity_2d(C.byref(g.c_grid()), _dt(ux), dx, nv, tp, ptr(ux), ptr(uy),
                                           stream_ptr(stream)), "fm_vortex_velocity_2d")


def vortex_velocity_grad_2d(g: GridSpec, dx: float, theta, lam_x, lam_y, stream=None):
    """d<lam, u(theta)>/d theta as a device FP64 tensor of 3K entries."""
    th, nv, tp = _theta_arg(theta)
    work = torch.empty(592 * 3 * nv, dtype=torch.float64, device=lam_x.device)
    grad = torch.empty(3 * nv, dtype=torch.float64, device=lam_x.device)
    check(_lib.lib().fm_vortex_velocity_grad_2d(C.byref(g.c_grid()), _dt(lam_x), dx, nv, tp, ptr(lam_x), ptr(lam_y),
                                                ptr(work), ptr(grad), stream_ptr(stream)),
          "fm_vortex_velocity_grad_2d")
    return grad


def vorticity_2d(g: GridSpec, dx: float, ux, uy, omega, stream=None):
    _chk_mac(g, (ux, uy), "u")
    check(_lib.lib().fm_vorticity_2d(C.byref(g.c_grid()), _dt(ux), dx, ptr(ux), ptr(uy), ptr(omega),
                                     stream_ptr(stream)), "fm_vorticity_2d")


def vorticity_loss_2d(g: GridSpec, dx: float, ux, uy, omega_target, lam_x, lam_y, work, part, loss, stream=None):
    """loss (device FP64, 1 entry) = sum (omega - omega*)^2; lam = (d omega/d u)^T 2 (omega - omega*)."""
    _chk_mac(g, (ux, uy), "u")
    check(_lib.lib().fm_vorticity_loss_2d(C.byref(g.c_grid()), _dt(ux), dx, ptr(ux), ptr(uy), ptr(omega_target),
                                          ptr(work), ptr(part), ptr(lam_x), ptr(lam_y), ptr(loss), stream_ptr(stream)),
          "fm_vorticity_loss_2d")


def _chk_gaussians(g: GridSpec, center, inv_radius, strength, dtype):
    n = int(inv_radius.shape[0])
    for name, t, shape in (("center", center, (n, g.dim)), ("inv_radius", inv_radius, (n,)),
                           ("strength", strength, (n, g.dim))):
        if tuple(t.shape) != shape:
            raise _lib.FlowmapError(1, f"{name} has shape {tuple(t.shape)}, expected {shape}")
        if t.dtype != dtype:
            raise _lib.FlowmapError(7, f"{name} is {t.dtype}, the fields are {dtype}")
    return n


def gaussian_force(g: GridSpec, dx: float, center, inv_radius, strength, f, stream=None):
    """apply_gausion_force_kernel: every face of ``f`` = the sum of the Gaussians
    reaching it (device parameter tensors: center n x dim, inv_radius n, strength n x dim)."""
    _chk_mac(g, f, "f")
    n = _chk_gaussians(g, center, inv_radius, strength, f[0].dtype)
    check(_lib.lib().fm_gaussian_force(C.byref(g.c_grid()), _dt(f[0]), dx, n, ptr(center), ptr(inv_radius),
                                       ptr(strength), *_mac3(f), stream_ptr(stream)), "fm_gaussian_force")


def gaussian_force_grad(g: GridSpec, dx: float, center, inv_radius, strength, adj_u, out=None, stream=None):
    """calculate_adj_gausion_force_kernel: (adj_center, adj_strength, penalty_center,
    penalty_strength), device FP64 tensors of shape n x dim (written into ``out`` if given)."""
    _chk_mac(g, adj_u, "adj_u")
    n = _chk_gaussians(g, center, inv_radius, strength, adj_u[0].dtype)
    if out is None:
        out = tuple(torch.empty((n, g.dim), dtype=torch.float64, device=adj_u[0].device) for _ in range(4))
    for t in out:
        if t.dtype != torch.float64 or tuple(t.shape) != (n, g.dim):
            raise _lib.FlowmapError(1, "gaussian_force_grad outputs are FP64 n x dim")
    check(_lib.lib().fm_gaussian_force_grad(C.byref(g.c_grid()), _dt(adj_u[0]), dx, n, ptr(center), ptr(inv_radius),
                                            ptr(strength), *_mac3(adj_u), *[ptr(t) for t in out],
                                            stream_ptr(stream)), "fm_gaussian_force_grad")
    return out


def viscous_force_2d(g: GridSpec, nu: float, dx: float, u, vis, adj=None, part=None, dot=None, stream=None):
    """calculate_viscous_force into ``vis``; with ``adj`` also dot += sum adj . vis / nu
    (calculate_viscous_force_adj; ``part``: FP64 scratch of 592, ``dot``: FP64 device scalar)."""
    _chk_mac(g, u, "u")
    _chk_mac(g, vis, "vis")
    a = [None, None]
    if adj is not None:
        _chk_mac(g, adj, "adj")
        a = [ptr(adj[0]), ptr(adj[1])]
    check(_lib.lib().fm_viscous_force_2d(C.byref(g.c_grid()), _dt(u[0]), nu, dx, ptr(u[0]), ptr(u[1]), ptr(vis[0]),
                                         ptr(vis[1]), a[0], a[1], ptr(part), ptr(dot), stream_ptr(stream)),
          "fm_viscous_force_2d")


def _mask_arg(g: GridSpec, mask):
    if tuple(mask.shape) != tuple(g.shape) or mask.dtype != torch.float32:
        raise _lib.FlowmapError(1, "mask: float32 cell-grid tensor expected")
    return ptr(mask)


def mask_velocity(g: GridSpec, mask, u, bvel=None, stream=None):
    """mask_velocity_by_boundary (bvel: (dim, *grid) tensor of u's dtype) or, with
    bvel None, mask_adj_velocity_by_boundary (zero on the faces of solid cells)."""
    _chk_mac(g, u, "u")
    if bvel is not None:
        _chk_vec(g, bvel, -1, "bvel")
    check(_lib.lib().fm_mask_velocity(C.byref(g.c_grid()), _dt(u[0]), _mask_arg(g, mask), ptr(bvel), *_mac3(u),
                                      stream_ptr(stream)), "fm_mask_velocity")


def mask_passive(g: GridSpec, mask, s, adjoint: bool = False, stream=None):
    """mask_passive_by_boundary, or mask_adj_passive_by_boundary with adjoint=True."""
    check(_lib.lib().fm_mask_passive(C.byref(g.c_grid()), _dt(s), _mask_arg(g, mask), ptr(s), int(adjoint),
                                     stream_ptr(stream)), "fm_mask_passive")
