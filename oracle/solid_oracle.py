"""Numpy restatement of the reference's obstacle path -- TEST INFRASTRUCTURE
ONLY (the oracle): the solid-aware MGPCG and the mask kernels.  The product
path never imports this module.

Parity unpinned: the reference ships no golden vectors for these routines; the
restatement follows, in the run's arithmetic type:

* MGPCG with a boundary mask (2D/vortex/mgpcg_solid.py:14-367, the 2D class
  MGPCG_2_solid :370-458): coarse masks by downsample_bm (a coarse cell is solid
  only when all its 2^dim children are, :114-127); the operator, the red-black
  Gauss-Seidel smoother, the residual restriction and the PCG updates act on
  fluid cells only, with neighbour counts and sums over in-domain fluid
  neighbours (:141-172); the restricted residual is scaled by 1/(dim-1) (:225);
  prolongation adds to every cell (:228-231); recentring subtracts the mean over
  all cells, solid ones included (:241-247).  The reference scatters the
  restriction with atomics (order undefined); here a coarse cell sums its
  children in lexicographic order (as the CUDA kernel does), and the PCG inner
  products are float64.
* apply_bc / divergence / subtract_grad_p with the mask (:383-445): the faces of
  solid cells and the domain walls are zeroed, the divergence of a solid cell
  is 0.
* mask_velocity_by_boundary / mask_passive_by_boundary and their adjoint forms
  (2D/vortex/init_conditions.py:549-583, 3D/init_conditions.py:536-578).  Where
  two adjacent solid cells write one face with different boundary velocities
  the reference races; here the cell on the face's high side wins, as in the
  CUDA kernel.
"""
import itertools

import numpy as np


def _axes_shift(x, a, d):
    """x shifted by d (+1 or -1) along axis a, with a validity mask."""
    n = x.shape[a]
    idx = np.arange(n) + d
    ok = (idx >= 0) & (idx < n)
    idx = np.clip(idx, 0, n - 1)
    shape = [1] * x.ndim
    shape[a] = n
    return np.take(x, idx, axis=a), ok.reshape(shape)


def downsample(fluid_fine):
    """downsample_bm: coarse solid iff every child is solid (fluid_fine: bool)."""
    dim = fluid_fine.ndim
    any_fluid = np.zeros(tuple(n // 2 for n in fluid_fine.shape), dtype=bool)
    for off in itertools.product((0, 1), repeat=dim):
        any_fluid |= fluid_fine[tuple(slice(o, None, 2) for o in off)]
    return any_fluid


def _nbr(z, fluid):
    """(count, sum) over in-domain fluid neighbours, summed per axis right then left."""
    t = z.dtype.type
    s = np.zeros_like(z)
    n = np.zeros_like(z)
    for a in range(z.ndim):
        for d in (1, -1):
            v, ok = _axes_shift(z, a, d)
            f, _ = _axes_shift(fluid, a, d)
            m = ok & f
            s = np.where(m, s + v, s)
            n = n + m.astype(z.dtype)
    return n.astype(z.dtype), s


def smooth(z, r, fluid, phase):
    t = z.dtype.type
    parity = sum(np.indices(z.shape)) & 1
    n, s = _nbr(z, fluid)
    with np.errstate(divide="ignore", invalid="ignore"):
        new = (r + s) / n
    upd = fluid & (parity == phase)
    z[upd] = new[upd].astype(z.dtype)


def restrict(z, r, fluid):
    """Coarse residual (children summed in lexicographic order, scaled by 1/(dim-1))."""
    dim = z.ndim
    t = z.dtype.type
    n, s = _nbr(z, fluid)
    res = r - (n * z - s)
    scale = t(1.0 / (dim - 1.0))
    rc = np.zeros(tuple(m // 2 for m in z.shape), dtype=z.dtype)
    for off in itertools.product((0, 1), repeat=dim):
        sl = tuple(slice(o, None, 2) for o in off)
        rc = np.where(fluid[sl], rc + res[sl] * scale, rc)
    return rc


def prolong(z, zc):
    for off in itertools.product((0, 1), repeat=z.ndim):
        sl = tuple(slice(o, None, 2) for o in off)
        z[sl] = z[sl] + zc


def masks(fluid0, levels):
    out = [fluid0]
    for _ in range(1, levels):
        out.append(downsample(out[-1]))
    return out


def vcycle(r0, fluid0, levels, pre_post=2, bottom=20):
    """apply_preconditioner (bottom smoothing as bottom/2 x (R,B) then bottom/2 x (B,R))."""
    fl = masks(fluid0, levels)
    r = [r0.copy()]
    z = [np.zeros_like(r0)]
    for l in range(levels - 1):
        for _ in range(pre_post):
            smooth(z[l], r[l], fl[l], 0)
            smooth(z[l], r[l], fl[l], 1)
        r.append(restrict(z[l], r[l], fl[l]))
        z.append(np.zeros_like(r[-1]))
    L = levels - 1
    for _ in range(bottom // 2):
        smooth(z[L], r[L], fl[L], 0)
        smooth(z[L], r[L], fl[L], 1)
    for _ in range(bottom // 2):
        smooth(z[L], r[L], fl[L], 1)
        smooth(z[L], r[L], fl[L], 0)
    for l in reversed(range(levels - 1)):
        prolong(z[l], z[l + 1])
        for _ in range(pre_post):
            smooth(z[l], r[l], fl[l], 1)
            smooth(z[l], r[l], fl[l], 0)
    return z[0]


def apply_A(p, fluid):
    n, s = _nbr(p, fluid)
    return np.where(fluid, n * p - s, 0).astype(p.dtype)


def solve(b, fluid0, levels, max_iters=400, abs_tol=1e-14, rel_tol=1e-16, eps=1e-12, pre_post=2, bottom=20,
          k=1.0):
    """MGPCG.solve on A x = k b (solve(), :249-367); returns (x, iterations, rTr)."""
    t = b.dtype.type
    N = b.size
    r = (b * t(k)).astype(b.dtype)
    x = np.zeros_like(b)
    p = np.zeros_like(b)
    fl = fluid0

    def dot(a, c):
        return float(np.sum((a.astype(np.float64) * c.astype(np.float64))[fl]))

    def recenter():
        r[...] = r - t(float(np.sum(r.astype(np.float64))) / N)

    recenter()
    z = vcycle(r, fl, levels, pre_post, bottom)
    p[fl] = z[fl]                                # update_p with p = 0
    old = dot(z, r)
    tol = max(abs_tol, old * rel_tol)
    it = 0
    rtr = old
    while it < max_iters:
        Ap = apply_A(p, fl)
        alpha = t(old / (dot(p, Ap) + eps))
        x[fl] = (x + alpha * p)[fl]
        r[fl] = (r - alpha * Ap)[fl]
        rtr = dot(r, r)
        if rtr < tol:
            return x, it, rtr
        recenter()
        z = vcycle(r, fl, levels, pre_post, bottom)
        new = dot(z, r)
        beta = t(new / (old + eps))
        p[fl] = (z + beta * p)[fl]
        old = new
        it += 1
    return x, it, rtr


def faces_of_solids(fluid, c):
    """Boolean mask of the component-c faces touching a solid cell."""
    solid = ~fluid
    shape = list(solid.shape)
    shape[c] += 1
    out = np.zeros(shape, dtype=bool)
    lo = [slice(None)] * solid.ndim
    hi = [slice(None)] * solid.ndim
    lo[c] = slice(0, -1)
    hi[c] = slice(1, None)
    out[tuple(lo)] |= solid
    out[tuple(hi)] |= solid
    return out


def apply_bc(u, fluid):
    for c, x in enumerate(u):
        sl = [slice(None)] * x.ndim
        sl[c] = 0
        x[tuple(sl)] = 0
        sl[c] = -1
        x[tuple(sl)] = 0
        x[faces_of_solids(fluid, c)] = 0


def divergence(u, fluid):
    acc = None
    for c, x in enumerate(u):
        lo = [slice(None)] * x.ndim
        hi = [slice(None)] * x.ndim
        lo[c] = slice(0, -1)
        hi[c] = slice(1, None)
        vl, vr = x[tuple(lo)], x[tuple(hi)]
        acc = vr - vl if acc is None else (acc + vr) - vl
    return np.where(fluid, acc, 0).astype(u[0].dtype)


def subtract_grad_p(u, p):
    for c, x in enumerate(u):
        n = p.shape[c]
        pad = [(0, 0)] * p.ndim
        pad[c] = (1, 1)
        pp = np.pad(p, pad)  # p = 0 outside: walls are zeroed by the apply_bc that follows
        lo = [slice(None)] * p.ndim
        hi = [slice(None)] * p.ndim
        lo[c] = slice(0, n + 1)
        hi[c] = slice(1, n + 2)
        x[...] = x - (pp[tuple(hi)] - pp[tuple(lo)])


def project(u, mask, levels, **kw):
    """MGPCG_2_solid.Poisson (:447-458): apply_bc, divergence, solve with k = -1,
    subtract_grad_p, apply_bc.  mask: cell array, solid where > 0."""
    fluid = ~(mask > 0)
    apply_bc(u, fluid)
    div = divergence(u, fluid)
    x, it, rtr = solve(div, fluid, levels, k=-1.0, **kw)
    subtract_grad_p(u, x)
    apply_bc(u, fluid)
    return x, it, rtr


def mask_velocity(u, mask, bvel=None):
    """mask_velocity_by_boundary (adjoint form: bvel=None gives 0)."""
    solid = mask >= 1
    for c, x in enumerate(u):
        val = np.zeros(solid.shape, dtype=x.dtype) if bvel is None else bvel[c].astype(x.dtype)
        lo = [slice(None)] * x.ndim
        hi = [slice(None)] * x.ndim
        lo[c] = slice(0, -1)
        hi[c] = slice(1, None)
        # the low-side cell first, the high-side cell (whose low face it is) wins
        x[tuple(hi)] = np.where(solid, val, x[tuple(hi)])
        x[tuple(lo)] = np.where(solid, val, x[tuple(lo)])


def mask_passive(s, mask):
    """mask_passive_by_boundary: a solid cell takes the mean of its fluid 3^dim
    neighbours (summed in lexicographic offset order), or 0."""
    solid = mask >= 1
    fluid = mask <= 0
    t = s.dtype.type
    acc = np.zeros_like(s)
    w = np.zeros_like(s)
    for off in itertools.product((-1, 0, 1), repeat=s.ndim):
        v, f, ok = s, fluid, np.ones(s.shape, dtype=bool)
        for a, d in enumerate(off):
            if d:
                v, o1 = _axes_shift(v, a, d)
                f, _ = _axes_shift(f, a, d)
                ok = ok & o1
        m = ok & f
        acc = np.where(m, acc + v, acc)
        w = w + m.astype(s.dtype)
    with np.errstate(divide="ignore", invalid="ignore"):
        avg = np.where(w > 0, acc / w, acc)
    s[solid] = avg[solid].astype(s.dtype)


def mask_adj_passive(s, mask):
    s[mask >= 1] = 0
