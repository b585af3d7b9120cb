"""CPU restatement of the 2D vortex problem's control map and vorticity loss.
TEST INFRASTRUCTURE ONLY: the parity checker for fm_vortex_velocity_2d,
fm_vortex_velocity_grad_2d, fm_vorticity_2d and fm_vorticity_loss_2d; never
used by the product.

  angular_vel_func            2D/vortex/init_conditions.py:142-145
  per-vortex velocity sum     2D/vortex/init_conditions.py:386-414 (core 0.02,
                              strength -0.01 * w; vf = first term, += the rest)
  split_central_vector        2D/vortex/taichi_utils.py:158-167 (clamped sample)
  get_central_vector, curl    2D/vortex/taichi_utils.py:153-156, 199-205
  calculate_dtheta_ind        2D/vortex/optimize_vortex.py:193-220 (finite
                              differences of the init map, epsilon 1e-5,
                              contracted with the adjoint velocity)
theta = [w_0..w_{K-1}, cx_0..cx_{K-1}, cy_0..cy_{K-1}].
"""
from __future__ import annotations

import numpy as np

CORE, STRENGTH = 0.02, -0.01


def angular_vel_func(r, rad, strength):
    r = r + r.dtype.type(1e-6)
    one = r.dtype.type(1.0)
    linear_vel = strength * (one / r) * (one - np.exp(-(r * r) / (rad * rad)))
    return (one / r) * linear_vel


def vortex_central(theta, n, dx, dtype=np.float64):
    """Velocity at the cell centres (2, n0, n1) in `dtype` arithmetic."""
    t = np.dtype(dtype).type
    n0, n1 = n
    K = len(theta) // 3
    X = (np.arange(n0, dtype=dtype)[:, None] + t(0.5)) * t(dx)
    Y = (np.arange(n1, dtype=dtype)[None, :] + t(0.5)) * t(dx)
    X, Y = np.broadcast_arrays(X, Y)
    vx = np.zeros((n0, n1), dtype)
    vy = np.zeros((n0, n1), dtype)
    for k in range(K):
        w, cx, cy = t(theta[k]), t(theta[K + k]), t(theta[2 * K + k])
        px, py = X - cx, Y - cy
        r = np.sqrt(px * px + py * py)
        fw = angular_vel_func(r, t(CORE), t(STRENGTH)) * w
        vx = vx + fw * -py
        vy = vy + fw * px
    return np.stack([vx, vy])


def split_central_vector(vc):
    """Cell centres -> faces, clamped samples: u_x[i] = 0.5 (c[i] + c[i-1])."""
    t = vc.dtype.type
    cx, cy = vc
    lo = np.concatenate([cx[:1], cx], axis=0)
    hi = np.concatenate([cx, cx[-1:]], axis=0)
    ux = t(0.5) * (hi + lo)
    lo = np.concatenate([cy[:, :1], cy], axis=1)
    hi = np.concatenate([cy, cy[:, -1:]], axis=1)
    uy = t(0.5) * (hi + lo)
    return [ux, uy]


def vortex_faces(theta, n, dx, dtype=np.float64):
    return split_central_vector(vortex_central(theta, n, dx, dtype))


def central(ux, uy):
    t = ux.dtype.type
    return t(0.5) * (ux[1:] + ux[:-1]), t(0.5) * (uy[:, 1:] + uy[:, :-1])


def vorticity(ux, uy, dx):
    """curl with clamped samples of the centre velocity: (vr.y - vl.y - vt.x + vb.x) / (2 dx)."""
    t = ux.dtype.type
    cx, cy = central(ux, uy)
    n0, n1 = cx.shape
    ip = np.minimum(np.arange(n0) + 1, n0 - 1)
    im = np.maximum(np.arange(n0) - 1, 0)
    jp = np.minimum(np.arange(n1) + 1, n1 - 1)
    jm = np.maximum(np.arange(n1) - 1, 0)
    vr_y, vl_y = cy[ip, :], cy[im, :]
    vt_x, vb_x = cx[:, jp], cx[:, jm]
    return (vr_y - vl_y - vt_x + vb_x) / (t(2) * t(dx))


def vorticity_loss(ux, uy, omega_t, dx):
    d = vorticity(ux, uy, dx).astype(np.float64) - np.asarray(omega_t, np.float64)
    return float(np.sum(d * d))


def vorticity_adjoint(g, dx):
    """(d omega / d u)^T g by explicit scatter (FP64): faces (n0+1, n1), (n0, n1+1)."""
    g = np.asarray(g, np.float64)
    n0, n1 = g.shape
    h = 1.0 / (2.0 * dx)
    gcx = np.zeros((n0, n1))
    gcy = np.zeros((n0, n1))
    for a in range(n0):
        np.add.at(gcy, (min(a + 1, n0 - 1), slice(None)), g[a] * h)
        np.add.at(gcy, (max(a - 1, 0), slice(None)), -g[a] * h)
    for b in range(n1):
        np.add.at(gcx, (slice(None), min(b + 1, n1 - 1)), -g[:, b] * h)
        np.add.at(gcx, (slice(None), max(b - 1, 0)), g[:, b] * h)
    lx = np.zeros((n0 + 1, n1))
    ly = np.zeros((n0, n1 + 1))
    lx[1:] += 0.5 * gcx
    lx[:-1] += 0.5 * gcx
    ly[:, 1:] += 0.5 * gcy
    ly[:, :-1] += 0.5 * gcy
    return [lx, ly]


def split_adjoint(lx, ly):
    lx = np.asarray(lx, np.float64)
    ly = np.asarray(ly, np.float64)
    gx = 0.5 * (lx[:-1] + lx[1:])
    gx[0] += 0.5 * lx[0]
    gx[-1] += 0.5 * lx[-1]
    gy = 0.5 * (ly[:, :-1] + ly[:, 1:])
    gy[:, 0] += 0.5 * ly[:, 0]
    gy[:, -1] += 0.5 * ly[:, -1]
    return gx, gy


def theta_grad_fd(theta, lam, n, dx, eps=1e-5):
    """calculate_dtheta (2D/vortex/optimize_vortex.py:193-220) in FP64: forward
    differences of the init map (no projection), contracted with lam."""
    base = vortex_faces(theta, n, dx)
    out = []
    for i in range(len(theta)):
        th = np.array(theta, np.float64)
        th[i] += eps
        pert = vortex_faces(th, n, dx)
        out.append(float(sum(np.sum(np.asarray(l, np.float64) * (p - b) / eps) for l, p, b in zip(lam, pert, base))))
    return np.array(out)


def theta_grad(theta, lam, n, dx, h=1e-7):
    """The same contraction with central differences of the centre velocity
    (step h), far more accurate than the reference's forward differences."""
    gx, gy = split_adjoint(*lam)
    out = []
    for i in range(len(theta)):
        tp = np.array(theta, np.float64)
        tm = tp.copy()
        tp[i] += h
        tm[i] -= h
        d = (vortex_central(tp, n, dx) - vortex_central(tm, n, dx)) / (2 * h)
        out.append(float(np.sum(gx * d[0]) + np.sum(gy * d[1])))
    return np.array(out)
