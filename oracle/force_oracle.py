"""Numpy restatement of the reference's Gaussian control forces and their
parameter adjoint -- TEST INFRASTRUCTURE ONLY (the oracle): the product path
never imports this module.

Parity unpinned: the reference ships no golden vectors for these kernels; the
restatement follows the reference code line by line, in the arithmetic type
of the run (float32 or float64), with the per-face operation order of:

* apply_gausion_force_kernel (3D/lfm_midpoint_simulator.py:316-344,
  2D/shape/lfm_midpoint_simulator.py:282-299): f.fill(0), then for each face
  and each Gaussian I in ascending order, if |p - c_I|^2 r_I < 5:
  f += exp(-d^2 r_I) s_I[c] with d = |p - c_I|.
* calculate_adj_gausion_force_kernel (3D/lfm_midpoint_diff_simulator.py:71-110,
  2D/shape/lfm_midpoint_diff_simulator.py:75-103): per Gaussian, sums over the
  faces it reaches.  The reference accumulates with atomics (order undefined);
  here the per-face terms are summed in float64.

The per-face test is evaluated as d = sqrt(sum (p - c)^2), q = (d * d) * r,
q < 5, without fused multiply-adds, as the CUDA kernels do.
"""
import numpy as np


def face_positions(res, c, dx, dtype):
    """X_c of the reference (3D/taichi_utils.py:95-128): axis c at i*dx, the
    others at (i + 0.5)*dx, in the run's arithmetic type; broadcastable axes."""
    dim = len(res)
    out = []
    for a in range(dim):
        n = res[a] + (1 if a == c else 0)
        i = np.arange(n).astype(dtype)
        x = (i if a == c else i + dtype(0.5)) * dtype(dx)
        shape = [1] * dim
        shape[a] = n
        out.append(x.reshape(shape))
    return out


def _weight(P, c, r, dtype):
    dp = [P[a] - c[a] for a in range(len(P))]
    s2 = dp[0] * dp[0]
    for a in range(1, len(P)):
        s2 = s2 + dp[a] * dp[a]
    with np.errstate(invalid="ignore", over="ignore"):
        d = np.sqrt(s2)
        q = (d * d) * r
        m = q < dtype(5)
        e = np.exp(-np.where(m, q, dtype(0))).astype(dtype)
    return m, e, dp


def gaussian_force(res, dx, center, inv_radius, strength):
    """Face forces f_c (list of arrays of the parameters' dtype)."""
    dtype = center.dtype.type
    dim = len(res)
    f = []
    for c in range(dim):
        P = face_positions(res, c, dx, dtype)
        shape = tuple(res[a] + (1 if a == c else 0) for a in range(dim))
        fc = np.zeros(shape, dtype=dtype)
        for I in range(inv_radius.shape[0]):
            m, e, _ = _weight(P, center[I], inv_radius[I], dtype)
            m = np.broadcast_to(m, shape)
            fc[m] = fc[m] + np.broadcast_to(e, shape)[m] * strength[I, c]
        f.append(fc)
    return f


def gaussian_force_grad(res, dx, center, inv_radius, strength, adj):
    """(adj_center, adj_strength, penalty_center, penalty_strength), float64 n x dim."""
    dtype = center.dtype.type
    dim = len(res)
    n = inv_radius.shape[0]
    adj_c, adj_s = np.zeros((n, dim)), np.zeros((n, dim))
    pen_c, pen_s = np.zeros((n, dim)), np.zeros((n, dim))
    two = dtype(2)
    for c in range(dim):
        P = face_positions(res, c, dx, dtype)
        shape = adj[c].shape
        for I in range(n):
            m, e, dp = _weight(P, center[I], inv_radius[I], dtype)
            m = np.broadcast_to(m, shape)
            if not m.any():
                continue
            e = np.broadcast_to(e, shape)[m]
            a = adj[c][m]
            r, s = inv_radius[I], strength[I, c]
            f = e * s
            adj_s[I, c] += np.sum((e * a).astype(np.float64))
            pen_s[I, c] += np.sum(((two * f) * e).astype(np.float64))
            ga = (s * e) * two
            gp = (((two * f) * s) * e) * two
            for b in range(dim):
                d = np.broadcast_to(dp[b], shape)[m]
                adj_c[I, b] += np.sum((((ga * d) * r) * a).astype(np.float64))
                pen_c[I, b] += np.sum(((gp * d) * r).astype(np.float64))
    return adj_c, adj_s, pen_c, pen_s


def random_gaussians(n, dim, dx, seed, dtype=np.float64):
    """Seeded synthetic parameters shaped as the reference's optimisers draw them:
    2D (2D/shape/optimize_shape_G_R.py:20-52): inverse radii 1/(k dx)^2 with k
    from {1..6, 8, 9, 10}, centres uniform in [0.2, 0.8]^2, strength magnitude
    U(5e-3, 2e-2) * 2 in a uniform direction; 3D (3D/optimize_shape_G_R.py:20-53):
    k from {1, 1, 1, 1, 2..9}, centres uniform in [0, 1]^3.  The 3D optimiser
    starts from zero strengths (a zero force); here 3D strengths are drawn like
    the 2D ones, in a uniform direction on the sphere, so the force is not zero."""
    rng = np.random.default_rng(seed)
    if dim == 2:
        ks, lo, hi = np.array([1, 2, 3, 4, 5, 6, 8, 9, 10], dtype=np.float64), 0.2, 0.8
    else:
        ks, lo, hi = np.array([1, 1, 1, 1, 2, 3, 4, 5, 6, 7, 8, 9], dtype=np.float64), 0.0, 1.0
    inv_r = 1.0 / (rng.choice(ks, size=n) * dx) ** 2
    center = rng.uniform(lo, hi, size=(n, dim))
    mag = rng.uniform(5e-3, 2e-2, size=n) * 2.0
    if dim == 2:
        ang = rng.uniform(0, 2 * np.pi, size=n)
        strength = np.stack([mag * np.cos(ang), mag * np.sin(ang)], axis=1)
    else:
        v = rng.normal(size=(n, 3))
        strength = mag[:, None] * v / np.linalg.norm(v, axis=1, keepdims=True)
    return center.astype(dtype), inv_r.astype(dtype), strength.astype(dtype)
