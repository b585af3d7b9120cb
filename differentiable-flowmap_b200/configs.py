"""Workload presets and seeded synthetic inputs.

The reference optimises real experiments (Gaussian control forces, image
masks); the benchmark configurations below use seeded synthetic inputs of the
same shapes instead (numpy PCG64 generators, seeds fixed per config).
"""
from __future__ import annotations

import math
import os
from dataclasses import replace

import numpy as np
import torch

from .simulator import FlowmapConfig, SolverConfig


def split_central_vector(vc: np.ndarray) -> list:
    """Cell-centred vector (dim, *res) -> MAC faces, clamped sampling
    (3D/taichi_utils.py:170-183, 2D/vortex/taichi_utils.py:158-167)."""
    dim = vc.shape[0]
    out = []
    for c in range(dim):
        v = vc[c]
        lo = np.concatenate([v.take([0], axis=c), v], axis=c)      # index i-1 clamped
        hi = np.concatenate([v, v.take([-1], axis=c)], axis=c)     # index i clamped
        out.append(0.5 * (hi + lo))
    return out


def smooth_ball(res, center, radius, dx):
    """Sphere/disc density with a one-cell tanh edge."""
    axes = [(np.arange(n) + 0.5) * dx for n in res]
    X = np.meshgrid(*axes, indexing="ij")
    r = np.sqrt(sum((x - c) ** 2 for x, c in zip(X, center)))
    return 0.5 * (1.0 - np.tanh((r - radius) / dx))


def shape3d_config(res=128, steps=150, reinit_every=8, rk=4, dtype=torch.float32, store_dtype=None,
                   backward_u=True, rel_tol=1e-6, abs_tol=0.0, max_iters=400, check_every=0, coarse_bf16=False):
    """3D smoke shape transition, 128^3: 150 steps, reinit every 8, RK4,
    dt = 0.0085 (3D/hyperparameters.py:268-295 with the stated overrides)."""
    n = int(math.log2(res))
    solver = SolverConfig(base_level=3, levels=n - 3 + 1, bottom=50, bottom_mode=0, max_iters=max_iters,
                          abs_tol=abs_tol, rel_tol=rel_tol, eps=1e-12 if dtype == torch.float32 else 0.0,
                          check_every=check_every, coarse_bf16=coarse_bf16)
    return FlowmapConfig(res=(res, res, res), dx=1.0 / res, dt=0.0085, total_steps=steps,
                         reinit_every=reinit_every, RK_number=rk, backward_u=backward_u, add_passive_scalar=True,
                         dtype=dtype, store_dtype=store_dtype, solver=solver)


def shape3d_inputs(res=128, seed_target=20, seed_u=21, u_std=0.01):
    """rho0: sphere r=0.15 at the centre; rho*: union of two spheres with radii
    U[0.08, 0.14], centres U[0.3, 0.7]^3; u0 cell-centred N(0, u_std^2) split to faces."""
    dx = 1.0 / res
    shape = (res, res, res)
    rho0 = smooth_ball(shape, (0.5, 0.5, 0.5), 0.15, dx)
    rng = np.random.default_rng(seed_target)
    radii = rng.uniform(0.08, 0.14, size=2)
    centers = rng.uniform(0.3, 0.7, size=(2, 3))
    rho_t = np.maximum(smooth_ball(shape, centers[0], radii[0], dx), smooth_ball(shape, centers[1], radii[1], dx))
    rng = np.random.default_rng(seed_u)
    uc = rng.normal(0.0, u_std, size=(3,) + shape)
    u0 = split_central_vector(uc)
    return u0, rho0, rho_t


# ---------------------------------------------------------------------------
# The reference's own data files (copied into tests/golden/reference_fixtures.npz
# by tests/golden/make_reference_fixtures.py)
# ---------------------------------------------------------------------------
REFERENCE_FIXTURES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                                  "reference_fixtures.npz")


def reference_fixtures(path: str = REFERENCE_FIXTURES) -> dict:
    """The reference's data arrays: leaf_mask (2D/vortex/data/leaf_mask_256_scaled.npz),
    density_{G,R}_2d (2D/shape/data/density_*_arial_scaled_shifted_0.8.npy) and
    density_{G,R}_3d (3D/model/density_*_centered_1.2x_128x128.npy)."""
    with np.load(path) as d:
        return {k: d[k] for k in d.files}


def extrude_glyph(glyph: np.ndarray, nz: int = 128) -> np.ndarray:
    """A 128x128 glyph density extruded along z the way the reference's 3D shape
    experiment does it (3D/optimize_shape_G_R.py:204-218): planes nz/2-16 ..
    nz/2+15 hold glyph * (1 - |k - nz/2| / 16)^0.1, the rest are zero (FP32)."""
    nx, ny = glyph.shape
    out = np.zeros((nx, ny, nz), dtype=np.float32)
    c = nz // 2
    for k in range(c - 16, c + 16):
        out[:, :, k] = glyph * (1 - abs(k - c) / 16) ** 0.1
    return out


def shape3d_glyph_inputs(fixtures: dict, seed_u=21, u_std=0.01):
    """The 3D shape experiment's own densities at 128^3: rho0 = the extruded G
    glyph, rho* = the extruded R glyph; u0 cell-centred N(0, u_std^2) split to faces."""
    rho0 = extrude_glyph(fixtures["density_G_3d"])
    rho_t = extrude_glyph(fixtures["density_R_3d"])
    rng = np.random.default_rng(seed_u)
    u0 = split_central_vector(rng.normal(0.0, u_std, size=(3,) + rho0.shape))
    return u0, rho0, rho_t


def shape2d_glyph_inputs(fixtures: dict, seed_u=12, u_std=0.01):
    """The 2D shape experiment's own densities at 256^2 (G glyph -> R glyph);
    u0 cell-centred N(0, u_std^2) split to faces."""
    rng = np.random.default_rng(seed_u)
    u0 = split_central_vector(rng.normal(0.0, u_std, size=(2, 256, 256)))
    return u0, fixtures["density_G_2d"].astype(np.float64), fixtures["density_R_2d"].astype(np.float64)


def shape2d_config(res=256, steps=200, reinit_every=12, rk=2, dt=0.01, dtype=torch.float32, store_dtype=None,
                   backward_u=True, rel_tol=1e-6, abs_tol=0.0, max_iters=400, check_every=0):
    """2D smoke shape transition, 256^2, 200 steps, reinit every 12, RK2, MGPCG 5 levels."""
    solver = SolverConfig(base_level=4, levels=int(math.log2(res)) - 4 + 1, bottom=20, bottom_mode=1,
                          max_iters=max_iters, abs_tol=abs_tol, rel_tol=rel_tol,
                          eps=1e-12 if dtype == torch.float32 else 0.0, check_every=check_every)
    return FlowmapConfig(res=(res, res), dx=1.0 / res, dt=dt, total_steps=steps, reinit_every=reinit_every,
                         RK_number=rk, backward_u=backward_u, add_passive_scalar=True, dtype=dtype,
                         store_dtype=store_dtype, solver=solver)


def vortex2d_config(res=256, steps=100, reinit_every=10, rk=2, dtype=torch.float32, rel_tol=1e-6, abs_tol=0.0,
                    max_iters=400, check_every=0, boundary_mask=None):
    """2D vortex optimisation: res^2, dx = 1/res, dt = 0.5 dx, 100 steps, reinit
    every 10, RK2, solid-style MGPCG (base level 4: 5 levels at 256^2, 20 bottom
    sweeps as 10 x (R,B) + 10 x (B,R)), no passive scalar; an optional obstacle
    mask (solid > 0) selects the solid-aware solver and the mask kernels."""
    solver = SolverConfig(base_level=4, levels=max(2, int(math.log2(res)) - 4 + 1), bottom=20, bottom_mode=1,
                          max_iters=max_iters, abs_tol=abs_tol, rel_tol=rel_tol,
                          eps=1e-12 if dtype == torch.float32 else 0.0, check_every=check_every)
    return FlowmapConfig(res=(res, res), dx=1.0 / res, dt=0.5 / res, total_steps=steps, reinit_every=reinit_every,
                         RK_number=rk, backward_u=True, add_passive_scalar=False, dtype=dtype, solver=solver,
                         boundary_mask=boundary_mask)


def leaf_mask(res=256, center=(0.5, 0.35), length=0.22, width=0.07, angle=0.6):
    """A synthetic leaf-shaped obstacle (solid = 1) standing in for the
    reference vortex experiment's leaf mask (2D/vortex/lfm_midpoint_simulator.py:
    406, a data file): the intersection of two discs (a lens) rotated by
    ``angle``, plus a one-cell-wide stem."""
    x = (np.arange(res) + 0.5) / res
    X, Y = np.meshgrid(x, x, indexing="ij")
    c, s_ = math.cos(angle), math.sin(angle)
    u = (X - center[0]) * c + (Y - center[1]) * s_
    v = -(X - center[0]) * s_ + (Y - center[1]) * c
    R = (length ** 2 + width ** 2) / (2 * width)
    lens = ((u ** 2 + (v - (R - width)) ** 2) < R ** 2) & ((u ** 2 + (v + (R - width)) ** 2) < R ** 2)
    stem = (np.abs(v) < 0.5 / res) & (u < -length) & (u > -length - 0.08)
    return (lens | stem).astype(np.float32)


def vortex2d_theta(seed=0, nv=4):
    """theta = [w_0..w_{K-1}, cx_0..cx_{K-1}, cy_0..cy_{K-1}]: strengths U[-1,1],
    centres U[0.25,0.75]^2."""
    rng = np.random.default_rng(seed)
    w = rng.uniform(-1.0, 1.0, nv)
    c = rng.uniform(0.25, 0.75, (nv, 2))
    return np.concatenate([w, c[:, 0], c[:, 1]])


def shape2d_inputs(res=256, seed_rect=10, seed_disc=11, seed_u=12, u_std=0.01):
    """rho0: union of 3 rectangles (sides U[0.1,0.3]); rho*: union of 3 discs
    (radii U[0.05,0.15]); u0 cell-centred N(0, u_std^2) split to faces."""
    dx = 1.0 / res
    x = (np.arange(res) + 0.5) * dx
    X, Y = np.meshgrid(x, x, indexing="ij")
    rng = np.random.default_rng(seed_rect)
    rho0 = np.zeros((res, res))
    for _ in range(3):
        sx, sy = rng.uniform(0.1, 0.3, size=2)
        x0, y0 = rng.uniform(0.1, 0.9 - sx), rng.uniform(0.1, 0.9 - sy)
        rho0 = np.maximum(rho0, ((X >= x0) & (X <= x0 + sx) & (Y >= y0) & (Y <= y0 + sy)).astype(np.float64))
    rng = np.random.default_rng(seed_disc)
    rho_t = np.zeros((res, res))
    for _ in range(3):
        r = rng.uniform(0.05, 0.15)
        c = rng.uniform(0.2, 0.8, size=2)
        rho_t = np.maximum(rho_t, smooth_ball((res, res), c, r, dx))
    rng = np.random.default_rng(seed_u)
    u0 = split_central_vector(rng.normal(0.0, u_std, size=(2, res, res)))
    return u0, rho0, rho_t


# ---------------------------------------------------------------------------
# Mixed-precision Poisson benchmark (256^3 cell-centred, Neumann walls)
# ---------------------------------------------------------------------------
def spectrum_velocity(res, seed=30, dtype=np.float32):
    """Random cell-centred velocity (dim, *res) with an isotropic E(k) ~ k^(-5/3)
    spectrum: per-mode amplitude |k|^(-11/6), uniform random phases, |k| >= 1,
    the mean and the Nyquist planes zeroed; built by inverse FFT, unit RMS."""
    rng = np.random.default_rng(seed)
    res = tuple(res)
    dim = len(res)
    ks = [np.fft.fftfreq(n, d=1.0 / n) for n in res[:-1]] + [np.fft.rfftfreq(res[-1], d=1.0 / res[-1])]
    K = np.meshgrid(*ks, indexing="ij")
    kmag = np.sqrt(sum(k.astype(np.float64) ** 2 for k in K))
    amp = np.zeros_like(kmag)
    amp[kmag >= 1] = kmag[kmag >= 1] ** (-11.0 / 6.0)
    for k, n in zip(K, res):
        amp[np.abs(k) == n // 2] = 0.0  # Nyquist planes
    out = np.empty((dim,) + res, dtype=np.float64)
    for c in range(dim):
        phase = rng.uniform(0.0, 2.0 * np.pi, size=amp.shape)
        out[c] = np.fft.irfftn(amp * np.exp(1j * phase), s=res, axes=tuple(range(dim)))
    out /= np.sqrt(np.mean(out ** 2))
    return out.astype(dtype)


def divergence_rhs(u_faces, dtype=np.float32):
    """Cell divergence of a MAC velocity with zero normal velocity on the walls
    (apply_bc + divergence, 3D/mgpcg.py:368-399): sum over axes of u[i+1] - u[i]."""
    dim = len(u_faces)
    div = None
    for c, f in enumerate(u_faces):
        f = np.array(f, dtype=np.float64, copy=True)
        idx0 = [slice(None)] * dim
        idx1 = [slice(None)] * dim
        idx0[c] = 0
        idx1[c] = -1
        f[tuple(idx0)] = 0.0
        f[tuple(idx1)] = 0.0
        d = np.diff(f, axis=c)
        div = d if div is None else div + d
    return div.astype(dtype)


def poisson_spectrum_rhs(res=256, seed=30):
    """RHS of the mixed-precision Poisson benchmark: the divergence of the
    seeded k^(-5/3) velocity, cell-centred -> faces -> divergence (FP32)."""
    vc = spectrum_velocity((res,) * 3 if np.isscalar(res) else res, seed=seed)
    return divergence_rhs(split_central_vector(vc))
