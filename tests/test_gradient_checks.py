"""Gradient checks on the GPU: the adjoint gradient against central finite
differences of the forward loss (FP64), and the autograd wrapper.

The reference's adjoint (3D/lfm_midpoint_diff_simulator.py) is a discretised
continuous adjoint, not the transpose of the discrete forward map, so it agrees
with finite differences only approximately; the CPU oracle (the reference
algorithm restated) shows the same agreement on these inputs: for smooth
velocity fields about 10-17 % relative error with cosine similarity > 0.99,
and far worse on grid-scale noise.  The thresholds below are set to that
behaviour; exact parity with the reference adjoint is tested in
test_sim_parity.py.
"""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _smooth(rng, shape, amp, kmax=3):
    """Sum of low-frequency modes on a grid of `shape` (2D or 3D), max |.| = amp."""
    axes = [(np.arange(n) + 0.5) / n for n in shape]
    X = np.meshgrid(*axes, indexing="ij")
    f = np.zeros(shape)
    for ks in np.ndindex(*([kmax] * len(shape))):
        term = rng.normal() / sum((k + 1) ** 2 for k in ks)
        for x, k in zip(X, ks):
            term = term * np.sin(np.pi * (k + 1) * x + rng.uniform(0, 6))
        f += term
    return amp * f / np.abs(f).max()


def _setup(res=(32, 32), steps=12, R=4, rk=2, dt=0.01):
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    dim = len(res)
    solver = S.SolverConfig(levels=max(2, int(np.log2(min(res))) - 2), bottom=50, max_iters=60, abs_tol=0.0,
                            rel_tol=1e-24, eps=0.0, check_every=0)
    cfg = S.FlowmapConfig(res=res, dx=1.0 / res[0], dt=dt, total_steps=steps, reinit_every=R, RK_number=rk,
                          dtype=torch.float64, solver=solver)
    sim = S.LFM_Diff_Simulator(config=cfg)
    rng = np.random.default_rng(3)
    u0 = C.split_central_vector(np.stack([_smooth(rng, res, 0.5) for _ in range(dim)]))
    rho0 = C.smooth_ball(res, (0.5,) * dim, 0.25, 1.0 / res[0])
    rho_t = C.smooth_ball(res, (0.55, 0.45, 0.5)[:dim], 0.2, 1.0 / res[0])
    return sim, [torch.tensor(x, device="cuda") for x in u0], rho0, rho_t


def _loss(sim, u0, rho0, rho_t):
    sim.init(theta=u0, init_passive_np=rho0)
    while not sim.forward_step_midpoint()[1]:
        pass
    diff = sim.passive - torch.as_tensor(rho_t, device="cuda")
    return float((diff ** 2).sum())


def _agreement(ad, fd):
    ad, fd = np.asarray(ad), np.asarray(fd)
    cos = float(ad @ fd / (np.linalg.norm(ad) * np.linalg.norm(fd)))
    rel = float(np.linalg.norm(ad - fd) / np.linalg.norm(fd))
    return cos, rel


@pytest.mark.parametrize("res,rk", [((32, 32), 2), ((16, 16, 16), 4)])
def test_directional_derivatives_vs_central_fd(cuda, res, rk):
    sim, u0, rho0, rho_t = _setup(res=res, rk=rk)
    loss, grad = sim.gradient(u0, rho0, rho_t)
    rng = np.random.default_rng(7)
    ads, fds = [], []
    for _ in range(6):
        d = [torch.tensor(_smooth(rng, tuple(x.shape), 1.0), device="cuda") for x in u0]
        h = 1e-4
        lp = _loss(sim, [x + h * y for x, y in zip(u0, d)], rho0, rho_t)
        lm = _loss(sim, [x - h * y for x, y in zip(u0, d)], rho0, rho_t)
        fds.append((lp - lm) / (2 * h))
        ads.append(float(sum((g * y).sum() for g, y in zip(grad, d))))
    cos, rel = _agreement(ads, fds)
    assert cos > 0.95 and rel < 0.3, (cos, rel, ads, fds)


def test_fd_on_32_random_entries(cuda):
    sim, u0, rho0, rho_t = _setup()
    loss, grad = sim.gradient(u0, rho0, rho_t)
    rng = np.random.default_rng(13)
    h = 1e-3 * max(float(x.abs().max()) for x in u0)
    fds, ads = [], []
    for _ in range(32):
        c = int(rng.integers(len(u0)))
        idx = tuple(int(rng.integers(1, n - 1)) for n in u0[c].shape)
        up = [x.clone() for x in u0]
        um = [x.clone() for x in u0]
        up[c][idx] += h
        um[c][idx] -= h
        fds.append((_loss(sim, up, rho0, rho_t) - _loss(sim, um, rho0, rho_t)) / (2 * h))
        ads.append(float(grad[c][idx]))
    cos, rel = _agreement(ads, fds)
    assert cos > 0.97 and rel < 0.3, (cos, rel)


def test_autograd_function(cuda):
    A = importlib.import_module("differentiable-flowmap_b200.autograd")
    sim, u0, rho0, rho_t = _setup(steps=8)
    u = [x.clone().requires_grad_(True) for x in u0]
    L = A.flowmap_loss(sim, u, rho0, rho_t)
    (3.0 * L).backward()
    loss, grad = sim.gradient(u0, rho0, rho_t)
    assert abs(float(L.detach()) - loss) <= 1e-12 * abs(loss)
    for a, b in zip(u, grad):
        assert torch.allclose(a.grad, 3.0 * b, rtol=1e-12, atol=0)


def test_autograd_loss_without_gradients_runs_no_adjoint(cuda):
    """Under torch.no_grad the loss costs one forward pass: the same kernel
    launches as run_forward alone, no adjoint kernel, and the same loss; a
    backward after an intervening forward pass rebuilds its own trajectory."""
    A = importlib.import_module("differentiable-flowmap_b200.autograd")
    lib = importlib.import_module("differentiable-flowmap_b200._lib")
    sim, u0, rho0, rho_t = _setup(steps=8)
    loss, grad = sim.gradient(u0, rho0, rho_t)
    torch.cuda.synchronize()
    lib.launch_count(reset=True)
    sim.run_forward(u0, rho0)
    torch.cuda.synchronize()
    n_forward = lib.launch_count(reset=True)
    sim.gradient(u0, rho0, rho_t)
    torch.cuda.synchronize()
    n_gradient = lib.launch_count(reset=True)
    with torch.no_grad():
        L = A.flowmap_loss(sim, u0, rho0, rho_t)
    torch.cuda.synchronize()
    n_nograd = lib.launch_count(reset=True)
    assert n_nograd == n_forward < n_gradient, (n_nograd, n_forward, n_gradient)
    assert abs(float(L.detach()) - loss) <= 1e-12 * abs(loss)
    # a forward pass of other inputs between forward and backward
    u = [x.clone().requires_grad_(True) for x in u0]
    L = A.flowmap_loss(sim, u, rho0, rho_t)
    sim.run_forward([0.5 * x for x in u0], rho0)
    L.backward()
    for a, b in zip(u, grad):
        assert torch.equal(a.grad, b)
