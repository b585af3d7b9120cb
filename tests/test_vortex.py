"""2D vortex problem (control map theta -> u0, final-vorticity loss, dL/dtheta).

CPU: the oracle's transposes pass dot-product tests, and its analytic-grade
theta gradient agrees with the reference's forward-difference method
(2D/vortex/optimize_vortex.py:193-220).
GPU: every vortex kernel against the oracle (FP64 to round-off, FP32 to 1e-5),
the full gradient against the oracle simulator in FP64, and dL/dtheta against
central finite differences of the loss.
"""
import importlib

import numpy as np
import pytest
import torch

import vortex_oracle as V
from oracle import MGParams
from sim_oracle import OracleSim


def _C():
    return importlib.import_module("differentiable-flowmap_b200.configs")


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


# ------------------------------------------------------------------ CPU
def test_oracle_transposes_dot_product():
    rng = np.random.default_rng(0)
    n, dx = (24, 20), 1 / 24
    ux, uy = rng.standard_normal((n[0] + 1, n[1])), rng.standard_normal((n[0], n[1] + 1))
    g = rng.standard_normal(n)
    lx, ly = V.vorticity_adjoint(g, dx)
    a, b = np.sum(V.vorticity(ux, uy, dx) * g), np.sum(lx * ux) + np.sum(ly * uy)
    assert abs(a - b) <= 1e-12 * abs(a)
    vc = rng.standard_normal((2,) + n)
    fx, fy = V.split_central_vector(vc)
    gx, gy = V.split_adjoint(ux, uy)
    a, b = np.sum(fx * ux) + np.sum(fy * uy), np.sum(gx * vc[0]) + np.sum(gy * vc[1])
    assert abs(a - b) <= 1e-12 * abs(a)


def test_oracle_theta_grad_matches_reference_fd():
    rng = np.random.default_rng(1)
    n, dx = (32, 32), 1 / 32
    theta = _C().vortex2d_theta(3)
    lam = [rng.standard_normal((n[0] + 1, n[1])), rng.standard_normal((n[0], n[1] + 1))]
    a, b = V.theta_grad(theta, lam, n, dx), V.theta_grad_fd(theta, lam, n, dx)
    assert _rel(b, a) < 2e-3  # forward differences with epsilon 1e-5


# ------------------------------------------------------------------ GPU
PRECS = [("f64", torch.float64, np.float64, 1e-12), ("f32", torch.float32, np.float32, 1e-5)]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(64, 64), (48, 40)])
@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p[0])
def test_vortex_velocity_and_vorticity(fm, cuda, shape, prec):
    _, tdt, ndt, tol = prec
    dx = 1.0 / shape[0]
    g = fm.GridSpec(shape)
    theta = _C().vortex2d_theta(5)
    u = [torch.empty(g.face_shape(c), dtype=tdt, device=cuda) for c in range(2)]
    fm.kernels.vortex_velocity_2d(g, dx, theta, u[0], u[1])
    ref = V.vortex_faces(theta, shape, dx, ndt)
    for c in range(2):
        assert _rel(u[c].cpu().numpy(), ref[c]) < tol
    rng = np.random.default_rng(2)
    ur = [rng.standard_normal(g.face_shape(c)).astype(ndt) for c in range(2)]
    om = torch.empty(shape, dtype=tdt, device=cuda)
    fm.kernels.vorticity_2d(g, dx, torch.tensor(ur[0], device=cuda), torch.tensor(ur[1], device=cuda), om)
    assert _rel(om.cpu().numpy(), V.vorticity(ur[0], ur[1], dx)) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(64, 64), (48, 40)])
@pytest.mark.parametrize("prec", PRECS, ids=lambda p: p[0])
def test_vorticity_loss_seed_and_theta_grad(fm, cuda, shape, prec):
    _, tdt, ndt, tol = prec
    dx = 1.0 / shape[0]
    g = fm.GridSpec(shape)
    rng = np.random.default_rng(4)
    ur = [rng.standard_normal(g.face_shape(c)).astype(ndt) for c in range(2)]
    omt = rng.standard_normal(shape).astype(ndt)
    du = [torch.tensor(x, device=cuda) for x in ur]
    lam = [torch.empty_like(x) for x in du]
    work = torch.empty(shape, dtype=tdt, device=cuda)
    part = torch.empty(592, dtype=torch.float64, device=cuda)
    loss = torch.empty(1, dtype=torch.float64, device=cuda)
    fm.kernels.vorticity_loss_2d(g, dx, du[0], du[1], torch.tensor(omt, device=cuda), lam[0], lam[1], work, part, loss)
    om = V.vorticity(ur[0], ur[1], dx)
    d = om.astype(np.float64) - omt.astype(np.float64)
    assert abs(float(loss) - float(np.sum(d * d))) <= 10 * tol * float(np.sum(d * d))
    ref = V.vorticity_adjoint((2 * d).astype(ndt), dx)
    for c in range(2):
        assert _rel(lam[c].cpu().numpy(), ref[c]) < tol
    theta = _C().vortex2d_theta(6)
    gt = fm.kernels.vortex_velocity_grad_2d(g, dx, theta, lam[0], lam[1]).cpu().numpy()
    assert _rel(gt, V.theta_grad(theta, [x.cpu().numpy() for x in lam], shape, dx)) < 1e-6


def _vortex_setup(fm, n, steps, R, dtype, target_seed=1):
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    vx = importlib.import_module("differentiable-flowmap_b200.vortex")
    cfg = _C().vortex2d_config(res=n, steps=steps, reinit_every=R, dtype=dtype, rel_tol=1e-26 if dtype ==
                               torch.float64 else 1e-6, max_iters=200)
    sim = S.LFM_Diff_Simulator(config=cfg)
    prob = vx.VortexProblem(sim)
    omt = prob.final_vorticity(_C().vortex2d_theta(target_seed))
    return cfg, sim, prob, omt


@pytest.mark.gpu
@pytest.mark.parametrize("n,steps,R", [(32, 8, 4), (256, 20, 10), (192, 10, 10)],
                         ids=["32", "256-config0-size", "192-batch-size"])
def test_vortex_gradient_matches_oracle_fp64(fm, cuda, n, steps, R):
    """The vortex gradient (theta -> u0 -> steps -> vorticity loss -> adjoint ->
    dL/dtheta) against the oracle: at a small grid, at the 2D vortex benchmark's
    256^2 over two reinit intervals, and at one of the batched instances' 192^2
    grids, whose dx = 1/192 is not a power of two."""
    cfg, sim, prob, omt = _vortex_setup(fm, n, steps, R, torch.float64)
    theta = _C().vortex2d_theta(0)
    loss, dth = prob.gradient(theta, omt)
    lam = [x.cpu().numpy() for x in sim.adj_u]
    mg = MGParams(cfg.solver.levels, 2, 20, 1, 200, 0.0, 1e-26, 0.0)
    o = OracleSim((n, n), 1.0 / n, 0.5 / n, R, steps, rk=2, backward_u=True, passive=False, prec="f64", mg=mg)
    l_ref, g_ref = o.gradient_vorticity(V.vortex_faces(theta, (n, n), 1.0 / n), omt.cpu().numpy())
    assert abs(loss - l_ref) <= 1e-9 * abs(l_ref)
    num = sum(np.sum((a - b) ** 2) for a, b in zip(lam, g_ref))
    den = sum(np.sum(b ** 2) for b in g_ref)
    assert (num / den) ** 0.5 < 1e-7
    assert _rel(dth, V.theta_grad(theta, g_ref, (n, n), 1.0 / n)) < 1e-6


@pytest.mark.gpu
def test_vortex_theta_gradient_vs_central_fd(fm, cuda):
    """The adjoint is the reference's discretised continuous adjoint, so it
    matches finite differences of the discrete loss only approximately."""
    n, steps, R = 64, 20, 10
    cfg, sim, prob, omt = _vortex_setup(fm, n, steps, R, torch.float64)
    theta = _C().vortex2d_theta(0)
    loss, dth = prob.gradient(theta, omt)

    def L(th):
        om = prob.final_vorticity(th)
        return float(((om - omt).double() ** 2).sum())

    fd = []
    for i in range(len(theta)):
        h = 1e-5
        tp, tm = np.array(theta), np.array(theta)
        tp[i] += h
        tm[i] -= h
        fd.append((L(tp) - L(tm)) / (2 * h))
    fd = np.array(fd)
    cos = float(dth @ fd / (np.linalg.norm(dth) * np.linalg.norm(fd)))
    rel = float(np.linalg.norm(dth - fd) / np.linalg.norm(fd))
    assert cos > 0.95 and rel < 0.3, (cos, rel, dth, fd)


@pytest.mark.gpu
def test_batched_instances_equal_unbatched_runs(fm, cuda):
    """Concurrent instances of uneven sizes (one stream and host thread each)
    reproduce separate unbatched runs bit for bit."""
    B = importlib.import_module("differentiable-flowmap_b200.batch")
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    vx = importlib.import_module("differentiable-flowmap_b200.vortex")
    sizes = (32, 48, 64, 32, 48)
    bat = B.BatchedVortex(sizes, steps=8, reinit_every=4)
    conc = bat.gradients(concurrent=True)
    seq = bat.gradients(concurrent=False)
    for (la, da), (lb, db) in zip(conc, seq):
        assert la == lb and np.array_equal(da, db)
    # a separately built single instance
    cfg = _C().vortex2d_config(res=48, steps=8, reinit_every=4)
    prob = vx.VortexProblem(S.LFM_Diff_Simulator(config=cfg))
    omt = prob.final_vorticity(_C().vortex2d_theta(200 + 1))
    loss, dth = prob.gradient(_C().vortex2d_theta(100 + 1), omt)
    assert loss == conc[1][0] and np.array_equal(dth, conc[1][1])
