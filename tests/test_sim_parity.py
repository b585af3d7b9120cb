"""End-to-end parity of the CUDA simulator (forward leapfrog steps with
reinitialisation + adjoint backtrack) against the oracle's restatement of the
reference control flow, on the same seeded inputs.

FP64 CUDA vs FP64 oracle: loss to 1e-9 relative, gradient dL/du0 to 1e-7
(relative L2) -- only summation order and the solvers' iteration paths differ,
both solved to machine precision.  FP32 CUDA vs FP64 oracle: gradient relative
L2 error <= 1e-3 (the FP32 drop-in's accuracy on these short runs).
"""
import importlib

import numpy as np
import pytest
import torch

from oracle import MGParams
from sim_oracle import OracleSim

pytestmark = pytest.mark.gpu

CASES = {
    # name: (res, steps, R, rk, backward_u, dt)
    "3d_rk4_partial_interval": ((16, 16, 16), 10, 4, 4, True, 0.02),
    "3d_rk2_ckpt": ((16, 16, 16), 8, 4, 2, False, 0.02),
    "2d_rk2": ((32, 32), 12, 5, 2, True, 0.01),
    "2d_rk4_ckpt": ((32, 32), 9, 3, 4, False, 0.01),
}


def _inputs(res, seed=0):
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    dx = 1.0 / res[0]
    rng = np.random.default_rng(seed)
    dim = len(res)
    uc = rng.normal(0.0, 0.3, size=(dim,) + tuple(res))
    u0 = C.split_central_vector(uc)
    c = (0.5,) * dim
    rho0 = C.smooth_ball(res, c, 0.25, dx)
    rho_t = C.smooth_ball(res, tuple(0.45 + 0.1 * rng.uniform(size=dim)), 0.2, dx)
    return u0, rho0, rho_t


def _levels(res):
    return max(2, int(np.log2(min(res))) - 3 + 1)


def _run_cuda(fm, name, dtype):
    res, steps, R, rk, bu, dt = CASES[name]
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    tight = dtype == torch.float64
    solver = S.SolverConfig(levels=_levels(res), bottom=50, max_iters=40 if tight else 200,
                            abs_tol=0.0, rel_tol=1e-22 if tight else 1e-12, eps=0.0 if tight else 1e-12)
    cfg = S.FlowmapConfig(res=res, dx=1.0 / res[0], dt=dt, total_steps=steps, reinit_every=R, RK_number=rk,
                          backward_u=bu, dtype=dtype, solver=solver)
    sim = S.LFM_Diff_Simulator(config=cfg)
    u0, rho0, rho_t = _inputs(res)
    loss, grad = sim.gradient(u0, rho0, rho_t)
    return loss, [g.double().cpu().numpy() for g in grad], sim


def _run_oracle(name):
    res, steps, R, rk, bu, dt = CASES[name]
    mg = MGParams(_levels(res), 2, 50, 0, 40, 0.0, 1e-22, 0.0)
    o = OracleSim(res, 1.0 / res[0], dt, R, steps, rk=rk, backward_u=bu, prec="f64", mg=mg)
    u0, rho0, rho_t = _inputs(res)
    loss, grad = o.gradient(u0, rho0, rho_t)
    return loss, grad, o


def _rel_l2(a, b):
    num = np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(a, b)))
    den = np.sqrt(sum(np.sum(y ** 2) for y in b))
    return num / den


@pytest.fixture(scope="module")
def oracle_results():
    return {}


@pytest.mark.parametrize("name", list(CASES))
def test_fp64_gradient_matches_oracle(fm, cuda, name, oracle_results):
    lo, go, _ = oracle_results.setdefault(name, _run_oracle(name))
    lc, gc, sim = _run_cuda(fm, name, torch.float64)
    assert abs(lc - lo) / abs(lo) < 1e-9
    assert np.linalg.norm(np.concatenate([g.ravel() for g in go])) > 0
    assert _rel_l2(gc, go) < 1e-7
    # final state also matches
    assert sim.step_num[None] == 0


@pytest.mark.parametrize("name", list(CASES))
def test_fp32_gradient_close_to_fp64_oracle(fm, cuda, name, oracle_results):
    lo, go, _ = oracle_results.setdefault(name, _run_oracle(name))
    lc, gc, _ = _run_cuda(fm, name, torch.float32)
    assert abs(lc - lo) / abs(lo) < 1e-4
    assert _rel_l2(gc, go) < 1e-3
