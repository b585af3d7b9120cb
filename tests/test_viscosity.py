"""The 2D viscous term (calculate_viscous_force / calculate_viscous_force_adj,
2D/vortex/flowmap.py:4-35) and the simulator's viscous path.

* fm_viscous_force_2d equals the oracle's restatement bit for bit in FP32 and
  FP64 (the kernel rounds each operation in the reference's order, no FMA
  contraction, IEEE division); the adjoint sum adj . vis / nu to 1e-12 (FP64
  reduction order differs); nu = 0 adds nothing to the sum.
* the simulator with viscosity (FP64) against the oracle's restatement: loss to
  1e-9, dL/du0 to 1e-7 relative L2, adj_viscous to 1e-8 relative.
"""
import ctypes as C
import importlib

import numpy as np
import pytest
import torch

from oracle import MGParams
from sim_oracle import OracleSim, viscous_force


def test_oracle_viscous_force_known_answers():
    """A linear field has zero Laplacian inside; the index clamp makes the
    boundary rows one-sided (the reference's sample())."""
    n0, n1, dx = 9, 8, 0.125
    x = np.add.outer(np.arange(n0) * 0.3, np.arange(n1) * -0.2)
    v = viscous_force([x], 0.01, dx)[0]
    assert np.abs(v[1:-1, 1:-1]).max() < 1e-12
    # row 0: s(i-1) = s(0): 0.01 * (x[1,j] - x[0,j]) / dx^2 = 0.01 * 0.3 * 64
    assert abs(v[0, 3] - 0.01 * 0.3 * 64) < 1e-12


def test_viscous_force_arguments_rejected_without_device(fm):
    lib = fm._lib.lib()
    g2 = fm._lib.Grid(2, (C.c_int * 3)(8, 8, 1))
    g3 = fm._lib.Grid(3, (C.c_int * 3)(8, 8, 8))
    P = C.c_void_p(1)
    assert lib.fm_viscous_force_2d(C.byref(g3), 0, 0.1, 0.1, P, P, P, P, None, None, None, None, None) == 1
    assert lib.fm_viscous_force_2d(C.byref(g2), 0, 0.1, 0.0, P, P, P, P, None, None, None, None, None) == 2
    assert lib.fm_viscous_force_2d(C.byref(g2), 0, 0.1, 0.1, P, P, P, P, P, None, P, P, None) == 2  # one adj
    assert lib.fm_viscous_force_2d(C.byref(g2), 0, 0.1, 0.1, P, P, P, P, P, P, None, P, None) == 2  # no part


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("res", [(32, 32), (37, 21)])
def test_viscous_force_bitwise_and_adjoint_sum(fm, cuda, dtype, res):
    K = importlib.import_module("differentiable-flowmap_b200.kernels")
    npt = np.float32 if dtype == torch.float32 else np.float64
    g = K.GridSpec(res)
    rng = np.random.default_rng(3)
    u = [rng.normal(size=g.face_shape(c)).astype(npt) for c in range(2)]
    a = [rng.normal(size=g.face_shape(c)).astype(npt) for c in range(2)]
    nu, dx = 2e-3, 1.0 / res[0]
    want = viscous_force(u, nu, dx)
    du = [torch.tensor(x, device="cuda") for x in u]
    da = [torch.tensor(x, device="cuda") for x in a]
    vis = [torch.empty_like(x) for x in du]
    part = torch.empty(592, dtype=torch.float64, device="cuda")
    dot = torch.full((1,), 0.5, dtype=torch.float64, device="cuda")
    K.viscous_force_2d(g, nu, dx, du, vis, adj=da, part=part, dot=dot)
    torch.cuda.synchronize()
    for c in range(2):
        np.testing.assert_array_equal(vis[c].cpu().numpy(), want[c])
    ref = 0.5 + sum(float(np.sum((a[c] * want[c] / npt(nu)).astype(np.float64))) for c in range(2))
    assert abs(float(dot) - ref) <= 1e-12 * max(1.0, abs(ref))
    K.viscous_force_2d(g, 0.0, dx, du, vis, adj=da, part=part, dot=dot)  # nu = 0: vis = 0, no sum
    torch.cuda.synchronize()
    assert abs(float(dot) - ref) <= 1e-12 * max(1.0, abs(ref))
    assert all(float(v.abs().max()) == 0.0 for v in vis)


CASES = {
    # name: (steps, R, rk, backward_u)
    "rk2": (8, 3, 2, True),
    "rk4_ckpt": (7, 4, 4, False),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_simulator_with_viscosity_matches_oracle(fm, cuda, name):
    steps, R, rk, bu = CASES[name]
    res, dt, nu = (32, 32), 0.01, 2e-3
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    Cf = importlib.import_module("differentiable-flowmap_b200.configs")
    rng = np.random.default_rng(5)
    u0 = Cf.split_central_vector(rng.normal(0.0, 0.2, size=(2,) + res))
    rho0 = Cf.smooth_ball(res, (0.5, 0.5), 0.25, 1 / 32)
    rho_t = Cf.smooth_ball(res, (0.55, 0.45), 0.2, 1 / 32)
    mg = MGParams(3, 2, 50, 0, 40, 0.0, 1e-22, 0.0)
    o = OracleSim(res, 1 / 32, dt, R, steps, rk=rk, backward_u=bu, prec="f64", mg=mg, viscosity=nu)
    lo, go = o.gradient(u0, rho0, rho_t)
    o0 = OracleSim(res, 1 / 32, dt, R, steps, rk=rk, backward_u=bu, prec="f64", mg=mg)
    l0, _ = o0.gradient(u0, rho0, rho_t)
    assert abs(l0 - lo) > 1e-6 * abs(lo)  # the term matters on this run
    solver = S.SolverConfig(levels=3, bottom=50, max_iters=40, abs_tol=0.0, rel_tol=1e-22, eps=0.0)
    cfg = S.FlowmapConfig(res=res, dx=1 / 32, dt=dt, total_steps=steps, reinit_every=R, RK_number=rk,
                          backward_u=bu, dtype=torch.float64, solver=solver, viscosity=nu)
    sim = S.LFM_Diff_Simulator(config=cfg)
    lc, gc = sim.gradient(u0, rho0, rho_t)
    gc = [x.cpu().numpy() for x in gc]
    num = np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(gc, go)))
    den = np.sqrt(sum(np.sum(y ** 2) for y in go))
    assert abs(lc - lo) / abs(lo) < 1e-9
    assert num / den < 1e-7
    av = float(sim.adj_viscous.to_numpy()[0])
    assert o.adj_viscous != 0.0
    assert abs(av - o.adj_viscous) <= 1e-8 * abs(o.adj_viscous)
