"""BFECC_clamp and use_short_BFECC variants of the forward and adjoint steps.

clamp_u (3D/flowmap.py:324-334) limits the BFECC result to the extrema of the
first pass's axis neighbours; use_short_BFECC (3D/lfm_midpoint_simulator.py:725-745,
3D/lfm_midpoint_diff_simulator.py:440-485) replaces the per-step semi-Lagrangian
advection by BFECC through one-step maps.  The CUDA path (FP64) is compared with
the oracle's restatement on the same seeded inputs: loss to 1e-9 relative,
gradient dL/du0 to 1e-7 relative L2 (the tolerances of the default path's
parity test).  fm_clamp_extrema itself is compared element by element: it only
selects among its inputs, so it is bit-exact in both precisions.
"""
import importlib

import numpy as np
import pytest
import torch

from oracle import MGParams
from sim_oracle import OracleSim, clamp_u

VARIANTS = {
    # name: (res, steps, R, rk, backward_u, dt, clamp, short)
    "3d_clamp_rk4": ((16, 16, 16), 6, 4, 4, True, 0.02, True, False),
    "3d_short_rk2_ckpt": ((16, 16, 16), 6, 3, 2, False, 0.02, False, True),
    "3d_short_clamp": ((16, 16, 16), 5, 4, 4, True, 0.02, True, True),
    "2d_short_rk4": ((32, 32), 8, 3, 4, True, 0.01, False, True),
    "2d_short_clamp_ckpt": ((32, 32), 7, 4, 2, False, 0.01, True, True),
}


def _inputs(res, seed=1):
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    dx = 1.0 / res[0]
    rng = np.random.default_rng(seed)
    dim = len(res)
    u0 = C.split_central_vector(rng.normal(0.0, 0.3, size=(dim,) + tuple(res)))
    rho0 = C.smooth_ball(res, (0.5,) * dim, 0.25, dx)
    rho_t = C.smooth_ball(res, tuple(0.45 + 0.1 * rng.uniform(size=dim)), 0.2, dx)
    return u0, rho0, rho_t


def _levels(res):
    return max(2, int(np.log2(min(res))) - 3 + 1)


def _rel_l2(a, b):
    num = np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(a, b)))
    den = np.sqrt(sum(np.sum(y ** 2) for y in b))
    return num / den


def _run_cuda(name, dtype):
    res, steps, R, rk, bu, dt, clamp, short = VARIANTS[name]
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    tight = dtype == torch.float64
    solver = S.SolverConfig(levels=_levels(res), bottom=50, max_iters=40 if tight else 200,
                            abs_tol=0.0, rel_tol=1e-22 if tight else 1e-12, eps=0.0 if tight else 1e-12)
    cfg = S.FlowmapConfig(res=res, dx=1.0 / res[0], dt=dt, total_steps=steps, reinit_every=R, RK_number=rk,
                          backward_u=bu, dtype=dtype, solver=solver, BFECC_clamp=clamp, use_short_BFECC=short)
    sim = S.LFM_Diff_Simulator(config=cfg)
    loss, grad = sim.gradient(*_inputs(res))
    return loss, [g.double().cpu().numpy() for g in grad]


def _run_oracle(name):
    res, steps, R, rk, bu, dt, clamp, short = VARIANTS[name]
    mg = MGParams(_levels(res), 2, 50, 0, 40, 0.0, 1e-22, 0.0)
    o = OracleSim(res, 1.0 / res[0], dt, R, steps, rk=rk, backward_u=bu, prec="f64", mg=mg,
                  bfecc_clamp=clamp, short_bfecc=short)
    return o.gradient(*_inputs(res))


@pytest.fixture(scope="module")
def oracle_results():
    return {}


def test_oracle_clamp_u_is_neighbour_clamp():
    """clamp_u on a hand-made field: centre excluded, boundary neighbours repeat."""
    u1 = np.array([[0.0, 5.0, 0.0], [1.0, 9.0, 2.0], [0.0, 3.0, 0.0]])
    u = np.full_like(u1, 100.0)
    out = clamp_u(u, u1)
    # (1,1): neighbours 5,1,2,3 -> max 5 (the centre's 9 is not a bound)
    assert out[1, 1] == 5.0
    # (0,0): neighbours u1[0,0] (clamped i-1), u1[1,0], u1[0,0] (clamped j-1), u1[0,1] -> max 5
    assert out[0, 0] == 5.0
    assert np.all(clamp_u(-u, u1) <= 3.0)


def test_clamp_removes_bfecc_overshoot():
    """Short BFECC of a 0/1 indicator overshoots [0, 1]; with BFECC_clamp the
    passive scalar stays inside it (up to the first pass's rounding)."""
    res = (16, 16)
    u0, _, _ = _inputs(res)
    x = (np.arange(16) + 0.5) / 16
    X, Y = np.meshgrid(x, x, indexing="ij")
    rho = (((X - 0.5) ** 2 + (Y - 0.5) ** 2) < 0.09).astype(np.float64)
    ext = {}
    for clamp in (False, True):
        o = OracleSim(res, 1.0 / 16, 0.05, 4, 3, rk=2, prec="f64", mg=MGParams(2, 2, 20, 0, 10, 0.0, 1e-20, 0.0),
                      short_bfecc=True, bfecc_clamp=clamp)
        o.init(u0, rho)
        for _ in range(3):
            o.step_midpoint()
        ext[clamp] = (o.passive.min(), o.passive.max())
    assert ext[False][0] < -0.01 and ext[False][1] > 1.01
    assert ext[True][0] >= -1e-12 and ext[True][1] <= 1 + 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(VARIANTS))
def test_fp64_variant_gradient_matches_oracle(fm, cuda, name, oracle_results):
    lo, go = oracle_results.setdefault(name, _run_oracle(name))
    lc, gc = _run_cuda(name, torch.float64)
    assert abs(lc - lo) / abs(lo) < 1e-9
    assert np.linalg.norm(np.concatenate([g.ravel() for g in go])) > 0
    assert _rel_l2(gc, go) < 1e-7


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["3d_short_clamp", "2d_short_rk4"])
def test_fp32_variant_close_to_fp64_oracle(fm, cuda, name, oracle_results):
    lo, go = oracle_results.setdefault(name, _run_oracle(name))
    lc, gc = _run_cuda(name, torch.float32)
    assert abs(lc - lo) / abs(lo) < 1e-4
    assert _rel_l2(gc, go) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("res", [(9, 12, 7), (33, 20)])
def test_clamp_extrema_bitwise(fm, cuda, dtype, res):
    K = importlib.import_module("differentiable-flowmap_b200.kernels")
    g = K.GridSpec(res)
    rng = np.random.default_rng(len(res))
    for face in [-1] + list(range(len(res))):
        shape = tuple(res) if face < 0 else g.face_shape(face)
        src = rng.normal(size=shape) * 1.5
        ref = rng.normal(size=shape)
        want = clamp_u(src.astype(np.float32) if dtype == torch.float32 else src,
                       ref.astype(np.float32) if dtype == torch.float32 else ref)
        s = torch.tensor(src, dtype=dtype, device="cuda")
        r = torch.tensor(ref, dtype=dtype, device="cuda")
        d = torch.empty_like(s)
        K.clamp_extrema(g, s, r, d)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d.cpu().numpy(), want)
