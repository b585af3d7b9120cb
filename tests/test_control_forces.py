"""Gaussian control forces (apply_gausion_force / calculate_adj_gausion_force)
and the simulator's control-force path.

* oracle known answers (CPU): a Gaussian centred on a face gives exactly s
  there, exp(-1) s one cell away, nothing at q = 5 (the cutoff is strict); the
  strength adjoint makes sum(adj . f) linear in s; the centre and penalty sums
  match central finite differences of sum(adj . f) and sum f_I^2.
* fm_gaussian_force vs the oracle (GPU): FP64 to 1e-12 and FP32 to 2e-6 of the
  field's scale (the per-face inclusion test rounds identically on both sides,
  only exp differs), on tile-ragged 2D/3D grids with 300 Gaussians (two
  chunks of the tile cull) and the edge cases r = 0, r < 0, r = NaN, a centre
  outside the domain, a support smaller than a cell, n = 0.
* fm_gaussian_force_grad vs the oracle: FP64 to 1e-10, FP32 to 1e-4 of each
  output's scale.
* simulator with control forces vs the oracle's restatement (FP64): loss to
  1e-9, dL/du0 and every step's parameter gradients to 1e-7 relative L2.
"""
import ctypes as C
import importlib

import numpy as np
import pytest
import torch

import force_oracle as FO
from oracle import MGParams
from sim_oracle import OracleSim


def _edge_gaussians(dim, dx, dtype):
    c = np.full((6, dim), 0.5)
    r = np.array([0.0, -2.0, np.nan, 1.0 / (3 * dx) ** 2, 1.0 / (2 * dx) ** 2, 1e6 / dx ** 2])
    c[3, 0] = -0.05          # centre outside the domain, support reaching in
    c[5] = 0.5 + 0.5 * dx    # support far below a cell: reaches no face
    s = np.tile(np.linspace(0.01, 0.03, dim), (6, 1))
    return c.astype(dtype), r.astype(dtype), s.astype(dtype)


def _params(res, n, seed, dtype, edges=True):
    dx = 1.0 / res[0]
    c, r, s = FO.random_gaussians(n, len(res), dx, seed, dtype)
    if edges:
        ce, re, se = _edge_gaussians(len(res), dx, dtype)
        c, r, s = np.concatenate([c, ce]), np.concatenate([r, re]), np.concatenate([s, se])
    return c, r, s


# ------------------------------------------------------------------ CPU: oracle
def test_oracle_single_gaussian_known_answers():
    res, dx = (16, 16), 1.0 / 16
    c = np.array([[8 * dx, 8.5 * dx]])      # exactly on x-face (8, 8)
    r = np.array([1.0 / dx ** 2])
    s = np.array([[0.7, 0.0]])
    fx, fy = FO.gaussian_force(res, dx, c, r, s)
    assert fx[8, 8] == 0.7
    assert abs(fx[9, 8] - 0.7 * np.exp(-1.0)) < 1e-15
    assert abs(fx[10, 8] - 0.7 * np.exp(-4.0)) < 1e-15
    assert fx[8, 10] > 0                      # q = 4
    assert fx[11, 8] == 0.0                   # q = 9
    assert np.all(fy == 0.0)
    # q = 5 exactly (offsets 2 and 1 cells) is outside the strict cutoff, up to rounding of d*d
    p = np.array([10 * dx, 9.5 * dx])
    d = np.sqrt(np.sum((p - c[0]) ** 2))
    assert (fx[10, 9] == 0.0) == (not ((d * d) * r[0] < 5))


def test_oracle_strength_adjoint_is_exact_linearisation():
    res, dx = (24, 20), 1.0 / 24
    c, r, s = FO.random_gaussians(30, 2, dx, 3)
    rng = np.random.default_rng(4)
    adj = [rng.normal(size=(25, 20)), rng.normal(size=(24, 21))]
    f = FO.gaussian_force(res, dx, c, r, s)
    _, adj_s, _, _ = FO.gaussian_force_grad(res, dx, c, r, s, adj)
    lhs = sum(np.sum(a * x) for a, x in zip(adj, f))
    assert abs(lhs - np.sum(adj_s * s)) < 1e-12 * max(1.0, abs(lhs))


def _near_cutoff(res, dx, c, r, eps=1e-3):
    for comp in range(len(res)):
        P = FO.face_positions(res, comp, dx, np.float64)
        d2 = sum((P[a] - c[a]) ** 2 for a in range(len(res)))
        if np.any(np.abs(d2 * r - 5.0) < eps * 5.0):
            return True
    return False


@pytest.mark.parametrize("res", [(20, 24), (10, 12, 8)])
def test_oracle_center_and_penalty_match_finite_differences(res):
    dx = 1.0 / res[0]
    dim = len(res)
    c, r, s = FO.random_gaussians(12, dim, dx, 7)
    rng = np.random.default_rng(8)
    adj = [rng.normal(size=tuple(res[a] + (a == k) for a in range(dim))) for k in range(dim)]
    adj_c, _, pen_c, pen_s = FO.gaussian_force_grad(res, dx, c, r, s, adj)

    def obj(I, cc, ss, which):
        f = FO.gaussian_force(res, dx, cc[I:I + 1], r[I:I + 1], ss[I:I + 1])
        if which == "adj":
            return sum(np.sum(adj[k] * f[k]) for k in range(dim))
        return sum(np.sum(f[k] ** 2) for k in range(dim))

    h = 1e-6
    checked = 0
    for I in range(len(r)):
        if _near_cutoff(res, dx, c[I], r[I], eps=1e-3):
            continue
        checked += 1
        for a in range(dim):
            cp, cm = c.copy(), c.copy()
            cp[I, a] += h
            cm[I, a] -= h
            fd = (obj(I, cp, s, "adj") - obj(I, cm, s, "adj")) / (2 * h)
            assert abs(fd - adj_c[I, a]) <= 1e-5 * max(1.0, abs(fd))
            fdp = (obj(I, cp, s, "pen") - obj(I, cm, s, "pen")) / (2 * h)
            assert abs(fdp - pen_c[I, a]) <= 1e-5 * max(1.0, abs(fdp))
            sp, sm = s.copy(), s.copy()
            sp[I, a] += h
            sm[I, a] -= h
            fds = (obj(I, c, sp, "pen") - obj(I, c, sm, "pen")) / (2 * h)
            assert abs(fds - pen_s[I, a]) <= 1e-6 * max(1.0, abs(fds))
    assert checked >= 6


def test_gaussian_force_arguments_rejected_without_device(fm):
    lib = fm._lib.lib()
    g2 = fm._lib.Grid(2, (C.c_int * 3)(8, 8, 1))
    g3 = fm._lib.Grid(3, (C.c_int * 3)(8, 8, 8))
    P = C.c_void_p(1)
    assert lib.fm_gaussian_force(C.byref(g2), 0, 0.1, -1, P, P, P, P, P, None, None) == 2       # n < 0
    assert lib.fm_gaussian_force(C.byref(g2), 0, 0.0, 1, P, P, P, P, P, None, None) == 2        # dx <= 0
    assert lib.fm_gaussian_force(C.byref(g2), 0, 0.1, 1, None, P, P, P, P, None, None) == 2     # no centres
    assert lib.fm_gaussian_force(C.byref(g3), 0, 0.1, 1, P, P, P, P, P, None, None) == 2        # no f_z
    assert lib.fm_gaussian_force(C.byref(g3), 9, 0.1, 1, P, P, P, P, P, P, None) == 7           # dtype
    assert lib.fm_gaussian_force_grad(C.byref(g2), 0, 0.1, 2, P, P, P, P, P, None, None, None, None, None,
                                      None) == 2                                                 # no outputs
    assert lib.fm_gaussian_force_grad(C.byref(g2), 0, 0.1, 1 << 25, P, P, P, P, P, None, P, P, P, P,
                                      None) == 2                                                 # n too large


# ------------------------------------------------------------------ GPU: kernels
def _dev(x, dtype):
    return torch.tensor(np.ascontiguousarray(x), dtype=dtype, device="cuda")


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("res", [(48, 40), (33, 17), (20, 16, 24), (12, 9, 17)])
def test_gaussian_force_matches_oracle(fm, cuda, dtype, res):
    K = importlib.import_module("differentiable-flowmap_b200.kernels")
    npt = np.float64 if dtype == torch.float64 else np.float32
    g = K.GridSpec(res)
    dx = 1.0 / res[0]
    c, r, s = _params(res, 300, len(res) * 100 + res[1], npt)
    want = FO.gaussian_force(res, dx, c, r, s)
    f = [torch.full(g.face_shape(k), 7.0, dtype=dtype, device="cuda") for k in range(len(res))]
    K.gaussian_force(g, dx, _dev(c, dtype), _dev(r, dtype), _dev(s, dtype), f)
    torch.cuda.synchronize()
    scale = max(np.abs(w).max() for w in want)
    assert scale > 0
    tol = 1e-12 if dtype == torch.float64 else 2e-6
    for k in range(len(res)):
        np.testing.assert_allclose(f[k].cpu().numpy(), want[k], rtol=0, atol=tol * scale)
    # the faces no Gaussian reaches are exactly zero on both sides
    for k in range(len(res)):
        assert np.array_equal(f[k].cpu().numpy() == 0, want[k] == 0)
    # n = 0 writes zeros everywhere
    K.gaussian_force(g, dx, _dev(c[:0], dtype), _dev(r[:0], dtype), _dev(s[:0], dtype), f)
    torch.cuda.synchronize()
    assert all(float(x.abs().max()) == 0.0 for x in f)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("res", [(40, 36), (16, 20, 12)])
def test_gaussian_force_grad_matches_oracle(fm, cuda, dtype, res):
    K = importlib.import_module("differentiable-flowmap_b200.kernels")
    npt = np.float64 if dtype == torch.float64 else np.float32
    g = K.GridSpec(res)
    dx = 1.0 / res[0]
    c, r, s = _params(res, 80, 11 + len(res), npt)
    rng = np.random.default_rng(5)
    adj = [rng.normal(size=g.face_shape(k)).astype(npt) for k in range(len(res))]
    want = FO.gaussian_force_grad(res, dx, c, r, s, adj)
    got = K.gaussian_force_grad(g, dx, _dev(c, dtype), _dev(r, dtype), _dev(s, dtype), [_dev(a, dtype) for a in adj])
    torch.cuda.synchronize()
    tol = 1e-10 if dtype == torch.float64 else 1e-4
    for gv, wv in zip(got, want):
        gv = gv.cpu().numpy()
        scale = np.abs(wv).max()
        assert scale > 0
        np.testing.assert_allclose(gv, wv, rtol=0, atol=tol * scale)
    # NaN radius and the sub-cell support reach no face: all four sums are zero
    for gv in got:
        assert float(gv[-4].abs().max()) == 0.0 and float(gv[-1].abs().max()) == 0.0


# ------------------------------------------------------------------ GPU: simulator
SIM_CASES = {
    # name: (res, steps, R, rk, backward_u, dt, gaussians per step, adjoint reads the stored forces)
    "2d_rk2": ((32, 32), 8, 3, 2, True, 0.01, 40, True),
    "2d_rk2_reevaluated": ((32, 32), 8, 3, 2, True, 0.01, 40, False),
    "2d_rk4_ckpt": ((32, 32), 7, 4, 4, False, 0.01, 40, True),
    "3d_rk4": ((16, 16, 16), 6, 4, 4, True, 0.02, 30, True),
}


def _sim_inputs(res, steps, ng, npt):
    C_ = importlib.import_module("differentiable-flowmap_b200.configs")
    dx = 1.0 / res[0]
    dim = len(res)
    rng = np.random.default_rng(3)
    u0 = C_.split_central_vector(rng.normal(0.0, 0.2, size=(dim,) + tuple(res)))
    rho0 = C_.smooth_ball(res, (0.5,) * dim, 0.25, dx)
    rho_t = C_.smooth_ball(res, (0.55,) * dim, 0.2, dx)
    forces = []
    for n in range(steps):
        c, r, s = FO.random_gaussians(ng, dim, dx, 1000 + n, npt)
        forces.append((c, r, s * 20.0))  # strong enough to move the loss visibly
    return u0, rho0, rho_t, forces


def _levels(res):
    return max(2, int(np.log2(min(res))) - 3 + 1)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SIM_CASES))
def test_simulator_with_control_forces_matches_oracle(fm, cuda, name):
    res, steps, R, rk, bu, dt, ng, store = SIM_CASES[name]
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    u0, rho0, rho_t, forces = _sim_inputs(res, steps, ng, np.float64)
    mg = MGParams(_levels(res), 2, 50, 0, 40, 0.0, 1e-22, 0.0)
    o = OracleSim(res, 1.0 / res[0], dt, R, steps, rk=rk, backward_u=bu, prec="f64", mg=mg, control_forces=forces)
    lo, go = o.gradient(u0, rho0, rho_t)

    solver = S.SolverConfig(levels=_levels(res), bottom=50, max_iters=40, abs_tol=0.0, rel_tol=1e-22, eps=0.0)
    cfg = S.FlowmapConfig(res=res, dx=1.0 / res[0], dt=dt, total_steps=steps, reinit_every=R, RK_number=rk,
                          backward_u=bu, dtype=torch.float64, solver=solver, add_control_force=True, control_num=64,
                          store_control_force=store)
    sim = S.LFM_Diff_Simulator(config=cfg)
    paras = [{"c": c, "r": r, "s": s, "n": len(r)} for c, r, s in forces]
    lc, gc = sim.gradient(u0, rho0, rho_t, control_forces=paras)
    gc = [x.cpu().numpy() for x in gc]

    def rel(a, b):
        num = np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(a, b)))
        den = np.sqrt(sum(np.sum(y ** 2) for y in b))
        return 0.0 if num == 0.0 else num / den  # the last step's adjoint velocity is zero on both sides

    assert abs(lc - lo) / abs(lo) < 1e-9
    assert rel(gc, go) < 1e-7
    assert sorted(sim.control_force_grads) == list(range(steps))
    for n in range(steps):
        got = [t.cpu().numpy() for t in sim.control_force_grads[n]]
        want = o.cf_grads[n]
        for k in range(4):
            assert rel([got[k]], [want[k]]) < 1e-7, (n, k)
    # the forces matter: the run without them has a different loss
    o2 = OracleSim(res, 1.0 / res[0], dt, R, steps, rk=rk, backward_u=bu, prec="f64", mg=mg)
    l2, _ = o2.gradient(u0, rho0, rho_t)
    assert abs(l2 - lo) > 1e-6 * abs(lo)


@pytest.mark.gpu
def test_reference_style_step_api(fm, cuda):
    """The reference driver's calls: forward_step_midpoint / backtrack_step_midpoint
    with control_force_para dicts, then .to_numpy() of the gradient fields."""
    res, steps = (32, 32), 4
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    u0, rho0, rho_t, forces = _sim_inputs(res, steps, 20, np.float32)
    cfg = S.FlowmapConfig(res=res, dx=1 / 32, dt=0.01, total_steps=steps, reinit_every=3, RK_number=2,
                          add_control_force=True, control_num=32)
    sim = S.LFM_Diff_Simulator(config=cfg)
    sim.init(theta=u0, init_passive_np=rho0)
    while True:
        c, r, s = forces[sim.step_num[None] + 1]
        _, final = sim.forward_step_midpoint(True, True, control_force_para={"c": c, "r": r, "s": s, "n": len(r)})
        if final:
            break
    sim.init_gradient(target_passive=rho_t)
    while True:
        c, r, s = forces[sim.step_num[None] - 1]
        _, done = sim.backtrack_step_midpoint(False, False, control_force_para={"c": c, "r": r, "s": s, "n": len(r)})
        g = sim.adj_gaussion_force_strength.to_numpy()
        assert g.shape == (32, 2) and np.all(g[20:] == 0) and np.all(np.isfinite(g))
        if done:
            break
