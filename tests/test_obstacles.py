"""Obstacle path: the solid-aware MGPCG (2D/vortex/mgpcg_solid.py) and the mask
kernels (2D/vortex/init_conditions.py:549-583, 3D/init_conditions.py:536-578).

CPU (oracle, solid_oracle.py): downsample_bm's all-children rule; a masked
projection leaves zero divergence in fluid cells and zero velocity on the
faces of solid cells; mask_passive averages fluid neighbours; the C ABI
rejects bad arguments without a device.
GPU: fm_solid_vcycle equals the oracle's V-cycle bit for bit (FP32 and FP64,
2D and 3D, masks with holes and odd shapes); fm_solid_project matches the
oracle's projection over the same 60 PCG iterations (FP64 to 1e-9 of the
field scale, FP32 to 2e-4); the mask
kernels equal the oracle bit for bit; the simulator with an obstacle (FP64)
matches the oracle's restatement: loss to 1e-9, dL/du0 to 1e-7 relative L2.
"""
import ctypes as C
import importlib

import numpy as np
import pytest
import torch

import solid_oracle as SO
from oracle import MGParams
from sim_oracle import OracleSim


def _mask2d(res, seed=0):
    """A disc, a thin wall and a one-cell pocket, seeded."""
    n0, n1 = res
    x = (np.arange(n0) + 0.5) / n0
    y = (np.arange(n1) + 0.5) / n1
    X, Y = np.meshgrid(x, y, indexing="ij")
    rng = np.random.default_rng(seed)
    cx, cy = 0.4 + 0.2 * rng.uniform(size=2)
    m = ((X - cx) ** 2 + (Y - cy) ** 2 < 0.12 ** 2).astype(np.float32)
    m[n0 // 5, n1 // 4: n1 // 2] = 1.0          # a wall one cell thick
    m[3 * n0 // 4, 3 * n1 // 4] = 1.0           # a single solid cell
    return m


def _mask3d(res):
    x = [(np.arange(n) + 0.5) / n for n in res]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    m = ((X - 0.45) ** 2 + (Y - 0.55) ** 2 + (Z - 0.5) ** 2 < 0.2 ** 2).astype(np.float32)
    m[2, :, :] = np.where(Y[2] < 0.5, 1.0, m[2])
    return m


def _mac(res, rng, dtype):
    dim = len(res)
    return [rng.normal(size=tuple(res[a] + (a == c) for a in range(dim))).astype(dtype) for c in range(dim)]


# ------------------------------------------------------------------ CPU
def test_downsample_all_children_rule():
    f = np.ones((4, 4), dtype=bool)
    f[0:2, 0:2] = False          # all four children solid -> coarse solid
    f[2, 2] = False              # one child solid -> coarse fluid
    c = SO.downsample(f)
    assert c.tolist() == [[False, True], [True, True]]


@pytest.mark.parametrize("res", [(32, 24), (16, 16, 8)])
def test_oracle_masked_projection_is_divergence_free(res):
    rng = np.random.default_rng(1)
    mask = _mask2d(res) if len(res) == 2 else _mask3d(res)
    fluid = ~(mask > 0)
    u = _mac(res, rng, np.float64)
    levels = 3 if len(res) == 2 else 2
    # the reference's tolerance (rTr < max(1e-14, 1e-16 zTr0)); recentring over all
    # cells, solid ones included, leaves a floor near rTr ~ 1e-15 in FP64
    x, it, rtr = SO.project(u, mask, levels, abs_tol=1e-14, rel_tol=1e-16, max_iters=200)
    div = SO.divergence(u, fluid)
    assert np.abs(div[fluid]).max() < 1e-6
    for c in range(len(res)):
        assert np.all(u[c][SO.faces_of_solids(fluid, c)] == 0)
    assert np.all(x[~fluid] == 0)
    assert it < 200


def test_oracle_mask_passive_mean_of_fluid_neighbours():
    s = np.arange(25, dtype=np.float64).reshape(5, 5)
    m = np.zeros((5, 5), np.float32)
    m[2, 2] = 1.0
    m[0, 0] = 1.0
    SO.mask_passive(s, m)
    nb = [s[i, j] for i in (1, 2, 3) for j in (1, 2, 3) if (i, j) != (2, 2)]
    assert s[2, 2] == sum(nb) / 8.0
    assert s[0, 0] == (1.0 + 5.0 + 6.0) / 3.0


def test_solid_arguments_rejected_without_device(fm):
    lib = fm._lib.lib()
    g = fm._lib.Grid(2, (C.c_int * 3)(32, 32, 1))
    h = C.c_void_p()
    P = fm._lib.MGParams(3, 2, 20, 1, 400, 1e-14, 1e-16, 1e-12, 4, 0)
    assert lib.fm_solid_create(C.byref(g), 0, None, None, C.byref(h)) == 2
    bad = fm._lib.MGParams(7, 2, 20, 1, 400, 1e-14, 1e-16, 1e-12, 4, 0)  # 32 not divisible by 2^6
    assert lib.fm_solid_create(C.byref(g), 0, C.byref(bad), None, C.byref(h)) == 1
    bf = fm._lib.MGParams(3, 2, 20, 1, 400, 1e-14, 1e-16, 1e-12, 4, 1)   # BF16 coarse levels: not here
    assert lib.fm_solid_create(C.byref(g), 0, C.byref(bf), None, C.byref(h)) == 2
    assert lib.fm_solid_project(None, None, None, None, None, None, None, None) == 2
    assert lib.fm_solid_vcycle(None, None, None, None) == 2
    assert lib.fm_mask_velocity(C.byref(g), 0, None, None, None, None, None, None) == 2
    assert lib.fm_mask_passive(C.byref(g), 0, None, None, 0, None) == 2
    assert P.levels == 3


# ------------------------------------------------------------------ GPU
def _solid(res, mask, dtype, levels, **kw):
    M = importlib.import_module("differentiable-flowmap_b200.mgpcg")
    return M.SolidMGPCG(res, torch.tensor(mask), dtype, levels=levels, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("res", [(64, 48), (40, 24), (32, 32, 16)])
def test_solid_vcycle_bitwise(fm, cuda, dtype, res):
    npt = np.float32 if dtype == torch.float32 else np.float64
    mask = _mask2d(res) if len(res) == 2 else _mask3d(res)
    levels = 3 if len(res) == 2 else 2
    S = _solid(res, mask, dtype, levels)
    r = np.random.default_rng(2).normal(size=res).astype(npt)
    for _ in range(2):  # the hierarchy keeps nothing between calls
        z = S.apply_preconditioner(torch.tensor(r, device="cuda"))
        torch.cuda.synchronize()
        want = SO.vcycle(r, ~(mask > 0), levels)
        np.testing.assert_array_equal(z.cpu().numpy(), want)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("res", [(64, 48), (32, 32, 16)])
def test_solid_project_matches_oracle(fm, cuda, dtype, res):
    npt = np.float32 if dtype == torch.float32 else np.float64
    mask = _mask2d(res) if len(res) == 2 else _mask3d(res)
    levels = 3 if len(res) == 2 else 2
    tight = dtype == torch.float64
    # an unreachable tolerance: both sides run the same 60 iterations (the masked
    # system's recentring floor is near rTr ~ 1e-15 in FP64)
    kw = dict(abs_tol=0.0, rel_tol=1e-30, max_iters=60)
    S = _solid(res, mask, dtype, levels, **kw)
    u = _mac(res, np.random.default_rng(3), npt)
    want = [x.copy() for x in u]
    x64, it, _ = SO.project(want, mask, levels, **kw)
    du = [torch.tensor(x, device="cuda") for x in u]
    p = torch.empty(res, dtype=dtype, device="cuda")
    S.project(du, p_out=p)
    torch.cuda.synchronize()
    assert S.last_iters == it == 60
    scale = max(np.abs(w).max() for w in want)
    tol = 1e-9 if tight else 2e-4
    for c in range(len(res)):
        np.testing.assert_allclose(du[c].cpu().numpy(), want[c], rtol=0, atol=tol * scale)
    np.testing.assert_allclose(p.cpu().numpy(), x64, rtol=0, atol=tol * np.abs(x64).max())


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("res", [(24, 20), (12, 10, 8)])
def test_mask_kernels_bitwise(fm, cuda, dtype, res):
    K = importlib.import_module("differentiable-flowmap_b200.kernels")
    npt = np.float32 if dtype == torch.float32 else np.float64
    g = K.GridSpec(res)
    rng = np.random.default_rng(4)
    mask = (rng.uniform(size=res) < 0.3).astype(np.float32) * rng.choice([0.5, 1.0, 2.0], size=res).astype(np.float32)
    u = _mac(res, rng, npt)
    bvel = rng.normal(size=(len(res),) + tuple(res)).astype(npt)
    s = rng.normal(size=res).astype(npt)
    dm = torch.tensor(mask, device="cuda")
    du = [torch.tensor(x, device="cuda") for x in u]
    da = [torch.tensor(x, device="cuda") for x in u]
    ds, dsa = torch.tensor(s, device="cuda"), torch.tensor(s, device="cuda")
    K.mask_velocity(g, dm, du, torch.tensor(bvel, device="cuda"))
    K.mask_velocity(g, dm, da)
    K.mask_passive(g, dm, ds)
    K.mask_passive(g, dm, dsa, adjoint=True)
    torch.cuda.synchronize()
    wu, wa = [x.copy() for x in u], [x.copy() for x in u]
    SO.mask_velocity(wu, mask, bvel)
    SO.mask_velocity(wa, mask)
    ws, wsa = s.copy(), s.copy()
    SO.mask_passive(ws, mask)
    SO.mask_adj_passive(wsa, mask)
    for c in range(len(res)):
        np.testing.assert_array_equal(du[c].cpu().numpy(), wu[c])
        np.testing.assert_array_equal(da[c].cpu().numpy(), wa[c])
    np.testing.assert_array_equal(ds.cpu().numpy(), ws)
    np.testing.assert_array_equal(dsa.cpu().numpy(), wsa)


CASES = {
    # name: (steps, R, rk, backward_u)
    "rk2": (8, 3, 2, True),
    "rk4_ckpt": (7, 4, 4, False),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_simulator_with_obstacle_matches_oracle(fm, cuda, name):
    steps, R, rk, bu = CASES[name]
    res, dt = (32, 32), 0.01
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    Cf = importlib.import_module("differentiable-flowmap_b200.configs")
    rng = np.random.default_rng(6)
    u0 = Cf.split_central_vector(rng.normal(0.0, 0.2, size=(2,) + res))
    rho0 = Cf.smooth_ball(res, (0.3, 0.5), 0.2, 1 / 32)
    rho_t = Cf.smooth_ball(res, (0.7, 0.5), 0.2, 1 / 32)
    mask = _mask2d(res, seed=3)
    mg = MGParams(3, 2, 20, 1, 40, 0.0, 1e-30, 0.0)  # 40 iterations per solve on both sides
    o = OracleSim(res, 1 / 32, dt, R, steps, rk=rk, backward_u=bu, prec="f64", mg=mg, mask=mask)
    lo, go = o.gradient(u0, rho0, rho_t)
    solver = S.SolverConfig(levels=3, bottom=20, bottom_mode=1, max_iters=40, abs_tol=0.0, rel_tol=1e-30, eps=0.0,
                            check_every=4)
    cfg = S.FlowmapConfig(res=res, dx=1 / 32, dt=dt, total_steps=steps, reinit_every=R, RK_number=rk,
                          backward_u=bu, dtype=torch.float64, solver=solver, boundary_mask=mask)
    sim = S.LFM_Diff_Simulator(config=cfg)
    assert type(sim.solver).__name__ == "SolidMGPCG"
    lc, gc = sim.gradient(u0, rho0, rho_t)
    gc = [x.cpu().numpy() for x in gc]
    num = np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(gc, go)))
    den = np.sqrt(sum(np.sum(y ** 2) for y in go))
    assert abs(lc - lo) / abs(lo) < 1e-9
    assert num / den < 1e-7
    fluid = ~(mask > 0)
    for c in range(2):
        assert np.all(gc[c][SO.faces_of_solids(fluid, c)] == 0)  # the adjoint velocity is masked


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_solid_vcycle_bitwise_on_the_reference_leaf_mask(fm, cuda, dtype):
    """The reference experiment's own obstacle (2D/vortex/data/leaf_mask_256_scaled.npz,
    7922 solid cells) at its size, 256^2 with the vortex solver's 5 levels, 20
    bottom sweeps as 10 x (R,B) + 10 x (B,R): bit-exact against the oracle."""
    Cf = importlib.import_module("differentiable-flowmap_b200.configs")
    mask = Cf.reference_fixtures()["leaf_mask"].astype(np.float32)
    assert mask.shape == (256, 256) and int(mask.sum()) == 7922
    npt = np.float32 if dtype == torch.float32 else np.float64
    S = _solid((256, 256), mask, dtype, 5, bottom=20, bottom_mode=1)
    r = np.random.default_rng(9).normal(size=(256, 256)).astype(npt)
    z = S.apply_preconditioner(torch.tensor(r, device="cuda"))
    torch.cuda.synchronize()
    want = SO.vcycle(r, ~(mask > 0), 5, bottom=20)
    np.testing.assert_array_equal(z.cpu().numpy(), want)
