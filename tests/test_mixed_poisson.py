"""Mixed-precision Poisson solve (fm_mgpcg_solve_dc): FP32 MGPCG inner solves
inside an FP64 defect correction, on the seeded k^-5/3 divergence RHS.

Checked against (1) an independent FP64 residual computed here with numpy,
(2) an FP64 MGPCG solve of the same system on the GPU and (3) the FP64 oracle
(the reference solver restated, 3D/mgpcg.py:207-289), pressures compared in the
mean-zero gauge (the all-Neumann operator is singular).
"""
import numpy as np
import pytest
import torch

from oracle import MGParams, Oracle

pytestmark = pytest.mark.gpu


def _laplacian64(x):
    """A x for the all-Neumann 5/7-point operator (diag = in-domain neighbours)."""
    out = np.zeros_like(x)
    for a in range(x.ndim):
        d = np.diff(x, axis=a)  # x[i+1] - x[i]
        lo = [slice(None)] * x.ndim
        hi = [slice(None)] * x.ndim
        lo[a] = slice(0, -1)
        hi[a] = slice(1, None)
        out[tuple(lo)] -= d  # x[i] - x[i+1]
        out[tuple(hi)] += d  # x[i+1] - x[i], i.e. x[j] - x[j-1] at j = i+1
    return out


def _gauge(x):
    x = np.asarray(x, np.float64)
    return x - x.mean()


def _rhs(C, shape, seed=30):
    return C.divergence_rhs(C.split_central_vector(C.spectrum_velocity(shape, seed=seed)))


@pytest.mark.parametrize("shape", [(64, 64, 64), (128, 96), (48, 32, 40)])
def test_mixed_solve_reaches_fp64_residual(fm, cuda, shape):
    import importlib

    C = importlib.import_module("differentiable-flowmap_b200.configs")
    b = _rhs(C, shape)
    levels = max(2, int(np.log2(min(shape))) - 3 + 1)
    while any(n % (1 << (levels - 1)) for n in shape):
        levels -= 1
    sol = fm.MGPCG(shape, torch.float32, levels=levels, abs_tol=0.0, rel_tol=1e-8, max_iters=100, check_every=0)
    x, outer, inner, rel = sol.solve_mixed(torch.tensor(b, device=cuda), rel_tol=1e-10, max_outer=12)
    xh = x.cpu().numpy()
    bh = b.astype(np.float64) - b.astype(np.float64).mean()
    res = np.linalg.norm(bh - _laplacian64(xh)) / np.linalg.norm(bh)
    assert rel <= 1e-10 and res <= 1.5e-10, (rel, res, outer, inner)
    assert 1 <= outer <= 6
    # FP64 MGPCG on the GPU, solved far past the mixed tolerance
    s64 = fm.MGPCG(shape, torch.float64, levels=levels, abs_tol=0.0, rel_tol=1e-24, eps=0.0, max_iters=300,
                   check_every=1)
    x64 = torch.zeros(shape, dtype=torch.float64, device=cuda)
    s64.solve(torch.tensor(bh, device=cuda), x64)
    ref = _gauge(x64.cpu().numpy())
    err = np.linalg.norm(_gauge(xh) - ref) / np.linalg.norm(ref)
    assert err < 1e-8, err


def test_mixed_solve_matches_oracle_fp64(fm, cuda):
    import importlib

    C = importlib.import_module("differentiable-flowmap_b200.configs")
    shape = (32, 32, 32)
    b = _rhs(C, shape, seed=31)
    o = Oracle(shape, "f64")
    bh = b.astype(np.float64)
    x_ref = np.zeros(shape)
    it, rtr, conv = o.mgpcg_solve(MGParams(3, 2, 50, 0, 200, 0.0, 1e-24, 0.0), bh, x_ref)
    assert conv
    sol = fm.MGPCG(shape, torch.float32, levels=3, abs_tol=0.0, rel_tol=1e-8, max_iters=100)
    x, outer, inner, rel = sol.solve_mixed(torch.tensor(b, device=cuda), rel_tol=1e-11)
    err = np.linalg.norm(_gauge(x.cpu().numpy()) - _gauge(x_ref)) / np.linalg.norm(_gauge(x_ref))
    assert rel <= 1e-11 and err < 1e-9, (rel, err)


@pytest.mark.parametrize("shape,levels", [((128, 128, 128), 5), ((1024, 1024), 8)])
def test_bf16_coarse_levels(fm, cuda, shape, levels):
    """BF16 storage of the per-level coarse grids (64^3 at 128^3; 512^2, 256^2
    at 1024^2): the mixed solve still reaches the FP64 tolerance, and one V-cycle
    stays within BF16 rounding of the FP32 V-cycle."""
    import importlib

    C = importlib.import_module("differentiable-flowmap_b200.configs")
    b = torch.tensor(_rhs(C, shape), device=cuda)
    s32 = fm.MGPCG(shape, torch.float32, levels=levels, abs_tol=0.0, rel_tol=1e-8, max_iters=100)
    sbf = fm.MGPCG(shape, torch.float32, levels=levels, abs_tol=0.0, rel_tol=1e-8, max_iters=100, coarse_bf16=True)
    z32 = s32.apply_preconditioner(b)
    zbf = sbf.apply_preconditioner(b)
    dz = float((zbf - z32).norm() / z32.norm())
    assert 0 < dz < 2e-2, dz  # BF16 keeps 8 significant bits on the coarse corrections
    x, outer, inner, rel = sbf.solve_mixed(b, rel_tol=1e-10, max_outer=12)
    x32, outer32, inner32, rel32 = s32.solve_mixed(b, rel_tol=1e-10, max_outer=12)
    assert rel <= 1e-10 and outer <= outer32 + 2, (rel, outer, inner, outer32, inner32)
    err = float((_gauge_t(x) - _gauge_t(x32)).norm() / _gauge_t(x32).norm())
    assert err < 1e-8, err


def _gauge_t(x):
    return x - x.mean()


def test_mixed_solve_fp64_rhs_and_limits(fm, cuda):
    """FP64 right-hand side; max_outer = 0 reports the initial residual and
    FM_ERR_NOT_CONVERGED; a zero right-hand side returns x = 0 at once."""
    import importlib

    C = importlib.import_module("differentiable-flowmap_b200.configs")
    shape = (32, 32)
    b = torch.tensor(_rhs(C, shape).astype(np.float64), device=cuda)
    sol = fm.MGPCG(shape, torch.float32, levels=3, abs_tol=0.0, rel_tol=1e-8, max_iters=100)
    x, outer, inner, rel = sol.solve_mixed(b, rel_tol=1e-10)
    assert rel <= 1e-10 and outer >= 1
    x0, outer0, inner0, rel0 = sol.solve_mixed(b, rel_tol=1e-10, max_outer=0)
    assert outer0 == 0 and inner0 == 0 and abs(rel0 - 1.0) < 1e-12 and not sol.last_converged
    assert float(x0.abs().max()) == 0.0
    z, oz, iz, rz = sol.solve_mixed(torch.zeros_like(b), rel_tol=1e-10)
    assert oz == 0 and float(z.abs().max()) == 0.0


# ---------------------------------------------------------------- fm_project_dc
def _div64(u):
    """-div of a MAC velocity with the wall faces zeroed, in FP64 (numpy)."""
    out = None
    for c, f in enumerate(u):
        f = np.array(f, dtype=np.float64, copy=True)
        lo = [slice(None)] * f.ndim
        hi = [slice(None)] * f.ndim
        lo[c], hi[c] = 0, -1
        f[tuple(lo)] = 0.0
        f[tuple(hi)] = 0.0
        d = np.diff(f, axis=c)
        out = d if out is None else out + d
    return -out


@pytest.mark.parametrize("shape,levels", [((64, 64, 64), 4), ((256, 256), 5), ((48, 32, 40), 3)])
def test_project_dc_matches_fp64_projection(fm, cuda, shape, levels):
    """The FP32 projection with FP64 defect correction lands within FP32
    rounding of the FP64 projection of the same velocity, while the plain FP32
    projection at its tightest reachable tolerance stays far from it."""
    rng = np.random.default_rng(11)
    u = [rng.normal(size=tuple(n + (a == c) for a, n in enumerate(shape))).astype(np.float32)
         for c in range(len(shape))]
    s64 = fm.MGPCG(shape, torch.float64, levels=levels, abs_tol=0.0, rel_tol=1e-26, eps=0.0, max_iters=400,
                   check_every=0)
    u64 = [torch.tensor(x, dtype=torch.float64, device=cuda) for x in u]
    s64.project(u64)
    sdc = fm.MGPCG(shape, torch.float32, levels=levels, abs_tol=0.0, rel_tol=1e-6, max_iters=100, check_every=0,
                   dc_rel_tol=1e-10, dc_max_outer=8)
    udc = [torch.tensor(x, device=cuda) for x in u]
    p = torch.empty(shape, dtype=torch.float64, device=cuda)
    sdc.project(udc, p_out=p)
    st = sdc.stats(reset=True)
    assert st["not_converged"] == 0 and st["nonfinite"] == 0
    assert 1 <= st["solves"] <= 8  # inner solves, one per correction
    scale = max(float(x.abs().max()) for x in u64)
    err = max(float((a.double() - b).abs().max()) for a, b in zip(udc, u64)) / scale
    assert err < 2e-6, err
    # the FP64 residual of the returned pressure
    b = _div64(u)
    bh = b - b.mean()
    res = np.linalg.norm(bh - _laplacian64(p.cpu().numpy())) / np.linalg.norm(bh)
    assert res <= 1e-10, res
    # the plain FP32 projection at relative z.r 1e-8
    s32 = fm.MGPCG(shape, torch.float32, levels=levels, abs_tol=0.0, rel_tol=1e-8, max_iters=100, check_every=0)
    u32 = [torch.tensor(x, device=cuda) for x in u]
    s32.project(u32)
    err32 = max(float((a.double() - b).abs().max()) for a, b in zip(u32, u64)) / scale
    assert err < err32, (err, err32)


def test_project_dc_recorded_in_a_graph_equals_eager(fm, cuda):
    shape = (32, 32, 32)
    rng = np.random.default_rng(12)
    u = [rng.normal(size=tuple(n + (a == c) for a, n in enumerate(shape))).astype(np.float32) for c in range(3)]
    sdc = fm.MGPCG(shape, torch.float32, levels=3, abs_tol=0.0, rel_tol=1e-6, max_iters=100, check_every=0,
                   dc_rel_tol=1e-10, dc_max_outer=8)
    ue = [torch.tensor(x, device=cuda) for x in u]
    sdc.project(ue)
    ug = [torch.tensor(x, device=cuda) for x in u]
    src = [x.clone() for x in ug]
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        for a, b in zip(ug, src):
            a.copy_(b)
        sdc.project(ug)
    for _ in range(2):
        graph.replay()
        torch.cuda.synchronize()
        for a, b in zip(ug, ue):
            assert torch.equal(a, b)

