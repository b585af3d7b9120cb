"""Per-kernel adjoints: the backward passes of the autograd Functions in
differentiable-flowmap_b200/autograd.py (fm_*_adj kernels and the projection).

Three independent checks:

1. torch.autograd.gradcheck in FP64 on small grids: the full Jacobian of the
   CUDA forward kernel by central differences against the hand-written
   adjoint kernel (vector-Jacobian products), for every differentiable input.
2. The linear part against the FP64 oracle by the dot-product identity
   <A f, lam> = <f, A^T lam>: A f from the oracle's forward kernel, A^T lam
   from the CUDA adjoint.
3. The nonlinear part (velocity through the RK backtrace, sample positions,
   Jacobian rows) against central differences of the FP64 oracle's forward
   along random directions.
"""
import numpy as np
import pytest
import torch

from oracle import Oracle

pytestmark = pytest.mark.gpu

SMALL = [(5, 6, 7), (9, 11)]
MEDIUM = [(12, 16, 20), (24, 40)]


def _A(fm):
    import importlib

    return importlib.import_module("differentiable-flowmap_b200.autograd")


def _mac(rng, shape, scale, dev, grad=True):
    out = []
    for c in range(len(shape)):
        s = list(shape)
        s[c] += 1
        out.append(torch.tensor(rng.uniform(-scale, scale, size=s), dtype=torch.float64, device=dev,
                                requires_grad=grad))
    return out


def _pos(rng, node_shape, dx, dev, spread=2.5, grad=True):
    """Positions near the nodes of `node_shape`, a few far outside the box (clamped)."""
    dim = len(node_shape)
    base = np.stack(np.meshgrid(*[(np.arange(n) + 0.5) * dx for n in node_shape], indexing="ij"))
    p = base + rng.uniform(-spread * dx, spread * dx, size=base.shape)
    flat = p.reshape(dim, -1)
    flat[:, ::9] = rng.uniform(-0.3, 1.3, size=(dim, flat[:, ::9].shape[1]))
    return torch.tensor(p, dtype=torch.float64, device=dev, requires_grad=grad)


def _face(shape, c):
    s = list(shape)
    s[c] += 1
    return tuple(s)


def _gradcheck(fn, inputs):
    # atomic accumulation: repeated backward passes agree to rounding only
    assert torch.autograd.gradcheck(fn, inputs, eps=1e-6, atol=1e-6, rtol=1e-4, nondet_tol=1e-12)


@pytest.mark.parametrize("shape", SMALL, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("rk", [2, 4])
def test_advect_scalar_grid_gradcheck(fm, cuda, shape, rk):
    A = _A(fm)
    rng = np.random.default_rng(11)
    dx = 1.0 / shape[1]
    u0 = _mac(rng, shape, 1.0, cuda)
    s1 = torch.tensor(rng.uniform(-1, 1, size=shape), dtype=torch.float64, device=cuda, requires_grad=True)
    _gradcheck(lambda s, *u: A.advect_scalar_grid(list(u), s, dx, 0.7 * dx, rk), (s1, *u0))


@pytest.mark.parametrize("shape", SMALL, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("rk", [2, 4])
def test_advect_u_grid_gradcheck(fm, cuda, shape, rk):
    A = _A(fm)
    rng = np.random.default_rng(12)
    dx = 1.0 / shape[1]
    d = len(shape)
    u0 = _mac(rng, shape, 1.0, cuda)
    u1 = _mac(rng, shape, 1.0, cuda)
    _gradcheck(lambda *u: tuple(A.advect_u_grid(list(u[:d]), list(u[d:]), dx, 0.7 * dx, rk)), (*u0, *u1))
    # self-advection: the two paths' gradients add
    _gradcheck(lambda *u: tuple(A.advect_u_grid(list(u), list(u), dx, 0.7 * dx, rk)), tuple(u0))


@pytest.mark.parametrize("shape", SMALL, ids=lambda s: "x".join(map(str, s)))
def test_pullback_u_gradcheck(fm, cuda, shape):
    A = _A(fm)
    rng = np.random.default_rng(13)
    dx = 1.0 / shape[1]
    d = len(shape)
    u0 = _mac(rng, shape, 1.0, cuda)
    T = [torch.tensor(rng.uniform(-1, 1, size=(d,) + _face(shape, c)), dtype=torch.float64, device=cuda,
                      requires_grad=True) for c in range(d)]
    psi = [_pos(rng, _face(shape, c), dx, cuda) for c in range(d)]
    base = _mac(rng, shape, 1.0, cuda)

    def fn(*x):
        return tuple(A.pullback_u(list(x[:d]), list(x[d:2 * d]), list(x[2 * d:3 * d]), dx, 0.5, -1.0,
                                  list(x[3 * d:])))

    _gradcheck(fn, (*u0, *T, *psi, *base))
    _gradcheck(lambda *x: tuple(A.pullback_u(list(x[:d]), list(x[d:2 * d]), list(x[2 * d:]), dx)), (*u0, *T, *psi))


@pytest.mark.parametrize("shape", SMALL, ids=lambda s: "x".join(map(str, s)))
def test_pullback_scalar_gradcheck(fm, cuda, shape):
    A = _A(fm)
    rng = np.random.default_rng(14)
    dx = 1.0 / shape[1]
    s0 = torch.tensor(rng.uniform(-1, 1, size=shape), dtype=torch.float64, device=cuda, requires_grad=True)
    psi = _pos(rng, shape, dx, cuda)
    base = torch.tensor(rng.uniform(-1, 1, size=shape), dtype=torch.float64, device=cuda, requires_grad=True)
    _gradcheck(lambda s, p, b: A.pullback_scalar(s, p, dx, -1.0, -1.0, b), (s0, psi, base))
    _gradcheck(lambda s, p: A.pullback_scalar(s, p, dx), (s0, psi))


@pytest.mark.parametrize("shape", SMALL, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("rk", [2, 4])
def test_rk_grid_gradcheck(fm, cuda, shape, rk):
    """Flow map and Jacobian row marched through u: gradients in psi, T and u
    (the T update differentiated through the B-spline's second derivative)."""
    A = _A(fm)
    rng = np.random.default_rng(19)
    dx = 1.0 / shape[1]
    d = len(shape)
    u = _mac(rng, shape, 1.0, cuda)
    for face in [0, d - 1, -1]:
        node = _face(shape, face) if face >= 0 else shape
        psi = _pos(rng, node, dx, cuda, spread=1.5)
        if face >= 0:
            T = torch.tensor(rng.uniform(-1, 1, size=(d,) + node), dtype=torch.float64, device=cuda,
                             requires_grad=True)
            _gradcheck(lambda p, t, *v: A.rk_grid(list(v), p, t, face, dx, 0.7 * dx, rk), (psi, T, *u))
        else:
            _gradcheck(lambda p, *v: A.rk_grid(list(v), p, None, face, dx, 0.7 * dx, rk), (psi, *u))


@pytest.mark.parametrize("shape", SMALL, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("ab3,ind", [(False, 0), (True, 0), (True, 1), (True, 3)])
def test_accumulate_init_gradcheck(fm, cuda, shape, ab3, ind):
    A = _A(fm)
    rng = np.random.default_rng(20)
    dx = 1.0 / shape[1]
    d = len(shape)
    f = _mac(rng, shape, 1.0, cuda)
    init = _mac(rng, shape, 1.0, cuda)
    F = [torch.tensor(rng.uniform(-1, 1, size=(d,) + _face(shape, c)), dtype=torch.float64, device=cuda,
                      requires_grad=True) for c in range(d)]
    phi = [_pos(rng, _face(shape, c), dx, cuda) for c in range(d)]
    if ab3:
        Hp, Hpp = _mac(rng, shape, 1.0, cuda), _mac(rng, shape, 1.0, cuda)

        def fn(*x):
            out = A.accumulate_init(list(x[:d]), list(x[d:2 * d]), list(x[2 * d:3 * d]), list(x[3 * d:4 * d]),
                                    dx, 0.3, list(x[4 * d:5 * d]), list(x[5 * d:]), ind)
            return tuple(out[0] + out[1] + out[2])

        _gradcheck(fn, (*f, *init, *F, *phi, *Hp, *Hpp))
    else:
        _gradcheck(lambda *x: tuple(A.accumulate_init(list(x[:d]), list(x[d:2 * d]), list(x[2 * d:3 * d]),
                                                      list(x[3 * d:]), dx, 0.3)), (*f, *init, *F, *phi))


@pytest.mark.parametrize("shape", [(16, 16), (16, 16, 16)], ids=lambda s: "x".join(map(str, s)))
def test_project_is_self_adjoint(fm, cuda, shape):
    A = _A(fm)
    rng = np.random.default_rng(15)
    sol = fm.MGPCG(shape, torch.float64, levels=2, bottom=50, max_iters=60, abs_tol=1e-24, rel_tol=1e-26, eps=0.0)
    a = _mac(rng, shape, 1.0, cuda, grad=False)
    b = _mac(rng, shape, 1.0, cuda, grad=False)
    Pa, Pb = A.project(sol, a), A.project(sol, b)
    lhs = sum(torch.sum(x * y).item() for x, y in zip(Pa, b))
    rhs = sum(torch.sum(x * y).item() for x, y in zip(a, Pb))
    assert abs(lhs - rhs) < 1e-10 * max(abs(lhs), 1.0), (lhs, rhs)
    PPa = A.project(sol, Pa)  # idempotent
    assert max((x - y).abs().max().item() for x, y in zip(PPa, Pa)) < 1e-10
    # the backward pass is P of the incoming gradient
    u = _mac(rng, shape, 1.0, cuda)
    w = _mac(rng, shape, 1.0, cuda, grad=False)
    loss = sum(torch.sum(x * y) for x, y in zip(A.project(sol, u), w))
    loss.backward()
    Pw = A.project(sol, w)
    assert max((x.grad - y).abs().max().item() for x, y in zip(u, Pw)) < 1e-10
    if len(shape) == 2:
        assert torch.autograd.gradcheck(lambda *x: tuple(A.project(sol, list(x))), tuple(u), eps=1e-6, atol=1e-6,
                                        rtol=1e-4, fast_mode=True)


def _np(t):
    return t.detach().cpu().numpy()


def _dot(a, b):
    return float(sum(np.sum(np.asarray(x, np.float64) * np.asarray(y, np.float64)) for x, y in zip(a, b)))


@pytest.mark.parametrize("shape", MEDIUM, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("rk", [2, 4])
def test_advect_adjoints_match_oracle(fm, cuda, shape, rk):
    """Transpose in the sampled field (dot-product identity) and derivative in
    u0 (oracle central differences) of advect_scalar_grid and advect_u_grid."""
    rng = np.random.default_rng(16)
    o = Oracle(shape, "f64")
    g = fm.GridSpec(shape)
    d = len(shape)
    dx = 1.0 / shape[1]
    dt = 0.7 * dx
    u0 = [rng.uniform(-1, 1, size=_face(shape, c)) for c in range(d)]
    u1 = [rng.uniform(-1, 1, size=_face(shape, c)) for c in range(d)]
    s1 = rng.uniform(-1, 1, size=shape)
    lam_s = rng.uniform(-1, 1, size=shape)
    lam_u = [rng.uniform(-1, 1, size=_face(shape, c)) for c in range(d)]
    T = lambda a: torch.tensor(a, dtype=torch.float64, device=cuda)  # noqa: E731

    def fwd_s(u):
        out = np.zeros(shape)
        o.advect_scalar_grid(rk, u, s1, out, dx, dt)
        return out

    def fwd_u(u):
        out = [np.zeros(_face(shape, c)) for c in range(d)]
        o.advect_u_grid(rk, u, u1, out, dx, dt)
        return out

    # CUDA adjoints
    gs_u0 = [torch.zeros(_face(shape, c), dtype=torch.float64, device=cuda) for c in range(d)]
    gs_s1 = torch.zeros(shape, dtype=torch.float64, device=cuda)
    fm.kernels.advect_scalar_grid_adj(g, rk, dx, dt, [T(x) for x in u0], T(s1), T(lam_s), gs_u0, gs_s1)
    gu_u0 = [torch.zeros(_face(shape, c), dtype=torch.float64, device=cuda) for c in range(d)]
    gu_u1 = [torch.zeros(_face(shape, c), dtype=torch.float64, device=cuda) for c in range(d)]
    fm.kernels.advect_u_grid_adj(g, rk, dx, dt, [T(x) for x in u0], [T(x) for x in u1], [T(x) for x in lam_u],
                                 gu_u0, gu_u1)
    torch.cuda.synchronize()

    # linear part: <A f, lam> = <f, A^T lam>
    lhs = _dot([fwd_s(u0)], [lam_s])
    assert abs(lhs - _dot([s1], [_np(gs_s1)])) < 1e-12 * abs(lhs)
    out = fwd_u(u0)
    lhs = _dot(out, lam_u)
    assert abs(lhs - _dot(u1, [_np(x) for x in gu_u1])) < 1e-12 * abs(lhs)

    # u0 through the backtrace: directional central differences of the oracle
    h = 1e-6
    for trial in range(2):
        delta = [rng.standard_normal(_face(shape, c)) for c in range(d)]
        up = [x + h * y for x, y in zip(u0, delta)]
        um = [x - h * y for x, y in zip(u0, delta)]
        fd = (_dot([fwd_s(up)], [lam_s]) - _dot([fwd_s(um)], [lam_s])) / (2 * h)
        an = _dot(delta, [_np(x) for x in gs_u0])
        assert abs(fd - an) < 1e-6 * max(abs(an), 1e-3), ("scalar", trial, fd, an)
        fd = (_dot(fwd_u(up), lam_u) - _dot(fwd_u(um), lam_u)) / (2 * h)
        an = _dot(delta, [_np(x) for x in gu_u0])
        assert abs(fd - an) < 1e-6 * max(abs(an), 1e-3), ("u", trial, fd, an)


@pytest.mark.parametrize("shape", MEDIUM, ids=lambda s: "x".join(map(str, s)))
def test_pullback_adjoints_match_oracle(fm, cuda, shape):
    """pullback_u (advect_u) and pullback_scalar (advect_scalar): transpose in the
    sampled field, derivatives in psi and T by oracle central differences."""
    rng = np.random.default_rng(17)
    o = Oracle(shape, "f64")
    g = fm.GridSpec(shape)
    d = len(shape)
    dx = 1.0 / shape[1]
    u0 = [rng.uniform(-1, 1, size=_face(shape, c)) for c in range(d)]
    Tm = [rng.uniform(-1, 1, size=(d,) + _face(shape, c)) for c in range(d)]
    psi = [_np(_pos(rng, _face(shape, c), dx, cuda, grad=False)) for c in range(d)]
    lam = [rng.uniform(-1, 1, size=_face(shape, c)) for c in range(d)]
    s0 = rng.uniform(-1, 1, size=shape)
    psi_c = _np(_pos(rng, shape, dx, cuda, grad=False))
    lam_c = rng.uniform(-1, 1, size=shape)
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=cuda)  # noqa: E731
    Z = lambda a: torch.zeros(np.shape(a), dtype=torch.float64, device=cuda)  # noqa: E731

    def fwd_u(u, Tm_, psi_):
        out = [np.zeros(_face(shape, c)) for c in range(d)]
        o.advect_u(u, out, Tm_, psi_, dx)
        return _dot(out, lam)

    def fwd_s(s, p):
        out = np.zeros(shape)
        o.advect_scalar(s, out, p, dx)
        return _dot([out], [lam_c])

    g_u0, g_T, g_psi = [Z(x) for x in u0], [Z(x) for x in Tm], [Z(x) for x in psi]
    fm.kernels.pullback_u_adj(g, dx, [T(x) for x in u0], [T(x) for x in Tm], [T(x) for x in psi],
                              [T(x) for x in lam], 1.0, 0.0, g_u0, g_T, g_psi)
    g_s0, g_pc = Z(s0), Z(psi_c)
    fm.kernels.pullback_scalar_adj(g, dx, T(s0), T(psi_c), T(lam_c), 1.0, 0.0, g_s0, g_pc)
    torch.cuda.synchronize()

    lhs = fwd_u(u0, Tm, psi)
    assert abs(lhs - _dot(u0, [_np(x) for x in g_u0])) < 1e-12 * abs(lhs)
    assert abs(lhs - _dot(Tm, [_np(x) for x in g_T])) < 1e-12 * abs(lhs)  # linear in T as well
    lhs = fwd_s(s0, psi_c)
    assert abs(lhs - _dot([s0], [_np(g_s0)])) < 1e-12 * abs(lhs)

    h = 1e-7
    for trial in range(2):
        dp = [rng.standard_normal(x.shape) * dx for x in psi]
        fd = (fwd_u(u0, Tm, [x + h * y for x, y in zip(psi, dp)])
              - fwd_u(u0, Tm, [x - h * y for x, y in zip(psi, dp)])) / (2 * h)
        an = _dot(dp, [_np(x) for x in g_psi])
        assert abs(fd - an) < 1e-6 * max(abs(an), 1e-3), ("psi_f", trial, fd, an)
        dpc = rng.standard_normal(psi_c.shape) * dx
        fd = (fwd_s(s0, psi_c + h * dpc) - fwd_s(s0, psi_c - h * dpc)) / (2 * h)
        an = _dot([dpc], [_np(g_pc)])
        assert abs(fd - an) < 1e-6 * max(abs(an), 1e-3), ("psi_c", trial, fd, an)


def test_fp32_adjoint_matches_fp64(fm, cuda):
    """The FP32 adjoint kernels agree with the FP64 ones to FP32 rounding."""
    rng = np.random.default_rng(18)
    shape = (16, 20, 24)
    g = fm.GridSpec(shape)
    d = 3
    dx = 1.0 / shape[1]
    u0 = [rng.uniform(-1, 1, size=_face(shape, c)) for c in range(d)]
    s1 = rng.uniform(-1, 1, size=shape)
    lam = rng.uniform(-1, 1, size=shape)
    res = {}
    for dt_ in (torch.float32, torch.float64):
        T = lambda a: torch.tensor(a, dtype=dt_, device=cuda)  # noqa: E731
        gu = [torch.zeros(_face(shape, c), dtype=dt_, device=cuda) for c in range(d)]
        gs = torch.zeros(shape, dtype=dt_, device=cuda)
        fm.kernels.advect_scalar_grid_adj(g, 4, dx, 0.7 * dx, [T(x) for x in u0], T(s1), T(lam), gu, gs)
        res[dt_] = [_np(x).astype(np.float64) for x in gu] + [_np(gs).astype(np.float64)]
    for a, b in zip(res[torch.float32], res[torch.float64]):
        assert np.abs(a - b).max() < 2e-5 * np.abs(b).max()


@pytest.mark.parametrize("shape", MEDIUM, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("rk", [2, 4])
def test_rk_grid_adjoint_matches_oracle(fm, cuda, shape, rk):
    """dL/du, dL/dpsi, dL/dT of one march against central differences of the
    FP64 oracle's RK_grid (L = <psi', lam> + <T', mu>)."""
    rng = np.random.default_rng(21)
    o = Oracle(shape, "f64")
    g = fm.GridSpec(shape)
    d = len(shape)
    dx = 1.0 / shape[1]
    dt = 0.7 * dx
    face = d - 1
    node = _face(shape, face)
    u = [rng.uniform(-1, 1, size=_face(shape, c)) for c in range(d)]
    psi = _np(_pos(rng, node, dx, cuda, spread=1.5, grad=False))
    Tm = rng.uniform(-1, 1, size=(d,) + node)
    lam = rng.uniform(-1, 1, size=psi.shape)
    mu = rng.uniform(-1, 1, size=Tm.shape)
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=cuda)  # noqa: E731

    def L(u_, psi_, T_):
        p, t = psi_.copy(), T_.copy()
        o.RK_grid(rk, face, p, t, [np.ascontiguousarray(x) for x in u_], dx, dt)
        return _dot([p, t], [lam, mu])

    g_psi, g_T = torch.zeros_like(T(psi)), torch.zeros_like(T(Tm))
    g_u = [torch.zeros(_face(shape, c), dtype=torch.float64, device=cuda) for c in range(d)]
    fm.kernels.rk_grid_adj(g, rk, dx, dt, face, T(psi), T(Tm), [T(x) for x in u], T(lam), T(mu), g_psi, g_T, g_u)
    torch.cuda.synchronize()
    h = 1e-6
    for trial in range(2):
        du = [rng.standard_normal(x.shape) for x in u]
        dp = rng.standard_normal(psi.shape) * dx
        dT = rng.standard_normal(Tm.shape)
        fd = (L([x + h * y for x, y in zip(u, du)], psi, Tm) - L([x - h * y for x, y in zip(u, du)], psi, Tm)) / (2 * h)
        an = _dot(du, [_np(x) for x in g_u])
        assert abs(fd - an) < 1e-6 * max(abs(an), 1e-3), ("u", trial, fd, an)
        fd = (L(u, psi + h * dp, Tm) - L(u, psi - h * dp, Tm)) / (2 * h)
        an = _dot([dp], [_np(g_psi)])
        assert abs(fd - an) < 1e-6 * max(abs(an), 1e-3), ("psi", trial, fd, an)
        fd = (L(u, psi, Tm + h * dT) - L(u, psi, Tm - h * dT)) / (2 * h)
        an = _dot([dT], [_np(g_T)])
        assert abs(fd - an) < 1e-6 * max(abs(an), 1e-3), ("T", trial, fd, an)


@pytest.mark.parametrize("check_every", [4, 0], ids=["host-checked", "device-loop"])
@pytest.mark.parametrize("shape", [(16, 16), (16, 16, 16)], ids=lambda s: "x".join(map(str, s)))
def test_projection_of_a_zero_field_with_eps_zero(fm, cuda, shape, check_every):
    """A zero right-hand side (the backward pass of a loss that does not depend
    on the projected field) ends the solve at once: z.r = 0 means r = 0, and
    with eps = 0 the first step would otherwise divide 0 by 0."""
    import importlib

    M = importlib.import_module("differentiable-flowmap_b200.mgpcg")
    sol = fm.MGPCG(shape, torch.float64, levels=2, bottom=50, max_iters=60, abs_tol=1e-24, rel_tol=1e-26, eps=0.0,
                   check_every=check_every)
    u = [torch.zeros(_face(shape, c), dtype=torch.float64, device=cuda) for c in range(len(shape))]
    sol.project(u)
    torch.cuda.synchronize()
    assert all(torch.count_nonzero(x).item() == 0 for x in u)
    if len(shape) == 2:  # the masked solver: a solid block in the middle
        mask = torch.zeros(shape)
        mask[5:9, 6:10] = 1.0
        ssol = M.SolidMGPCG(shape, mask, torch.float64, levels=2, abs_tol=1e-24, rel_tol=1e-26, eps=0.0,
                            check_every=check_every)
        ssol.project(u)
        torch.cuda.synchronize()
        assert all(torch.count_nonzero(x).item() == 0 for x in u)


def test_fp32_march_and_pullback_adjoints_match_fp64(fm, cuda):
    """The FP32 march and pullback adjoint kernels agree with their FP64 versions to
    FP32 rounding (relative to each gradient's scale)."""
    rng = np.random.default_rng(22)
    shape = (16, 20, 24)
    g = fm.GridSpec(shape)
    d = 3
    dx = 1.0 / shape[1]
    u = [rng.uniform(-1, 1, size=_face(shape, c)) for c in range(d)]
    node = _face(shape, 2)
    psi = _np(_pos(rng, node, dx, cuda, spread=1.5, grad=False))
    Tm = rng.uniform(-1, 1, size=(d,) + node)
    lam, mu = rng.uniform(-1, 1, size=psi.shape), rng.uniform(-1, 1, size=Tm.shape)
    Tf = [rng.uniform(-1, 1, size=(d,) + _face(shape, c)) for c in range(d)]
    pf = [_np(_pos(rng, _face(shape, c), dx, cuda, grad=False)) for c in range(d)]
    lo = [rng.uniform(-1, 1, size=_face(shape, c)) for c in range(d)]
    res = {}
    for dt_ in (torch.float32, torch.float64):
        T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dt_, device=cuda)  # noqa: E731
        Z = lambda a: torch.zeros(np.shape(a), dtype=dt_, device=cuda)  # noqa: E731
        gp, gT, gu = Z(psi), Z(Tm), [Z(x) for x in u]
        fm.kernels.rk_grid_adj(g, 4, dx, 0.7 * dx, 2, T(psi), T(Tm), [T(x) for x in u], T(lam), T(mu), gp, gT, gu)
        hu, hT, hp = [Z(x) for x in u], [Z(x) for x in Tf], [Z(x) for x in pf]
        fm.kernels.pullback_u_adj(g, dx, [T(x) for x in u], [T(x) for x in Tf], [T(x) for x in pf],
                                  [T(x) for x in lo], 1.0, 0.0, hu, hT, hp)
        res[dt_] = [gp, gT] + gu + hu + hT + hp
    for a, b in zip(res[torch.float32], res[torch.float64]):
        a, b = _np(a).astype(np.float64), _np(b)
        assert np.abs(a - b).max() < 1e-4 * max(np.abs(b).max(), 1e-30)
