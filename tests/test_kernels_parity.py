"""Kernel-level parity: every CUDA entry point vs the CPU oracle on the same
seeded inputs (FP64 CUDA vs FP64 oracle, FP32 CUDA vs FP32 oracle).

Tolerances: FP64 agree to 1e-10 relative to the field scale (only summation
order differs); FP32 to 2e-5.
"""
import numpy as np
import pytest
import torch

from oracle import MGParams, Oracle

pytestmark = pytest.mark.gpu

GRIDS = [(16, 16, 16), (12, 16, 20), (32, 32), (24, 40)]
PRECS = [("f64", torch.float64, 1e-10), ("f32", torch.float32, 2e-5)]


def _rand_mac(rng, shape, scale):
    dim = len(shape)
    out = []
    for c in range(dim):
        s = list(shape)
        s[c] += 1
        out.append(rng.uniform(-scale, scale, size=s))
    return out


def _rand_pos(rng, shape, grid_shape, dx, spread=2.5):
    """Positions near the nodes of `grid_shape` plus a few outside the box."""
    dim = len(shape)
    base = np.stack(np.meshgrid(*[(np.arange(n) + 0.5) * dx for n in grid_shape], indexing="ij"))
    p = base + rng.uniform(-spread * dx, spread * dx, size=base.shape)
    p.reshape(dim, -1)[:, ::7] = rng.uniform(-0.1, 1.1, size=(dim, p.reshape(dim, -1)[:, ::7].shape[1]))
    return p


def _t(a, dtype, dev):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)


def _np(t):
    return t.detach().cpu().numpy().astype(np.float64)


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


@pytest.fixture(params=GRIDS, ids=lambda s: "x".join(map(str, s)))
def shape(request):
    return request.param


@pytest.fixture(params=PRECS, ids=lambda p: p[0])
def prec(request):
    return request.param


def setup(shape, prec, seed=0):
    rng = np.random.default_rng(seed)
    name, dtype, tol = prec
    o = Oracle(shape, name)
    dx = 1.0 / shape[1]
    return rng, o, dtype, tol, dx


@pytest.mark.parametrize("rk", [2, 4])
def test_advect_u_grid(fm, cuda, shape, prec, rk):
    rng, o, dtype, tol, dx = setup(shape, prec)
    g = fm.GridSpec(shape)
    u0 = _rand_mac(rng, shape, 1.0)
    u1 = _rand_mac(rng, shape, 1.0)
    dt = 0.7 * dx
    ref = [np.zeros_like(x, dtype=o.dtype) for x in u0]
    o.advect_u_grid(rk, [x.astype(o.dtype) for x in u0], [x.astype(o.dtype) for x in u1], ref, dx, dt)
    out = [torch.zeros(x.shape, dtype=dtype, device=cuda) for x in u0]
    fm.kernels.advect_u_grid(g, rk, dx, dt, [_t(x, dtype, cuda) for x in u0], [_t(x, dtype, cuda) for x in u1], out)
    torch.cuda.synchronize()
    for c in range(len(shape)):
        assert _rel(_np(out[c]), ref[c]) < tol


@pytest.mark.parametrize("rk", [2, 4])
def test_advect_scalar_grid(fm, cuda, shape, prec, rk):
    rng, o, dtype, tol, dx = setup(shape, prec, 1)
    g = fm.GridSpec(shape)
    u0 = _rand_mac(rng, shape, 1.0)
    s1 = rng.uniform(0, 1, size=shape)
    dt = 0.7 * dx
    ref = np.zeros(shape, o.dtype)
    o.advect_scalar_grid(rk, [x.astype(o.dtype) for x in u0], s1.astype(o.dtype), ref, dx, dt)
    out = torch.zeros(shape, dtype=dtype, device=cuda)
    fm.kernels.advect_scalar_grid(g, rk, dx, dt, [_t(x, dtype, cuda) for x in u0], _t(s1, dtype, cuda), out)
    torch.cuda.synchronize()
    assert _rel(_np(out), ref) < tol


@pytest.mark.parametrize("rk", [2, 4])
@pytest.mark.parametrize("face", [-1, 0, 1])
def test_rk_grid(fm, cuda, shape, prec, rk, face):
    rng, o, dtype, tol, dx = setup(shape, prec, 2)
    g = fm.GridSpec(shape)
    dim = len(shape)
    u = _rand_mac(rng, shape, 1.0)
    gshape = shape if face < 0 else g.face_shape(face)
    psi = _rand_pos(rng, shape, gshape, dx)
    T = None if face < 0 else rng.uniform(-1, 1, size=(dim,) + tuple(gshape))
    for dt in (0.6 * dx, -0.6 * dx):
        p_ref = psi.astype(o.dtype).copy()
        T_ref = None if T is None else T.astype(o.dtype).copy()
        o.RK_grid(rk, face, p_ref, T_ref, [x.astype(o.dtype) for x in u], dx, dt)
        p_d = _t(psi, dtype, cuda)
        T_d = None if T is None else _t(T, dtype, cuda)
        fm.kernels.rk_grid(g, rk, dx, dt, face, p_d, T_d, [_t(x, dtype, cuda) for x in u])
        torch.cuda.synchronize()
        assert _rel(_np(p_d), p_ref) < tol
        if T is not None:
            assert _rel(_np(T_d), T_ref) < tol * 10


def test_march_map_matches_per_grid(fm, cuda, shape, prec):
    rng, o, dtype, tol, dx = setup(shape, prec, 3)
    g = fm.GridSpec(shape)
    dim = len(shape)
    u = [_t(x, dtype, cuda) for x in _rand_mac(rng, shape, 1.0)]
    psi_c = _t(_rand_pos(rng, shape, shape, dx), dtype, cuda)
    psi_f = [_t(_rand_pos(rng, shape, g.face_shape(c), dx), dtype, cuda) for c in range(dim)]
    T_f = [_t(rng.uniform(-1, 1, size=(dim,) + g.face_shape(c)), dtype, cuda) for c in range(dim)]
    a = [x.clone() for x in [psi_c] + psi_f + T_f]
    for rk in (2, 4):
        fm.kernels.march_map(g, rk, dx, 0.5 * dx, a[0], a[1:1 + dim], a[1 + dim:], u)
        b = [x.clone() for x in [psi_c] + psi_f + T_f]
        fm.kernels.rk_grid(g, rk, dx, 0.5 * dx, -1, b[0], None, u)
        for c in range(dim):
            fm.kernels.rk_grid(g, rk, dx, 0.5 * dx, c, b[1 + c], b[1 + dim + c], u)
        for x, y in zip(a, b):
            assert torch.equal(x, y)
        a = [x.clone() for x in [psi_c] + psi_f + T_f]


def test_pullback_u_and_bfecc_epilogues(fm, cuda, shape, prec):
    rng, o, dtype, tol, dx = setup(shape, prec, 4)
    g = fm.GridSpec(shape)
    dim = len(shape)
    u0 = _rand_mac(rng, shape, 1.0)
    psi = [_rand_pos(rng, shape, g.face_shape(c), dx) for c in range(dim)]
    T = [rng.uniform(-1, 1, size=(dim,) + g.face_shape(c)) for c in range(dim)]
    base = _rand_mac(rng, shape, 1.0)
    ref = [np.zeros(g.face_shape(c), o.dtype) for c in range(dim)]
    o.advect_u([x.astype(o.dtype) for x in u0], ref, [x.astype(o.dtype) for x in T], [x.astype(o.dtype) for x in psi],
               dx)
    out = [torch.zeros(g.face_shape(c), dtype=dtype, device=cuda) for c in range(dim)]
    U0 = [_t(x, dtype, cuda) for x in u0]
    Td = [_t(x, dtype, cuda) for x in T]
    Pd = [_t(x, dtype, cuda) for x in psi]
    fm.kernels.pullback_u(g, dx, U0, out, Td, Pd)
    torch.cuda.synchronize()
    for c in range(dim):
        assert _rel(_np(out[c]), ref[c]) < tol
    # err = 0.5 * (pull - base) ; final = base - pull
    B = [_t(x, dtype, cuda) for x in base]
    fm.kernels.pullback_u(g, dx, U0, out, Td, Pd, alpha=0.5, beta=-1.0, base=B)
    for c in range(dim):
        assert _rel(_np(out[c]), 0.5 * (ref[c] - base[c])) < tol
    Bc = [x.clone() for x in B]
    fm.kernels.pullback_u(g, dx, U0, Bc, Td, Pd, alpha=-1.0, beta=-1.0, base=Bc)
    for c in range(dim):
        assert _rel(_np(Bc[c]), base[c] - ref[c]) < tol


def test_pullback_scalar(fm, cuda, shape, prec):
    rng, o, dtype, tol, dx = setup(shape, prec, 5)
    g = fm.GridSpec(shape)
    s0 = rng.uniform(0, 1, size=shape)
    psi = _rand_pos(rng, shape, shape, dx)
    ref = np.zeros(shape, o.dtype)
    o.advect_scalar(s0.astype(o.dtype), ref, psi.astype(o.dtype), dx)
    out = torch.zeros(shape, dtype=dtype, device=cuda)
    fm.kernels.pullback_scalar(g, dx, _t(s0, dtype, cuda), out, _t(psi, dtype, cuda))
    torch.cuda.synchronize()
    assert _rel(_np(out), ref) < tol


@pytest.mark.parametrize("ab3,ind", [(0, 0), (1, 0), (1, 1), (1, 2), (1, 5)])
def test_accumulate_init(fm, cuda, shape, prec, ab3, ind):
    rng, o, dtype, tol, dx = setup(shape, prec, 6)
    g = fm.GridSpec(shape)
    dim = len(shape)
    f = _rand_mac(rng, shape, 1.0)
    init = _rand_mac(rng, shape, 1.0)
    F = [rng.uniform(-1, 1, size=(dim,) + g.face_shape(c)) for c in range(dim)]
    phi = [_rand_pos(rng, shape, g.face_shape(c), dx) for c in range(dim)]
    Hp = _rand_mac(rng, shape, 1.0)
    Hpp = _rand_mac(rng, shape, 1.0)
    dt = -2 * 0.3 * dx
    cv = lambda L: [np.array(x, dtype=o.dtype, copy=True) for x in L]
    init_r, Hp_r, Hpp_r = cv(init), cv(Hp), cv(Hpp)
    if ab3:
        o.accumulate_init_new(cv(f), init_r, cv(F), cv(phi), Hp_r, Hpp_r, ind, dx, dt)
    else:
        o.accumulate_init(cv(f), init_r, cv(F), cv(phi), dx, dt)
    T_ = lambda L: [_t(x, dtype, cuda) for x in L]
    init_d, Hp_d, Hpp_d = T_(init), T_(Hp), T_(Hpp)
    if ab3:
        fm.kernels.accumulate_init(g, dx, dt, T_(f), init_d, T_(F), T_(phi), Hp_d, Hpp_d, ind)
    else:
        fm.kernels.accumulate_init(g, dx, dt, T_(f), init_d, T_(F), T_(phi))
    torch.cuda.synchronize()
    for c in range(dim):
        assert _rel(_np(init_d[c]), init_r[c]) < tol
        if ab3:
            assert _rel(_np(Hp_d[c]), Hp_r[c]) < tol
            assert _rel(_np(Hpp_d[c]), Hpp_r[c]) < tol


@pytest.mark.parametrize("ab3,ind", [(0, 0), (1, 1), (1, 4)])
def test_accumulate_init_pair_equals_two_calls(fm, cuda, shape, prec, ab3, ind):
    """fm_accumulate_init_pair equals accumulate_init followed by a plain one of the
    second field through the same maps, bit for bit (histories included)."""
    rng, o, dtype, tol, dx = setup(shape, prec, 7)
    g = fm.GridSpec(shape)
    dim = len(shape)
    T_ = lambda xs: [_t(x, dtype, cuda) for x in xs]  # noqa: E731
    f, f2, init = (_rand_mac(rng, shape, 1.0) for _ in range(3))
    F = [rng.uniform(-1, 1, size=(dim,) + g.face_shape(c)) for c in range(dim)]
    phi = [_rand_pos(rng, shape, g.face_shape(c), dx) for c in range(dim)]
    Hp, Hpp = _rand_mac(rng, shape, 1.0), _rand_mac(rng, shape, 1.0)
    a_init, a_hp, a_hpp = T_(init), T_(Hp), T_(Hpp)
    b_init, b_hp, b_hpp = T_(init), T_(Hp), T_(Hpp)
    if ab3:
        fm.kernels.accumulate_init(g, dx, -0.02, T_(f), a_init, T_(F), T_(phi), a_hp, a_hpp, ind)
    else:
        fm.kernels.accumulate_init(g, dx, -0.02, T_(f), a_init, T_(F), T_(phi))
    fm.kernels.accumulate_init(g, dx, -0.01, T_(f2), a_init, T_(F), T_(phi))
    fm.kernels.accumulate_init_pair(g, dx, -0.02, T_(f), b_init, T_(F), T_(phi), T_(f2), -0.01,
                                    b_hp if ab3 else None, b_hpp if ab3 else None, ind)
    torch.cuda.synchronize()
    for c in range(dim):
        assert torch.equal(a_init[c], b_init[c])
        if ab3:
            assert torch.equal(a_hp[c], b_hp[c]) and torch.equal(a_hpp[c], b_hpp[c])


@pytest.mark.parametrize("order", [3, 4])
def test_nabla_u_w(fm, cuda, shape, prec, order):
    rng, o, dtype, tol, dx = setup(shape, prec, 7)
    g = fm.GridSpec(shape)
    dim = len(shape)
    u = _rand_mac(rng, shape, 1.0)
    w = _rand_mac(rng, shape, 1.0)
    ref = [np.zeros(g.face_shape(c), o.dtype) for c in range(dim)]
    cv = lambda L: [np.array(x, dtype=o.dtype, copy=True) for x in L]
    o.calculate_nabla_u_w(cv(u), cv(w), ref, dx, order)
    out = [torch.zeros(g.face_shape(c), dtype=dtype, device=cuda) for c in range(dim)]
    fm.kernels.nabla_u_w(g, dx, [_t(x, dtype, cuda) for x in u], [_t(x, dtype, cuda) for x in w], out, order)
    torch.cuda.synchronize()
    for c in range(dim):
        assert _rel(_np(out[c]), ref[c]) < tol


def test_nabla_scalar_adjoint(fm, cuda, shape, prec):
    rng, o, dtype, tol, dx = setup(shape, prec, 8)
    g = fm.GridSpec(shape)
    dim = len(shape)
    s = rng.uniform(0, 1, size=shape)
    a = rng.uniform(-1, 1, size=shape)
    ref = [np.zeros(g.face_shape(c), o.dtype) for c in range(dim)]
    o.calculate_nabla_scalar_adjoint(s.astype(o.dtype), a.astype(o.dtype), ref, dx)
    out = [torch.zeros(g.face_shape(c), dtype=dtype, device=cuda) for c in range(dim)]
    fm.kernels.nabla_scalar_adjoint(g, dx, _t(s, dtype, cuda), _t(a, dtype, cuda), out)
    torch.cuda.synchronize()
    for c in range(dim):
        assert _rel(_np(out[c]), ref[c]) < tol


def test_reset_to_identity(fm, cuda, shape, prec):
    rng, o, dtype, tol, dx = setup(shape, prec, 9)
    g = fm.GridSpec(shape)
    dim = len(shape)
    psi_r = np.zeros((dim,) + tuple(shape), o.dtype)
    pf_r = [np.zeros((dim,) + g.face_shape(c), o.dtype) for c in range(dim)]
    Tf_r = [np.zeros((dim,) + g.face_shape(c), o.dtype) for c in range(dim)]
    o.reset_to_identity(psi_r, pf_r, Tf_r, dx)
    psi = torch.full((dim,) + tuple(shape), 7.0, dtype=dtype, device=cuda)
    pf = [torch.full((dim,) + g.face_shape(c), 7.0, dtype=dtype, device=cuda) for c in range(dim)]
    Tf = [torch.full((dim,) + g.face_shape(c), 7.0, dtype=dtype, device=cuda) for c in range(dim)]
    fm.kernels.reset_to_identity(g, dx, psi, pf, Tf)
    torch.cuda.synchronize()
    assert np.array_equal(_np(psi), psi_r)
    for c in range(dim):
        assert np.array_equal(_np(pf[c]), pf_r[c])
        assert np.array_equal(_np(Tf[c]), Tf_r[c])


def test_project_matches_oracle(fm, cuda, shape, prec):
    """Poisson(u): projected velocity vs the oracle solved to high accuracy."""
    rng, o, dtype, tol, dx = setup(shape, prec, 10)
    g = fm.GridSpec(shape)
    dim = len(shape)
    u = _rand_mac(rng, shape, 1.0)
    levels = max(2, int(np.log2(min(shape))) - 3 + 1)
    abs_tol = 1e-24 if prec[0] == "f64" else 0.0
    rel_tol = 1e-26 if prec[0] == "f64" else 1e-12
    eps = 0.0 if prec[0] == "f64" else 1e-12
    P = MGParams(levels, 2, 50, 0, 60, abs_tol, rel_tol, eps)
    ref = [x.astype(o.dtype).copy() for x in u]
    o.Poisson(P, ref)
    sol = fm.MGPCG(shape, dtype, levels=levels, bottom=50, max_iters=60, abs_tol=abs_tol, rel_tol=rel_tol, eps=eps)
    ud = [_t(x, dtype, cuda) for x in u]
    sol.project(ud)
    torch.cuda.synchronize()
    ptol = 1e-9 if prec[0] == "f64" else 5e-4
    for c in range(dim):
        assert _rel(_np(ud[c]), ref[c]) < ptol
    # projected field is discretely divergence-free
    div = np.zeros(shape, o.dtype)
    o.divergence([np.ascontiguousarray(_np(x), o.dtype) for x in ud], div)
    scale = max(np.abs(x).max() for x in u)
    assert np.abs(div).max() < (1e-9 if prec[0] == "f64" else 2e-3) * scale


def test_vcycle_iterations_match_oracle(fm, cuda):
    """Same preconditioner => same PCG convergence history length (FP64)."""
    shape = (32, 32, 32)
    rng = np.random.default_rng(11)
    o = Oracle(shape, "f64")
    b = rng.standard_normal(shape)
    b -= b.mean()
    P = MGParams(3, 2, 50, 0, 200, 0.0, 1e-20, 0.0)
    x_ref = np.zeros(shape)
    it_ref, rtr_ref, conv_ref = o.mgpcg_solve(P, b, x_ref)
    sol = fm.MGPCG(shape, torch.float64, levels=3, bottom=50, max_iters=200, abs_tol=0.0, rel_tol=1e-20,
                   eps=0.0, check_every=1)
    x = torch.zeros(shape, dtype=torch.float64, device=cuda)
    it, rtr = sol.solve(torch.tensor(b, device=cuda), x)
    assert conv_ref and sol.last_converged
    assert abs(it - it_ref) <= 1
    assert _rel(x.cpu().numpy(), x_ref) < 1e-8


# (shape, levels, pre_post, bottom, bottom_mode): the first cases run the coarse
# levels as one cluster launch (slabs of 2..8 planes, 2..8 CTAs; 128^3 after two
# per-level launches), (16,16,16)/2 and (48,48)/2 the single-CTA bottom kernel,
# (160,160)/2 per-sweep bottom launches.
VCYCLE_CASES = [
    ((128, 128, 128), 5, 2, 50, 0),
    ((32, 32, 32), 3, 2, 50, 0),
    ((64, 64, 64), 4, 2, 50, 0),
    ((24, 16, 32), 3, 2, 50, 0),
    ((64, 64), 4, 2, 50, 0),
    ((128, 96), 3, 1, 20, 1),
    ((32, 48, 16), 3, 3, 7, 1),
    ((64, 32), 5, 2, 0, 0),
    ((16, 16, 16), 2, 2, 50, 0),
    ((48, 48), 2, 2, 10, 1),
    ((160, 160), 2, 1, 3, 0),
    # innermost extents 18 / 42 (not multiples of 4) and an odd bottom extent (9)
    ((16, 16, 18), 2, 2, 50, 0),
    ((32, 42), 2, 2, 20, 1),
]


@pytest.mark.parametrize("case", VCYCLE_CASES, ids=lambda c: "x".join(map(str, c[0])) + f"-L{c[1]}-pp{c[2]}-b{c[3]}m{c[4]}")
@pytest.mark.parametrize("pname", ["f64", "f32"])
def test_vcycle_bitwise_matches_oracle(fm, cuda, case, pname):
    """One preconditioner application (apply_preconditioner, 3D/mgpcg.py:187-205)
    equals the oracle's sequential V-cycle bit for bit: same operations, same
    order, no FMA contraction, on every launch path of the coarse levels."""
    shape, levels, pre_post, bottom, mode = case
    dtype = torch.float64 if pname == "f64" else torch.float32
    o = Oracle(shape, pname)
    rng = np.random.default_rng(sum(shape) + levels)
    r = rng.standard_normal(shape).astype(o.dtype)
    P = MGParams(levels, pre_post, bottom, mode, 1, 0.0, 0.0, 0.0)
    z_ref = np.zeros(shape, o.dtype)
    o.mg_vcycle(P, r.copy(), z_ref)
    sol = fm.MGPCG(shape, dtype, levels=levels, pre_post=pre_post, bottom=bottom, bottom_mode=mode)
    z = sol.apply_preconditioner(torch.tensor(r, device=cuda))
    z2 = sol.apply_preconditioner(torch.tensor(r, device=cuda))  # the solver's buffers start dirty now
    zn = z.cpu().numpy()
    assert np.array_equal(zn, z_ref), np.abs(zn - z_ref).max()
    assert torch.equal(z, z2)


@pytest.mark.parametrize("shape", [(32, 32, 32), (64, 64)])
def test_project_device_mode_matches_host_mode(fm, cuda, shape):
    """check_every=0 (conditional WHILE graph, no host sync) gives the same
    projection and iteration count as the host-checked loop; stats count solves."""
    rng = np.random.default_rng(12)
    g = fm.GridSpec(shape)
    levels = int(np.log2(min(shape))) - 3 + 1
    u = [torch.tensor(rng.uniform(-1, 1, size=g.face_shape(c)), dtype=torch.float64, device=cuda)
         for c in range(len(shape))]
    a = [x.clone() for x in u]
    b = [x.clone() for x in u]
    host = fm.MGPCG(shape, torch.float64, levels=levels, rel_tol=1e-10, abs_tol=0.0, eps=0.0, check_every=1)
    dev = fm.MGPCG(shape, torch.float64, levels=levels, rel_tol=1e-10, abs_tol=0.0, eps=0.0, check_every=0)
    host.project(a)
    dev.project(b)
    st = dev.stats(reset=True)
    assert st["solves"] == 1 and st["not_converged"] == 0 and st["nonfinite"] == 0
    assert st["last_iters"] == host.last_iters
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    for _ in range(3):
        dev.project([x.clone() for x in u])
    st = dev.stats()
    assert st["solves"] == 3 and st["iterations"] == 3 * host.last_iters


@pytest.mark.parametrize("rk", [2, 4])
def test_paired_advection_equals_two_calls(fm, cuda, shape, rk):
    """fm_advect_u_grid_pair / fm_advect_scalar_grid_pair share one backtrace and
    reproduce two single calls bit for bit."""
    rng = np.random.default_rng(21)
    g = fm.GridSpec(shape)
    dx = 1.0 / shape[1]
    T_ = lambda L: [_t(x, torch.float32, cuda) for x in L]
    u0, u1, v1 = T_(_rand_mac(rng, shape, 1.0)), T_(_rand_mac(rng, shape, 1.0)), T_(_rand_mac(rng, shape, 1.0))
    a2, b2 = [torch.empty_like(x) for x in u0], [torch.empty_like(x) for x in u0]
    c2, d2 = [torch.empty_like(x) for x in u0], [torch.empty_like(x) for x in u0]
    fm.kernels.advect_u_grid_pair(g, rk, dx, -0.6 * dx, u0, u1, a2, v1, b2)
    fm.kernels.advect_u_grid(g, rk, dx, -0.6 * dx, u0, u1, c2)
    fm.kernels.advect_u_grid(g, rk, dx, -0.6 * dx, u0, v1, d2)
    for x, y in zip(a2 + b2, c2 + d2):
        assert torch.equal(x, y)
    s, t = _t(rng.uniform(size=shape), torch.float32, cuda), _t(rng.uniform(size=shape), torch.float32, cuda)
    s2, t2, s3, t3 = [torch.empty_like(s) for _ in range(4)]
    fm.kernels.advect_scalar_grid_pair(g, rk, dx, -0.6 * dx, u0, s, s2, t, t2)
    fm.kernels.advect_scalar_grid(g, rk, dx, -0.6 * dx, u0, s, s3)
    fm.kernels.advect_scalar_grid(g, rk, dx, -0.6 * dx, u0, t, t3)
    assert torch.equal(s2, s3) and torch.equal(t2, t3)


@pytest.mark.parametrize("order", [3, 4])
@pytest.mark.parametrize("big", [(40, 48, 72), (17, 35, 66)], ids=lambda s: "x".join(map(str, s)))
def test_adjoint_sources_multi_tile(fm, cuda, big, prec, order):
    """The 3D adjoint-source stencils on grids spanning several CTA tiles and
    i-chunks in every direction, with interior tiles (shared-weight fast paths)
    and ragged, clamped edges: nabla_u_w and nabla_scalar_adjoint vs the oracle."""
    rng, o, dtype, tol, dx = setup(big, prec, 17)
    g = fm.GridSpec(big)
    u = _rand_mac(rng, big, 1.0)
    w = _rand_mac(rng, big, 1.0)
    ref = [np.zeros(g.face_shape(c), o.dtype) for c in range(3)]
    cv = lambda L: [np.array(x, dtype=o.dtype, copy=True) for x in L]
    o.calculate_nabla_u_w(cv(u), cv(w), ref, dx, order)
    out = [torch.zeros(g.face_shape(c), dtype=dtype, device=cuda) for c in range(3)]
    fm.kernels.nabla_u_w(g, dx, [_t(x, dtype, cuda) for x in u], [_t(x, dtype, cuda) for x in w], out, order)
    torch.cuda.synchronize()
    for c in range(3):
        assert _rel(_np(out[c]), ref[c]) < tol
    if order == 3:
        s = rng.uniform(0, 1, size=big)
        a = rng.uniform(-1, 1, size=big)
        ref = [np.zeros(g.face_shape(c), o.dtype) for c in range(3)]
        o.calculate_nabla_scalar_adjoint(s.astype(o.dtype), a.astype(o.dtype), ref, dx)
        out = [torch.zeros(g.face_shape(c), dtype=dtype, device=cuda) for c in range(3)]
        fm.kernels.nabla_scalar_adjoint(g, dx, _t(s, dtype, cuda), _t(a, dtype, cuda), out)
        torch.cuda.synchronize()
        for c in range(3):
            assert _rel(_np(out[c]), ref[c]) < tol
