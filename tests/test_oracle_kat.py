"""Known-answer tests pinning the CPU oracle (no GPU).

The reference ships no golden vectors for this path, so the oracle is pinned
by properties the restated mathematics must satisfy exactly: B-spline
partition of unity and derivative consistency, exact reproduction of
polynomials by the interpolants, the boundary clamp band, the MGPCG solve
(A x = b to tolerance), projection giving a discretely divergence-free field,
FP32 vs FP64 agreement, and hand-computed values of the reference formulas.
"""
import numpy as np
import pytest

from oracle import MGParams, Oracle


@pytest.mark.parametrize("order", [2, 3, 4])
def test_bspline_partition_of_unity(order):
    o = Oracle((8, 8, 8))
    x = np.linspace(0, 1, 101)
    tot = sum(o.bspline(order, x - k) for k in range(-5, 6))
    dtot = sum(o.bspline(order, x - k, True) for k in range(-5, 6))
    assert np.abs(tot - 1).max() < 1e-13
    assert np.abs(dtot).max() < 1e-12


@pytest.mark.parametrize("order", [2, 3, 4])
def test_bspline_derivative_is_derivative(order):
    o = Oracle((8, 8, 8))
    x = np.linspace(-3, 3, 1201)
    h = 1e-6
    fd = (o.bspline(order, x + h) - o.bspline(order, x - h)) / (2 * h)
    assert np.abs(fd - o.bspline(order, x, True)).max() < 1e-5


def test_bspline_known_values():
    o = Oracle((8, 8, 8))
    # quadratic: N(0)=3/4, N(1)=1/8 ; cubic: N(0)=2/3, N(1)=1/6 ; quartic: N(0)=115/192
    assert o.bspline(2, np.array([0.0, 1.0, 1.5]))[:3].tolist() == [0.75, 0.125, 0.0]
    np.testing.assert_allclose(o.bspline(3, np.array([0.0, 1.0, 2.0])), [2 / 3, 1 / 6, 0.0], atol=1e-15)
    np.testing.assert_allclose(o.bspline(4, np.array([0.0, 2.5])), [115 / 192, 0.0], atol=1e-15)
    np.testing.assert_allclose(o.bspline(4, np.array([1.0])), [55 / 96 + 5 / 24 - 5 / 4 + 5 / 6 - 1 / 6], atol=1e-15)


@pytest.mark.parametrize("order", [2, 3, 4])
@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 24)])
def test_interp_reproduces_linear_fields(order, shape):
    dim = len(shape)
    n = shape[0]
    dx = 1.0 / shape[1]
    o = Oracle(shape)
    s = list(shape)
    s[0] += 1
    idx = np.meshgrid(*[np.arange(v) for v in s], indexing="ij")
    X = [idx[0] * dx] + [(idx[a] + 0.5) * dx for a in range(1, dim)]
    coef = [2.0, 3.0, -1.0][:dim]
    f = 1.0 + sum(c * x for c, x in zip(coef, X))
    rng = np.random.default_rng(0)
    for _ in range(20):
        # interior points (away from the clamp band)
        p = rng.uniform(4 * dx, (min(shape) - 5) * dx, size=dim)
        v, gr = o.interp_grad(order, f, p, dx, [0.0] + [0.5] * (dim - 1))
        assert abs(v - (1 + np.dot(coef, p))) < 1e-12
        np.testing.assert_allclose(gr, coef, atol=1e-10)


def test_interp_clamp_band():
    """Positions outside [1, n-2] (in index space) clamp to the band edge."""
    o = Oracle((16, 16, 16))
    dx = 1 / 16
    rng = np.random.default_rng(1)
    f = rng.standard_normal((17, 16, 16))
    v_lo, _ = o.interp_grad(2, f, [-0.3, 0.5, 0.5], dx, [0, 0.5, 0.5])
    v_edge, _ = o.interp_grad(2, f, [1 * dx, 0.5, 0.5], dx, [0, 0.5, 0.5])
    assert v_lo == v_edge
    v_hi, _ = o.interp_grad(2, f, [1.7, 0.5, 0.5], dx, [0, 0.5, 0.5])
    v_top, _ = o.interp_grad(2, f, [(17 - 2 - 1e-6) * dx, 0.5, 0.5], dx, [0, 0.5, 0.5])
    assert abs(v_hi - v_top) < 1e-12


@pytest.mark.parametrize("shape,levels", [((32, 32, 32), 3), ((64, 64), 4), ((16, 24, 32), 3)])
def test_mgpcg_solves(shape, levels):
    o = Oracle(shape)
    rng = np.random.default_rng(2)
    b = rng.standard_normal(shape)
    b -= b.mean()
    P = MGParams(levels, 2, 50, 0, 200, 0.0, 1e-24, 0.0)
    x = np.zeros(shape)
    it, rtr, conv = o.mgpcg_solve(P, b, x)
    assert conv and it < 60
    Ax = np.zeros(shape)
    o.laplacian(x, Ax)
    assert np.abs(Ax - b).max() < 1e-9


@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 32)])
def test_project_is_divergence_free_and_idempotent(shape):
    o = Oracle(shape)
    rng = np.random.default_rng(3)
    u = o.zeros_mac()
    for c in range(len(shape)):
        u[c][...] = rng.standard_normal(u[c].shape)
    P = MGParams(2, 2, 50, 0, 200, 0.0, 1e-26, 0.0)
    o.Poisson(P, u)
    div = o.zeros_cell()
    o.divergence(u, div)
    assert np.abs(div).max() < 1e-9
    u2 = [x.copy() for x in u]
    o.Poisson(P, u2)
    for a, b in zip(u, u2):
        assert np.abs(a - b).max() < 1e-9


def test_rk_grid_zero_velocity_is_identity():
    shape = (16, 16, 16)
    o = Oracle(shape)
    dx = 1 / 16
    psi, pf, Tf = o.zeros_cell(3), [o.zeros_face(c, 3) for c in range(3)], [o.zeros_face(c, 3) for c in range(3)]
    o.reset_to_identity(psi, pf, Tf, dx)
    p0, T0 = pf[1].copy(), Tf[1].copy()
    for rk in (2, 4):
        o.RK_grid(rk, 1, pf[1], Tf[1], o.zeros_mac(), dx, 0.1)
        assert np.array_equal(pf[1], p0) and np.array_equal(Tf[1], T0)


def test_rk_grid_uniform_flow_translates():
    """u = const: psi moves by -dt*u, T unchanged (grad u = 0)."""
    shape = (16, 16, 16)
    o = Oracle(shape)
    dx = 1 / 16
    u = o.zeros_mac()
    vel = [0.3, -0.2, 0.1]
    for c in range(3):
        u[c][...] = vel[c]
    psi, pf, Tf = o.zeros_cell(3), [o.zeros_face(c, 3) for c in range(3)], [o.zeros_face(c, 3) for c in range(3)]
    o.reset_to_identity(psi, pf, Tf, dx)
    p0 = pf[0].copy()
    o.RK_grid(4, 0, pf[0], Tf[0], u, dx, 0.05)
    for a in range(3):
        np.testing.assert_allclose(pf[0][a], p0[a] - 0.05 * vel[a], atol=1e-14)
    np.testing.assert_allclose(Tf[0][0], 1.0, atol=1e-14)


def test_accumulate_ab3_reference_formula():
    """The ind == 1 branch uses (23 Fv - 16 Fv + 5 H_prev)/12 (the reference's own formula)."""
    shape = (8, 8, 8)
    o = Oracle(shape)
    dx = 1 / 8
    f = o.zeros_mac()
    for c in range(3):
        f[c][...] = 1.0 + c
    init = o.zeros_mac()
    F, phi = [o.zeros_face(c, 3) for c in range(3)], [o.zeros_face(c, 3) for c in range(3)]
    psi = o.zeros_cell(3)
    o.reset_to_identity(psi, phi, F, dx)
    Hp = [np.full(o.face_shape(c), 0.5) for c in range(3)]
    Hpp = [np.full(o.face_shape(c), 0.25) for c in range(3)]
    o.accumulate_init_new(f, init, F, phi, Hp, Hpp, 1, dx, 0.1)
    for c in range(3):
        Fv = 1.0 + c
        np.testing.assert_allclose(init[c], (23 * Fv - 16 * Fv + 5 * 0.5) / 12 * 0.1, atol=1e-14)
        np.testing.assert_allclose(Hp[c], Fv, atol=1e-14)
        np.testing.assert_allclose(Hpp[c], 0.5, atol=1e-14)


@pytest.mark.parametrize("rk", [2, 4])
def test_f32_oracle_tracks_f64(rk):
    shape = (16, 16, 16)
    rng = np.random.default_rng(4)
    o64, o32 = Oracle(shape, "f64"), Oracle(shape, "f32")
    dx = 1 / 16
    u = [rng.uniform(-1, 1, size=o64.face_shape(c)) for c in range(3)]
    out64 = o64.zeros_mac()
    out32 = o32.zeros_mac()
    o64.advect_u_grid(rk, u, u, out64, dx, 0.03)
    u32 = [x.astype(np.float32) for x in u]
    o32.advect_u_grid(rk, u32, u32, out32, dx, 0.03)
    for a, b in zip(out64, out32):
        assert np.abs(a - b).max() < 1e-5
