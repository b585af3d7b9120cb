"""Host-side logic of the per-kernel autograd Functions, checked on the CPU
against the oracle: the Adams-Bashforth-3 coefficients that AccumulateInit's
backward pass applies must be the linear coefficients of the oracle's
accumulate_init_new (3D/flowmap.py:503-545, its ind == 1 formula included)."""
import importlib

import numpy as np
import pytest

from oracle import Oracle


def _A():
    return importlib.import_module("differentiable-flowmap_b200.autograd")


@pytest.mark.parametrize("ind", [0, 1, 2, 7])
def test_ab3_coefficients_match_oracle(ind):
    shape = (6, 7, 8)
    d, dx, dt = 3, 1.0 / 7, 0.37
    rng = np.random.default_rng(40 + ind)
    o = Oracle(shape, "f64")
    face = [tuple(n + (a == c) for a, n in enumerate(shape)) for c in range(d)]
    f = [rng.uniform(-1, 1, size=s) for s in face]
    F = [rng.uniform(-1, 1, size=(d,) + s) for s in face]
    phi = [np.stack(np.meshgrid(*[(np.arange(n) + (0.0 if a == c else 0.5)) * dx for a, n in enumerate(s)],
                                indexing="ij")) + rng.uniform(-0.5 * dx, 0.5 * dx, size=(d,) + s)
           for c, s in enumerate(face)]
    Hp = [rng.uniform(-1, 1, size=s) for s in face]
    Hpp = [rng.uniform(-1, 1, size=s) for s in face]
    zeros = [np.zeros(s) for s in face]
    # F . f(phi) per face node, from the oracle's pullback (advect_u)
    Fv = [np.zeros(s) for s in face]
    o.advect_u(f, Fv, F, phi, dx)
    c_fv, c_hp, c_hpp = _A()._ab3_coefs(True, ind, dt)

    init = [np.zeros(s) for s in face]
    hp, hpp = [x.copy() for x in zeros], [x.copy() for x in zeros]
    o.accumulate_init_new(f, init, F, phi, hp, hpp, ind, dx, dt)
    for c in range(d):
        np.testing.assert_allclose(init[c], c_fv * Fv[c], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(hp[c], Fv[c], rtol=1e-12, atol=1e-14)  # history shift: Hp' = F . f
    init = [np.zeros(s) for s in face]
    hp, hpp = [x.copy() for x in Hp], [x.copy() for x in Hpp]
    o.accumulate_init_new([x * 0 for x in f], init, F, phi, hp, hpp, ind, dx, dt)
    for c in range(d):
        np.testing.assert_allclose(init[c], c_hp * Hp[c] + c_hpp * Hpp[c], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(hpp[c], Hp[c], rtol=0, atol=0)  # Hpp' = Hp


def test_plain_accumulate_coefficient_is_dt():
    assert _A()._ab3_coefs(False, 5, 0.25) == (0.25, 0.0, 0.0)
