"""ctypes bindings for the CPU oracle (oracle/fm_oracle.c).

TEST INFRASTRUCTURE ONLY.  This module is the parity checker for the CUDA
library: only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import it.  The product path never does.

Functions take numpy arrays laid out as the C file documents (C-order scalar
planes; vector fields as ``(dim, *grid_shape)`` SoA arrays) and mirror the
reference's kernel names (3D/flowmap.py, 3D/mgpcg.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


class Grid(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int * 3)]


class MGParams(C.Structure):
    _fields_ = [
        ("levels", C.c_int),
        ("pre_post", C.c_int),
        ("bottom", C.c_int),
        ("bottom_mode", C.c_int),
        ("max_iters", C.c_int),
        ("abs_tol", C.c_double),
        ("rel_tol", C.c_double),
        ("eps", C.c_double),
    ]


def build():
    """Compile liboracle_f64.so / liboracle_f32.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_LIBS = {}


def _lib(prec):
    if prec not in _LIBS:
        path = os.path.join(_HERE, f"liboracle_{prec}.so")
        if not os.path.exists(path):
            build()
        _LIBS[prec] = C.CDLL(path)
    return _LIBS[prec]


def _ptr(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    """One precision ('f64' or 'f32') of the CPU restatement on one grid."""

    def __init__(self, shape, prec="f64"):
        self.dim = len(shape)
        n = list(shape) + [1] * (3 - len(shape))
        self.shape = tuple(shape)
        self.g = Grid(self.dim, (C.c_int * 3)(*n))
        self.prec = prec
        self.dtype = np.float64 if prec == "f64" else np.float32
        self.ct = C.c_double if prec == "f64" else C.c_float
        self.lib = _lib(prec)

    # ------------------------------------------------------------------ shapes
    def face_shape(self, c):
        s = list(self.shape)
        s[c] += 1
        return tuple(s)

    def zeros_cell(self, comps=None):
        return np.zeros(((comps,) if comps else ()) + self.shape, self.dtype)

    def zeros_face(self, c, comps=None):
        return np.zeros(((comps,) if comps else ()) + self.face_shape(c), self.dtype)

    def zeros_mac(self):
        return [self.zeros_face(c) for c in range(self.dim)]

    def _mac(self, u):
        u = list(u) + [None] * (3 - len(u))
        return [_ptr(x) for x in u]

    def _r(self, x):
        return self.ct(x)

    # ---------------------------------------------------------------- kernels
    def RK_grid(self, rk, face, psi, T, u, dx, dt):
        """RK2_grid/RK4_grid (face >= 0) or RK*_grid_only_psi (face = -1, T None)."""
        self.lib.fmo_rk_grid(C.byref(self.g), C.c_int(rk), self._r(dx), self._r(dt), C.c_int(face),
                             _ptr(psi), _ptr(T), *self._mac(u))

    def advect_u_grid(self, rk, u0, u1, u2, dx, dt):
        self.lib.fmo_advect_u_grid(C.byref(self.g), C.c_int(rk), self._r(dx), self._r(dt),
                                   *self._mac(u0), *self._mac(u1), *self._mac(u2))

    def advect_scalar_grid(self, rk, u0, s1, s2, dx, dt):
        self.lib.fmo_advect_scalar_grid(C.byref(self.g), C.c_int(rk), self._r(dx), self._r(dt),
                                        *self._mac(u0), _ptr(s1), _ptr(s2))

    def advect_u(self, u0, u1, T, psi, dx):
        """Impulse pullback u1_c = T_c . u0(psi_c) (reference advect_u)."""
        self.lib.fmo_pullback_u(C.byref(self.g), self._r(dx), *self._mac(u0), *self._mac(u1),
                                *self._mac(T), *self._mac(psi))

    def advect_scalar(self, s0, s1, psi, dx):
        self.lib.fmo_pullback_scalar(C.byref(self.g), self._r(dx), _ptr(s0), _ptr(s1), _ptr(psi))

    def accumulate_init(self, f, init, F, phi, dx, dt):
        self.lib.fmo_accumulate_init(C.byref(self.g), self._r(dx), self._r(dt), C.c_int(0), C.c_int(0),
                                     *self._mac(f), *self._mac(init), *self._mac(F), *self._mac(phi),
                                     *([None] * 6))

    def accumulate_init_new(self, f, init, F, phi, Hp, Hpp, ind, dx, dt):
        hs = []
        for c in range(3):
            hs += [_ptr(Hp[c]) if c < self.dim else None, _ptr(Hpp[c]) if c < self.dim else None]
        self.lib.fmo_accumulate_init(C.byref(self.g), self._r(dx), self._r(dt), C.c_int(1), C.c_int(ind),
                                     *self._mac(f), *self._mac(init), *self._mac(F), *self._mac(phi), *hs)

    def calculate_nabla_u_w(self, u, w, r, dx, order=None):
        if order is None:
            order = 3 if self.dim == 3 else 4
        self.lib.fmo_nabla_u_w(C.byref(self.g), C.c_int(order), self._r(dx), *self._mac(u), *self._mac(w),
                               *self._mac(r))

    def calculate_nabla_scalar_adjoint(self, s, adj, r, dx):
        self.lib.fmo_nabla_scalar_adjoint(C.byref(self.g), self._r(dx), _ptr(s), _ptr(adj), *self._mac(r))

    def reset_to_identity(self, psi, psi_f, T_f, dx):
        self.lib.fmo_reset_to_identity(C.byref(self.g), self._r(dx), _ptr(psi), *self._mac(psi_f),
                                       *self._mac(T_f))

    def apply_bc(self, u):
        self.lib.fmo_apply_bc(C.byref(self.g), *self._mac(u))

    def divergence(self, u, div):
        self.lib.fmo_divergence(C.byref(self.g), *self._mac(u), _ptr(div))

    def subtract_grad_p(self, p, u):
        self.lib.fmo_subtract_grad_p(C.byref(self.g), _ptr(p), *self._mac(u))

    def laplacian(self, p, Ap):
        self.lib.fmo_laplacian(C.byref(self.g), _ptr(p), _ptr(Ap))

    def mg_vcycle(self, params, r, z):
        self.lib.fmo_mg_vcycle(C.byref(self.g), C.byref(params), _ptr(r), _ptr(z))

    def mgpcg_solve(self, params, b, x):
        rtr = C.c_double(0)
        conv = C.c_int(0)
        it = self.lib.fmo_mgpcg_solve(C.byref(self.g), C.byref(params), _ptr(b), _ptr(x), C.byref(rtr),
                                      C.byref(conv))
        return it, rtr.value, bool(conv.value)

    def Poisson(self, params, u, p_out=None):
        """In-place projection of the MAC velocity ``u`` (reference solver.Poisson)."""
        rtr = C.c_double(0)
        conv = C.c_int(0)
        it = self.lib.fmo_project(C.byref(self.g), C.byref(params), *self._mac(u), _ptr(p_out), C.byref(rtr),
                                  C.byref(conv))
        return it, rtr.value, bool(conv.value)

    # ------------------------------------------------------------ point query
    def interp_grad(self, order, f, p, dx, BL):
        """interp_grad_{2,3,4}: returns (value, grad[dim]) at one position."""
        shape = list(f.shape) + [1] * (3 - f.ndim)
        s = (C.c_int * 3)(*shape)
        pp = np.zeros(3, self.dtype)
        pp[: len(p)] = p
        bl = np.full(3, 0.5, self.dtype)
        bl[: len(BL)] = BL
        out = np.zeros(4, self.dtype)
        self.lib.fmo_interp_grad(C.c_int(f.ndim), C.c_int(order), _ptr(np.ascontiguousarray(f, self.dtype)), s,
                                 _ptr(pp), self._r(dx), _ptr(bl), _ptr(out))
        return out[0], out[1 : 1 + f.ndim]

    def bspline(self, order, x, deriv=False):
        x = np.ascontiguousarray(x, self.dtype)
        y = np.zeros_like(x)
        self.lib.fmo_bspline(C.c_int(order), C.c_int(int(deriv)), _ptr(x), _ptr(y), C.c_long(x.size))
        return y
