"""C ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and rejects invalid arguments before touching the device."""
import ctypes as C

import pytest


def test_library_exports_every_header_symbol(fm):
    lib = fm._lib.lib()
    names = fm._lib.header_symbols()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_status_strings(fm):
    lib = fm._lib.lib()
    assert lib.fm_abi_version() == 1
    assert lib.fm_status_string(3) == b"MGPCG did not converge within max_iters"
    assert lib.fm_status_string(0) == b"ok"


def test_invalid_arguments_rejected_without_device(fm):
    lib = fm._lib.lib()
    bad_dim = fm._lib.Grid(4, (C.c_int * 3)(8, 8, 8))
    assert lib.fm_advect_u_grid(C.byref(bad_dim), 0, 2, 0.1, 0.1, *([None] * 9), None) == 1
    g = fm._lib.Grid(3, (C.c_int * 3)(8, 8, 8))
    assert lib.fm_advect_u_grid(C.byref(g), 5, 2, 0.1, 0.1, *([None] * 9), None) == 7  # dtype
    assert lib.fm_advect_u_grid(C.byref(g), 0, 3, 0.1, 0.1, *([None] * 9), None) == 2  # rk
    g2 = fm._lib.Grid(2, (C.c_int * 3)(8, 8, 4))
    assert lib.fm_rk_grid(C.byref(g2), 0, 2, 0.1, 0.1, 0, None, None, None, None, None, None) == 1  # nz != 1
    tiny = fm._lib.Grid(3, (C.c_int * 3)(3, 8, 8))
    assert lib.fm_nabla_u_w(C.byref(tiny), 0, 3, 0.1, *([None] * 9), None) == 1
    h = C.c_void_p()
    p = fm._lib.MGParams(1, 2, 50, 0, 400, 1e-12, 0.0, 1e-12, 4, 0)  # levels < 2
    assert lib.fm_mgpcg_create(C.byref(g), 0, C.byref(p), C.byref(h)) == 2
    p = fm._lib.MGParams(5, 2, 50, 0, 400, 1e-12, 0.0, 1e-12, 4, 0)  # 8 not divisible by 2^4
    assert lib.fm_mgpcg_create(C.byref(g), 0, C.byref(p), C.byref(h)) == 1
    p = fm._lib.MGParams(2, 2, 50, 0, 400, 1e-12, 0.0, 1e-12, 4, 1)  # BF16 coarse levels need an FP32 solver
    assert lib.fm_mgpcg_create(C.byref(g), 1, C.byref(p), C.byref(h)) == 2
    assert lib.fm_mgpcg_solve_dc(None, 0, None, None, None, 1e-10, 5, None, None, None, None) == 2
    assert lib.fm_project(None, None, None, None, None, None, None, None) == 2
    assert lib.fm_mg_vcycle(None, None, None, None) == 2
    assert lib.fm_clamp_extrema(C.byref(bad_dim), 0, -1, None, None, None, None) == 1
    assert lib.fm_clamp_extrema(C.byref(g), 0, 3, None, None, None, None) == 2  # face >= dim
    assert lib.fm_clamp_extrema(C.byref(g), 0, -1, None, None, None, None) == 2  # NULL fields
    assert lib.fm_fp32_fma_probe(0, 0, 16, None, None) == 2
    assert lib.fm_fp32_fma_probe(1, 4, 0, None, None) == 2
    assert lib.fm_tune_set(0, C.byref(g), 33) == 2


def test_no_cpu_fallback(fm):
    import torch

    g = fm.GridSpec((8, 8, 8))
    u = [torch.zeros(g.face_shape(c)) for c in range(3)]
    with pytest.raises(fm.FlowmapError):
        fm.kernels.advect_u_grid(g, 2, 0.1, 0.1, u, u, u)


def test_launch_counter_exported(fm):
    n0 = fm._lib.launch_count(reset=True)
    assert fm._lib.launch_count() == 0
    assert isinstance(n0, int)


def test_last_cuda_error_reported(fm):
    code, name = fm._lib.last_cuda_error()
    assert isinstance(code, int) and name.startswith("cuda")


def test_project_dc_arguments_rejected(fm):
    """fm_project_dc: a NULL solver, NULL fields or work, rel_tol <= 0: argument
    errors returned before any device work."""
    lib = fm._lib.lib()
    assert lib.fm_project_dc(None, None, None, None, None, 1e-10, 4, None, None) == 2


def test_adjoint_entry_points_reject_arguments_without_device(fm):
    """fm_*_adj: bad grids, dtypes, rk, missing inputs and partial gradient MACs
    are argument errors returned before any device work (only NULL pointers
    are passed)."""
    lib = fm._lib.lib()
    g = fm._lib.Grid(3, (C.c_int * 3)(8, 8, 8))
    bad_dim = fm._lib.Grid(4, (C.c_int * 3)(8, 8, 8))
    n = [None]
    assert lib.fm_advect_scalar_grid_adj(C.byref(bad_dim), 0, 2, 0.1, 0.1, *(n * 9), None) == 1
    assert lib.fm_advect_scalar_grid_adj(C.byref(g), 9, 2, 0.1, 0.1, *(n * 9), None) == 7
    assert lib.fm_advect_scalar_grid_adj(C.byref(g), 0, 3, 0.1, 0.1, *(n * 9), None) == 2
    assert lib.fm_advect_scalar_grid_adj(C.byref(g), 0, 2, 0.1, 0.1, *(n * 9), None) == 2
    assert lib.fm_advect_u_grid_adj(C.byref(g), 1, 4, 0.1, 0.1, *(n * 15), None) == 2
    assert lib.fm_pullback_u_adj(C.byref(g), 0, 0.1, *(n * 9), 1.0, 0.0, *(n * 15), None) == 2
    assert lib.fm_pullback_scalar_adj(C.byref(g), 0, 0.1, None, None, 1.0, 0.0, None, None, None, None, None) == 2
    tiny = fm._lib.Grid(2, (C.c_int * 3)(3, 8, 1))
    assert lib.fm_pullback_scalar_adj(C.byref(tiny), 0, 0.1, None, None, 1.0, 0.0, None, None, None, None,
                                      None) == 1
