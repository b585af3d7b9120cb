"""fm_project_noalloc: the allocation-free Poisson projection.

It serves callers that cannot allocate device memory themselves (for example
code running inside another runtime's preallocated pool).  The test calls it
through the C ABI twice in a row, on two different velocity fields, and checks
each result against the allocating path (fm_mgpcg_create + fm_project) on the
same input, and that the second call leaves the device's free memory
unchanged.  This file sorts last so that a run stopping at the first failure
has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

TOL = {torch.float32: 2e-5, torch.float64: 1e-10}  # the kernel parity tolerances


def _params(fm, levels):
    return fm._lib.MGParams(levels, 2, 50, 0, 400, 0.0, 1e-8, 1e-12, 4, 0)


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-30))


# (32, 32, 32) FP64 with 2 levels: the 16^3 coarsest level needs 64 KB of shared
# memory, so the allocating path runs its single-CTA bottom kernel with a raised
# limit while the allocation-free path runs per-sweep launches.
# (128, 128, 128) FP32 with 5 levels: the documented capacity of the scratch.
CASES = [
    ((32, 32, 32), 3, torch.float32), ((32, 32, 32), 3, torch.float64),
    ((64, 48), 4, torch.float32), ((64, 48), 4, torch.float64),
    ((32, 32, 32), 2, torch.float64),
    ((128, 128, 128), 5, torch.float32),
]


@pytest.mark.gpu
@pytest.mark.parametrize("shape,levels,dtype", CASES)
def test_noalloc_matches_allocating_projection_twice(fm, cuda, shape, levels, dtype):
    lib = fm._lib.lib()
    g = fm.GridSpec(shape)
    cg = g.c_grid()
    code = fm._lib.dtype_code(dtype)
    P = _params(fm, levels)
    handle = C.c_void_p()
    assert lib.fm_mgpcg_create(C.byref(cg), code, C.byref(P), C.byref(handle)) == 0
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(5)
    try:
        for call in range(2):
            u = [torch.tensor(rng.uniform(-1, 1, size=g.face_shape(c)), dtype=dtype, device=cuda)
                 for c in range(g.dim)]
            a = [x.clone() for x in u]
            b = [x.clone() for x in u]
            pa = [x.data_ptr() for x in a] + [None] * (3 - g.dim)
            pb = [x.data_ptr() for x in b] + [None] * (3 - g.dim)
            it_a, rtr_a = C.c_int(0), C.c_double(0)
            it_b, rtr_b = C.c_int(0), C.c_double(0)
            st_a = lib.fm_project(handle, pa[0], pa[1], pa[2], None, stream, C.byref(it_a), C.byref(rtr_a))
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            st_b = lib.fm_project_noalloc(C.byref(cg), code, C.byref(P), pb[0], pb[1], pb[2], stream,
                                          C.byref(it_b), C.byref(rtr_b))
            torch.cuda.synchronize()
            free_after = torch.cuda.mem_get_info()[0]
            assert st_a == 0 and st_b == 0, (call, st_a, st_b)
            assert it_a.value == it_b.value
            for x, y in zip(b, a):
                assert _rel(x, y) < TOL[dtype], call
            if call == 1:  # the first call on a device may load the library's module
                assert free_after == free_before
    finally:
        lib.fm_mgpcg_destroy(handle)


def test_noalloc_rejects_grids_beyond_its_scratch(fm):
    """256^3 FP32 needs ~350 MB of scratch: refused before the field pointers
    are looked at, so the query passes none and no device work is done."""
    lib = fm._lib.lib()
    cg = fm.GridSpec((256, 256, 256)).c_grid()
    P = _params(fm, 6)
    st = lib.fm_project_noalloc(C.byref(cg), 0, C.byref(P), None, None, None, None, None, None)
    assert st == 8
    assert b"static scratch" in lib.fm_status_string(st)


def test_noalloc_null_fields_on_a_grid_that_fits(fm):
    """A grid within the scratch with NULL fields: an argument error, returned
    before any device work."""
    lib = fm._lib.lib()
    cg = fm.GridSpec((32, 32, 32)).c_grid()
    P = _params(fm, 3)
    assert lib.fm_project_noalloc(C.byref(cg), 0, C.byref(P), None, None, None, None, None, None) == 2
