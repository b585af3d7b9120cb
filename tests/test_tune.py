"""Launch autotuner: the launch-shape table (fm_tune_set / fm_tune_get) and the
guarantee that tuning changes no result (the gather kernels and the adjoint-
source stencils compute every node independently, each with a fixed summation
order): a vortex gradient is bit for bit the same with every gather kernel
class forced to 64-thread blocks and the stencil tiles to their other height,
and a 3D gradient the same with 4- and 8-node stencil tiles."""
import ctypes as C
import importlib

import numpy as np
import pytest
import torch


def test_tune_table_arguments(fm):
    lib = fm._lib.lib()
    g = fm._lib.Grid(2, (C.c_int * 3)(96, 64, 1))
    assert lib.fm_tune_get(0, C.byref(g)) == 256
    assert lib.fm_tune_set(0, C.byref(g), 48) == 2      # not a multiple of 32
    assert lib.fm_tune_set(0, C.byref(g), 512) == 2     # above the kernels' launch bound
    assert lib.fm_tune_set(9, C.byref(g), 64) == 2      # no such kernel class
    assert lib.fm_tune_set(2, C.byref(g), 128) == 0
    assert lib.fm_tune_get(2, C.byref(g)) == 128
    other = fm._lib.Grid(2, (C.c_int * 3)(64, 96, 1))
    assert lib.fm_tune_get(2, C.byref(other)) == 256    # per shape
    assert lib.fm_tune_set(2, C.byref(g), 0) == 0
    assert lib.fm_tune_get(2, C.byref(g)) == 256


@pytest.mark.gpu
def test_block_sizes_change_no_result(fm, cuda):
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    Cf = importlib.import_module("differentiable-flowmap_b200.configs")
    vx = importlib.import_module("differentiable-flowmap_b200.vortex")
    T = importlib.import_module("differentiable-flowmap_b200.tune")
    res = 64
    cfg = Cf.vortex2d_config(res=res, steps=12, reinit_every=5)
    p = vx.VortexProblem(S.LFM_Diff_Simulator(config=cfg))
    th, omt = Cf.vortex2d_theta(3), p.final_vorticity(Cf.vortex2d_theta(4))
    T.reset((res, res))
    l0, d0 = p.gradient(th, omt)
    for k in T.KINDS:
        T.set_threads(k, (res, res), 8 if k == "adjoint_sources" else 64)
    l1, d1 = p.gradient(th, omt)
    report = T.autotune((res, res), reps=3)
    l2, d2 = p.gradient(th, omt)
    T.reset((res, res))
    assert l0 == l1 == l2
    assert np.array_equal(d0, d1) and np.array_equal(d0, d2)
    assert set(report) == set(T.KINDS)
    assert all(r["threads"] in (T.TILE_CANDIDATES[2] if k == "adjoint_sources" else T.CANDIDATES)
               for k, r in report.items())


def test_tune_python_table_helpers(fm):
    T = importlib.import_module("differentiable-flowmap_b200.tune")
    shape = (80, 48)
    T.reset(shape)
    assert all(T.get_threads(k, shape) == (16 if k == "adjoint_sources" else 256) for k in T.KINDS)
    T.set_threads("march", shape, 96)
    assert T.get_threads("march", shape) == 96 and T.get_threads("advect_u", shape) == 256
    T._cache[(shape, torch.float32, 2, T.CANDIDATES, 1)] = {"march": {"threads": 96, "us": {}}}
    T.reset(shape)
    assert T.get_threads("march", shape) == 256
    assert not any(key[0] == shape for key in T._cache)
    with pytest.raises(KeyError):
        T.set_threads("no_such_kernel", shape, 64)


def test_pdl_switch_round_trips(fm):
    prev = fm._lib.set_pdl(False)
    try:
        assert fm._lib.set_pdl(True) is False
        assert fm._lib.set_pdl(True) is True
    finally:
        fm._lib.set_pdl(prev)


def test_stencil_tile_table_arguments(fm):
    lib = fm._lib.lib()
    g3 = fm._lib.Grid(3, (C.c_int * 3)(32, 32, 32))
    g2 = fm._lib.Grid(2, (C.c_int * 3)(64, 64, 1))
    assert lib.fm_tune_get(6, C.byref(g3)) == 8 and lib.fm_tune_get(6, C.byref(g2)) == 16
    assert lib.fm_tune_set(6, C.byref(g3), 16) == 2     # 3D tiles are 4 or 8 nodes high
    assert lib.fm_tune_set(6, C.byref(g2), 4) == 2      # 2D tiles are 8 or 16
    assert lib.fm_tune_set(6, C.byref(g3), 4) == 0
    assert lib.fm_tune_get(6, C.byref(g3)) == 4
    assert lib.fm_tune_set(6, C.byref(g3), 0) == 0
    assert lib.fm_tune_get(6, C.byref(g3)) == 8


@pytest.mark.gpu
def test_stencil_tiles_change_no_result_3d(fm, cuda):
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    Cf = importlib.import_module("differentiable-flowmap_b200.configs")
    T = importlib.import_module("differentiable-flowmap_b200.tune")
    res = (32, 32, 32)
    cfg = Cf.shape3d_config(res=32, steps=5, reinit_every=4, rk=4, backward_u=False)
    sim = S.LFM_Diff_Simulator(config=cfg)
    u0, r0, rt = Cf.shape3d_inputs(32)
    out = []
    for tile in (8, 4):
        T.set_threads("adjoint_sources", res, tile)
        loss, grad = sim.gradient(u0, r0, rt)
        out.append((loss, [g.clone() for g in grad]))
    T.reset(res)
    assert out[0][0] == out[1][0]
    assert all(torch.equal(a, b) for a, b in zip(out[0][1], out[1][1]))
