"""Trajectory interop with the reference's RW_Cache .npy format.

CPU: the padded component-last layouts equal literal restatements of the
reference's scalar2vec / vec2mat loops (3D/taichi_utils.py:11-44) and unpack
back exactly; chunk files are named {name}_{first}_{last}.npy, hold
(n_steps, *frame) float32 buffers (a final partial chunk keeps the stale
frames of the previous chunk, as the reference's np.save of its whole buffer
does) and every frame reads back.
GPU: a forward run exported and imported into a fresh adjoint simulator gives
the same gradient, bit for bit, as the in-memory run (FP32 stores and the BF16
stores of the mixed form).
"""
import importlib
import os

import numpy as np
import pytest
import torch

RW = importlib.import_module("differentiable-flowmap_b200.rw_cache")


def _scalar2vec(u):
    """3D/taichi_utils.py:11-20 as loops: u[i,j,k][c] = u_c[i,j,k] over u_c's extent."""
    dim = len(u)
    shape = tuple(u[0].shape[a] + (0 if a == 0 else 1) for a in range(dim))
    out = np.zeros(shape + (dim,), dtype=np.float32)
    for c in range(dim):
        for idx in np.ndindex(*u[c].shape):
            out[idx + (c,)] = u[c][idx]
    return out


def _vec2mat(F):
    """3D/taichi_utils.py:35-44 as loops: F[i,j,k][c,:] = F_c[i,j,k], reshaped to dim*dim."""
    dim = len(F)
    res = [F[0].shape[1 + a] - (1 if a == 0 else 0) for a in range(dim)]
    out = np.zeros(tuple(r + 1 for r in res) + (dim, dim), dtype=np.float32)
    for c in range(dim):
        for idx in np.ndindex(*F[c].shape[1:]):
            out[idx + (c,)] = F[c][(slice(None),) + idx]
    return out.reshape(out.shape[:-2] + (dim * dim,))


@pytest.mark.parametrize("res", [(5, 4, 3), (6, 7)])
def test_layouts_match_reference_loops_and_round_trip(res):
    rng = np.random.default_rng(0)
    dim = len(res)
    u = [rng.normal(size=tuple(res[a] + (a == c) for a in range(dim))).astype(np.float32) for c in range(dim)]
    F = [rng.normal(size=(dim,) + tuple(res[a] + (a == c) for a in range(dim))).astype(np.float32)
         for c in range(dim)]
    pm = RW.pack_mac(u)
    np.testing.assert_array_equal(pm, _scalar2vec(u))
    for a, b in zip(RW.unpack_mac(pm, res), u):
        np.testing.assert_array_equal(a, b)
    pf = RW.pack_face_vectors(F)
    np.testing.assert_array_equal(pf, _vec2mat(F))
    for a, b in zip(RW.unpack_face_vectors(pf, res), F):
        np.testing.assert_array_equal(a, b)
    v = rng.normal(size=(dim,) + tuple(res)).astype(np.float32)
    pv = RW.pack_cell_vector(v)
    assert pv.shape == tuple(res) + (dim,) and pv[(0,) * dim + (1,)] == v[(1,) + (0,) * dim]
    np.testing.assert_array_equal(RW.unpack_cell_vector(pv), v)
    s = rng.normal(size=res).astype(np.float32)
    np.testing.assert_array_equal(RW.unpack_scalar(RW.pack_scalar(s)), s)


def test_chunk_files_names_contents_and_reads(tmp_path):
    d = str(tmp_path)
    cache = RW.RW_Cache(n_steps=100)
    frames = [np.full((3, 2, 1), j, dtype=np.float32) for j in range(250)]
    for j, f in enumerate(frames):
        cache.write_disk_with_cache(f, "u", d, j)
    cache.force_write("u", d)
    assert sorted(os.listdir(d)) == ["u_0_99.npy", "u_100_199.npy", "u_200_249.npy"]
    last = np.load(os.path.join(d, "u_200_249.npy"))
    assert last.shape == (100, 3, 2, 1) and last.dtype == np.float32
    assert last[49, 0, 0, 0] == 249 and last[50, 0, 0, 0] == 150  # stale tail of the previous chunk
    reader = RW.RW_Cache()
    for j in (0, 99, 100, 173, 249, 5):
        np.testing.assert_array_equal(reader.read_disk_with_cache("u", d, j), frames[j])
    with pytest.raises(ValueError):
        reader.read_disk_with_cache("u", d, 250)
    RW.RW_Cache.write_disk(12, "final_ind", d, 0)
    assert RW.RW_Cache.read_disk("final_ind", d, 0).tolist() == [12]


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True])
def test_exported_forward_reproduces_the_gradient(fm, cuda, tmp_path, mixed):
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    res, steps, R = (32, 32), 9, 3
    rng = np.random.default_rng(2)
    u0 = C.split_central_vector(rng.normal(0.0, 0.2, size=(2,) + res))
    rho0 = C.smooth_ball(res, (0.5, 0.5), 0.25, 1 / 32)
    rho_t = C.smooth_ball(res, (0.55, 0.5), 0.2, 1 / 32)
    solver = S.SolverConfig(levels=3, bottom=50, max_iters=200, abs_tol=0.0, rel_tol=1e-12, eps=1e-12)
    cfg = S.FlowmapConfig(res=res, dx=1 / 32, dt=0.01, total_steps=steps, reinit_every=R, RK_number=2,
                          backward_u=not mixed, store_dtype=torch.bfloat16 if mixed else None, solver=solver)
    a = S.LFM_Diff_Simulator(config=cfg)
    a.init(theta=u0, init_passive_np=rho0)
    while not a.forward_step_midpoint()[1]:
        pass
    RW.export_forward(a, str(tmp_path))
    la, ga = a.gradient(u0, rho0, rho_t)
    b = S.LFM_Diff_Simulator(config=cfg)
    assert RW.import_forward(b, str(tmp_path)) == steps
    b.init_gradient(target_passive=rho_t)
    while not b.backtrack_step_midpoint()[1]:
        pass
    assert b.loss == la
    for x, y in zip(b.adj_u, ga):
        assert torch.equal(x, y)
    assert sorted(os.listdir(os.path.join(str(tmp_path), "midpoint"))) == ["u_0_8.npy"]
