"""A whole forward + adjoint gradient recorded as one CUDA graph
(capture_gradient / GradientGraph) replays bit-identically to the eager
gradient: the same kernels in the same order, with every projection's PCG loop
as a device-side conditional WHILE node inside the recorded graph."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _mods():
    return (importlib.import_module("differentiable-flowmap_b200.simulator"),
            importlib.import_module("differentiable-flowmap_b200.configs"),
            importlib.import_module("differentiable-flowmap_b200.vortex"))


def test_vortex_graph_replay_equals_eager(fm, cuda):
    S, Cf, vx = _mods()
    cfg = Cf.vortex2d_config(res=64, steps=12, reinit_every=5)
    p = vx.VortexProblem(S.LFM_Diff_Simulator(config=cfg))
    omt = p.final_vorticity(Cf.vortex2d_theta(9))
    ta, tb = Cf.vortex2d_theta(3), Cf.vortex2d_theta(4)
    la, da = p.gradient(ta, omt)
    lb, db = p.gradient(tb, omt)
    g = p.capture(ta, omt)
    assert g.kernels > 0
    for th, l_ref, d_ref in ((tb, lb, db), (ta, la, da), (tb, lb, db)):
        l, d = p.graph_gradient(th)
        assert l == l_ref and np.array_equal(d, d_ref)
    st = g.stats()
    assert st["nonfinite"] == 0 and st["solves"] > 0
    # eager runs still work after replays, and replays after eager runs
    l, d = p.gradient(ta, omt)
    assert l == la and np.array_equal(d, da)
    l, d = p.graph_gradient(tb)
    assert l == lb and np.array_equal(d, db)


def test_shape3d_graph_replay_equals_eager(fm, cuda):
    S, Cf, _ = _mods()
    res = 32
    cfg = Cf.shape3d_config(res=res, steps=6, reinit_every=3)
    sim = S.LFM_Diff_Simulator(config=cfg)
    u0, rho0, rho_t = Cf.shape3d_inputs(res=res)
    dev = torch.device("cuda")
    u0 = [torch.as_tensor(x, dtype=torch.float32, device=dev).contiguous() for x in u0]
    rho0 = torch.as_tensor(rho0, dtype=torch.float32, device=dev).contiguous()
    rho_t = torch.as_tensor(rho_t, dtype=torch.float32, device=dev).contiguous()
    l0, g0 = sim.gradient(u0, rho0, rho_t)
    g0 = [x.cpu() for x in g0]
    graph = sim.capture_gradient(u0, rho0, rho_t)
    u0[0].mul_(0.5)  # new contents of the captured input
    l1, g1 = sim.gradient(u0, rho0, rho_t)
    g1 = [x.cpu() for x in g1]
    graph.replay()
    assert graph.loss() == l1
    assert all(torch.equal(a.cpu(), b) for a, b in zip(sim.adj_u, g1))
    u0[0].mul_(2.0)
    graph.replay()
    assert graph.loss() == l0
    assert all(torch.equal(a.cpu(), b) for a, b in zip(sim.adj_u, g0))


def test_batched_graphs_equal_eager(fm, cuda):
    B = importlib.import_module("differentiable-flowmap_b200.batch")
    bat = B.BatchedVortex((32, 48, 64, 48), steps=8, reinit_every=4, autotune=False)
    eager = bat.gradients(concurrent=True)
    bat.capture()
    for concurrent in (True, False):
        rep = bat.gradients(concurrent=concurrent, graphs=True)
        for (la, da), (lb, db) in zip(rep, eager):
            assert la == lb and np.array_equal(da, db)


def test_batch_as_one_graph_equals_eager(fm, cuda):
    """capture(single_graph=True): the whole batch's forward + adjoint as one graph
    (a branch per instance); each instance's result equals its eager run bit for
    bit, on two replays with different controls."""
    B = importlib.import_module("differentiable-flowmap_b200.batch")
    bat = B.BatchedVortex((32, 48, 64, 48), steps=8, reinit_every=4, autotune=False)
    eager = bat.gradients(concurrent=False)
    bat.capture(single_graph=True)
    assert bat.batch_graph is not None and bat.batch_kernels > 0
    rep = bat.gradients(graphs=True)
    for (la, da), (lb, db) in zip(rep, eager):
        assert la == lb and np.array_equal(da, db)
    for inst in bat.instances:  # new controls: the graph reads them from its input tensors
        inst.theta = inst.theta * 1.1
    rep2 = bat.gradients(graphs=True)
    bat.batch_graph = None  # back to eager for the reference
    eager2 = bat.gradients(concurrent=False)
    for (la, da), (lb, db) in zip(rep2, eager2):
        assert la == lb and np.array_equal(da, db)
    assert any(la != lb for (la, _), (lb, _) in zip(rep2, rep))


def test_capture_refuses_host_polled_configs(fm, cuda):
    S, Cf, _ = _mods()
    mask = Cf.leaf_mask(32)
    cfg = Cf.vortex2d_config(res=32, steps=4, reinit_every=2, boundary_mask=mask, check_every=4)
    sim = S.LFM_Diff_Simulator(config=cfg)
    u0 = [torch.zeros(sim.grid.face_shape(c), device="cuda") for c in range(2)]
    with pytest.raises(S.FlowmapError):
        sim.capture_gradient(u0, target_vorticity=torch.zeros(sim.grid.shape, device="cuda"))


def test_obstacle_gradient_device_loop_and_graph(fm, cuda):
    """The masked solver's device-side PCG loop (check_every = 0) equals host
    polling bit for bit, and a masked gradient replays from one graph."""
    S, Cf, vx = _mods()
    mask = Cf.leaf_mask(64)
    th, tgt = Cf.vortex2d_theta(3), Cf.vortex2d_theta(9)

    def problem(check_every):
        cfg = Cf.vortex2d_config(res=64, steps=10, reinit_every=5, boundary_mask=mask, check_every=check_every)
        return vx.VortexProblem(S.LFM_Diff_Simulator(config=cfg))

    host, dev = problem(4), problem(0)
    assert not host.sim.solver.device_mode and dev.sim.solver.device_mode
    omt = host.final_vorticity(tgt)
    host.sim.solver.stats(reset=True)  # count the gradient's solves only
    lh, dh = host.gradient(th, omt)
    sh = host.sim.solver_stats
    ld, dd = dev.gradient(th, omt)
    sd = dev.sim.solver_stats
    assert lh == ld and np.array_equal(dh, dd)
    for k in ("solves", "iterations", "not_converged", "nonfinite", "max_iters_seen"):
        assert sh[k] == sd[k], k
    dev.capture(th, omt)
    lg, dg = dev.graph_gradient(th)
    assert lg == lh and np.array_equal(dg, dh)
    st = dev.graph.stats()
    assert st["solves"] == sd["solves"] and st["iterations"] == sd["iterations"]


def test_solvers_of_different_sizes_coexist(fm, cuda):
    """The coarse-level kernels' shared-memory limit is process-wide: a solver
    created after a larger one must not lower it under the larger one's need
    (its first solve, and any solve recorded into a graph, comes later)."""
    M = importlib.import_module("differentiable-flowmap_b200.mgpcg")

    def make(n):
        return M.MGPCG((n, n), torch.float32, levels=5, bottom=20, bottom_mode=1, rel_tol=1e-6, abs_tol=0.0,
                       check_every=0)

    gen = torch.Generator(device="cuda").manual_seed(3)
    for first, second in ((256, 384), (384, 256)):
        a, b = make(first), make(second)
        for s, n in ((a, first), (b, second)):
            u = [torch.randn((n + 1, n) if c == 0 else (n, n + 1), device="cuda", generator=gen) for c in range(2)]
            s.project(u)
            st = s.stats(reset=True)
            assert st["solves"] == 1 and st["nonfinite"] == 0 and st["not_converged"] == 0


def test_programmatic_dependent_launch_changes_no_result(fm, cuda):
    """The solver kernels' programmatic dependent launch (on by default) only
    overlaps launch latency: a gradient is bit-identical with it switched off,
    eager and replayed from a graph."""
    S, Cf, vx = _mods()
    cfg = Cf.vortex2d_config(res=64, steps=10, reinit_every=5)
    p = vx.VortexProblem(S.LFM_Diff_Simulator(config=cfg))
    omt = p.final_vorticity(Cf.vortex2d_theta(9))
    th = Cf.vortex2d_theta(3)
    prev = fm._lib.set_pdl(True)
    try:
        l_on, d_on = p.gradient(th, omt)
        p.capture(th, omt)
        l_g, d_g = p.graph_gradient(th)
        fm._lib.set_pdl(False)
        l_off, d_off = p.gradient(th, omt)
    finally:
        fm._lib.set_pdl(prev)
    assert l_on == l_off == l_g
    assert np.array_equal(d_on, d_off) and np.array_equal(d_on, d_g)
