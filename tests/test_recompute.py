"""Interval checkpointing (FlowmapConfig.recompute): the forward keeps only
(u, passive) at the start of each reinit interval, and the adjoint replays each
interval's forward steps before undoing them.  The replay runs the same kernels
on the same inputs, so the gradient is bit-identical to the full-store run's
when the full store keeps the working dtype; with BF16 midpoint stores the
recompute run is the more accurate one (its midpoint velocities are exact)."""
import importlib

import numpy as np
import pytest
import torch

S = importlib.import_module("differentiable-flowmap_b200.simulator")
Cf = importlib.import_module("differentiable-flowmap_b200.configs")


@pytest.mark.parametrize("bad", [dict(backward_u=True), dict(backward_u=False, add_control_force=True),
                                 dict(backward_u=False, use_short_BFECC=True),
                                 dict(backward_u=False, trajectory_loss=True)])
def test_recompute_rejects_unsupported_options(bad):
    cfg = S.FlowmapConfig(recompute=True, **bad)
    with pytest.raises(S.FlowmapError):
        cfg.validate()


def test_recompute_accepts_the_checkpointed_form():
    S.FlowmapConfig(recompute=True, backward_u=False, store_dtype=torch.bfloat16).validate()
    S.FlowmapConfig(recompute=True, backward_u=False, ckpt_delta=True).validate()


@pytest.mark.parametrize("bad", [dict(recompute=False, backward_u=False),
                                 dict(recompute=True, backward_u=False, dtype=torch.float64)])
def test_checkpoint_differences_need_recompute_and_fp32(bad):
    with pytest.raises(S.FlowmapError):
        S.FlowmapConfig(ckpt_delta=True, **bad).validate()


def _shape_case(res, steps, R, **kw):
    cfg = Cf.shape3d_config(res=res, steps=steps, reinit_every=R, backward_u=False, **kw)
    u0, rho0, rho_t = Cf.shape3d_inputs(res=res)
    dev = torch.device("cuda")
    u0 = [torch.as_tensor(x, dtype=torch.float32, device=dev).contiguous() for x in u0]
    rho0 = torch.as_tensor(rho0, dtype=torch.float32, device=dev).contiguous()
    rho_t = torch.as_tensor(rho_t, dtype=torch.float32, device=dev).contiguous()
    return cfg, u0, rho0, rho_t


@pytest.mark.gpu
@pytest.mark.parametrize("steps,R", [(10, 4), (8, 4), (5, 8)])
def test_recompute_gradient_bit_identical_to_full_store(fm, cuda, steps, R):
    cfg, u0, rho0, rho_t = _shape_case(32, steps, R)
    from dataclasses import replace

    full = S.LFM_Diff_Simulator(config=cfg)
    lf, gf = full.gradient(u0, rho0, rho_t)
    rec = S.LFM_Diff_Simulator(config=replace(cfg, recompute=True))
    lr, gr = rec.gradient(u0, rho0, rho_t)
    assert lf == lr
    assert all(torch.equal(a, b) for a, b in zip(gf, gr))
    assert rec.trajectory_bytes() < full.trajectory_bytes()
    # a second gradient on the same simulator (checkpoints overwritten) agrees too
    lr2, gr2 = rec.gradient(u0, rho0, rho_t)
    assert lr2 == lr and all(torch.equal(a, b) for a, b in zip(gr, gr2))


@pytest.mark.gpu
def test_recompute_with_bf16_store_dtype_is_closer_to_fp64(fm, cuda):
    from dataclasses import replace

    cfg, u0, rho0, rho_t = _shape_case(32, 8, 4, store_dtype=torch.bfloat16)
    _, g16 = S.LFM_Diff_Simulator(config=cfg).gradient(u0, rho0, rho_t)
    _, grc = S.LFM_Diff_Simulator(config=replace(cfg, recompute=True)).gradient(u0, rho0, rho_t)
    c64 = replace(cfg, dtype=torch.float64, store_dtype=None)
    _, g64 = S.LFM_Diff_Simulator(config=c64).gradient([x.double() for x in u0], rho0.double(), rho_t.double())

    def err(g):
        num = sum(float(((a.double() - b) ** 2).sum()) for a, b in zip(g, g64))
        return (num / sum(float((b ** 2).sum()) for b in g64)) ** 0.5

    assert err(grc) <= err(g16)
    assert err(grc) < 1e-4


@pytest.mark.gpu
def test_delta_checkpoints_error_and_memory(fm, cuda):
    """ckpt_delta: velocity checkpoints as BF16 differences.  The gradient stays
    within 1e-4 of the FP64 run, closer than with plain BF16 checkpoints, and the
    checkpoints take less memory than FP32 ones."""
    from dataclasses import replace

    cfg, u0, rho0, rho_t = _shape_case(32, 24, 4)
    base = replace(cfg, recompute=True, backward_u=False)
    runs = {}
    for name, extra in (("f32", {}), ("bf16", dict(ckpt_dtype=torch.bfloat16)), ("delta", dict(ckpt_delta=True))):
        sim = S.LFM_Diff_Simulator(config=replace(base, **extra))
        runs[name] = (sim.gradient(u0, rho0, rho_t)[1], sim.trajectory_bytes())
    c64 = replace(base, dtype=torch.float64, recompute=False)
    _, g64 = S.LFM_Diff_Simulator(config=c64).gradient([x.double() for x in u0], rho0.double(), rho_t.double())

    def err(g):
        num = sum(float(((a.double() - b) ** 2).sum()) for a, b in zip(g, g64))
        return (num / sum(float((b ** 2).sum()) for b in g64)) ** 0.5

    assert err(runs["delta"][0]) < 1e-4
    assert err(runs["delta"][0]) <= err(runs["bf16"][0])
    assert runs["delta"][1] < runs["f32"][1]
    with pytest.raises(fm.FlowmapError):
        S.LFM_Diff_Simulator(config=replace(cfg, ckpt_delta=True))  # needs recompute


@pytest.mark.gpu
def test_recompute_vortex_and_graph_capture(fm, cuda):
    from dataclasses import replace

    vx = importlib.import_module("differentiable-flowmap_b200.vortex")
    cfg = Cf.vortex2d_config(res=64, steps=12, reinit_every=5)
    cfg = replace(cfg, backward_u=False)
    p_full = vx.VortexProblem(S.LFM_Diff_Simulator(config=cfg))
    p_rec = vx.VortexProblem(S.LFM_Diff_Simulator(config=replace(cfg, recompute=True)))
    omt = p_full.final_vorticity(Cf.vortex2d_theta(9))
    th = Cf.vortex2d_theta(3)
    lf, df = p_full.gradient(th, omt)
    lr, dr = p_rec.gradient(th, omt)
    assert lf == lr and np.array_equal(df, dr)
    p_rec.capture(th, omt)
    lg, dg = p_rec.graph_gradient(th)
    assert lg == lf and np.array_equal(dg, df)
