"""The overlapped step (FlowmapConfig.overlap: the flow-map march and the
adjoint's accumulate_init pullbacks on a second stream) launches the same
kernels on the same inputs as the one-stream step, so the gradient must be
bit-identical: eager, interval-checkpointed and replayed from a CUDA graph."""
import importlib
from dataclasses import replace

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _cfg(res, backward_u, recompute=False, overlap=True, dtype=torch.float32):
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    solver = S.SolverConfig(levels=2 if len(res) == 3 else 3, bottom=30, max_iters=60, abs_tol=0.0, rel_tol=1e-12,
                            check_every=0)
    return S.FlowmapConfig(res=res, dx=1.0 / res[0], dt=0.02, total_steps=11, reinit_every=4, RK_number=4,
                           backward_u=backward_u, recompute=recompute, overlap=overlap, dtype=dtype, solver=solver)


def _inputs(res):
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    rng = np.random.default_rng(4)
    dim = len(res)
    u0 = C.split_central_vector(rng.normal(0.0, 0.3, size=(dim,) + res))
    rho0 = C.smooth_ball(res, (0.5,) * dim, 0.25, 1.0 / res[0])
    rho_t = C.smooth_ball(res, (0.45, 0.55, 0.5)[:dim], 0.2, 1.0 / res[0])
    f = lambda x: torch.tensor(x, dtype=torch.float32, device="cuda")
    return [f(x) for x in u0], f(rho0), f(rho_t)


@pytest.mark.parametrize("res", [(16, 16, 16), (32, 24)])
@pytest.mark.parametrize("backward_u,recompute", [(True, False), (False, False), (False, True)])
def test_overlapped_step_is_bit_identical(cuda, res, backward_u, recompute):
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    u0, rho0, rho_t = _inputs(res)
    out = {}
    for ov in (False, True):
        sim = S.LFM_Diff_Simulator(config=_cfg(res, backward_u, recompute, ov))
        loss, grad = sim.gradient(u0, rho0, rho_t)
        out[ov] = (loss, [g.clone() for g in grad], sim)
    assert out[True][0] == out[False][0]
    for a, b in zip(out[True][1], out[False][1]):
        assert torch.equal(a, b)
    # the overlapped gradient recorded as one CUDA graph and replayed
    sim = out[True][2]
    graph = sim.capture_gradient(u0, rho0, rho_t)
    graph.replay()
    torch.cuda.synchronize()
    for a, b in zip(sim.adj_u, out[False][1]):
        assert torch.equal(a, b)
