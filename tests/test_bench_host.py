"""bench.py host logic that needs no GPU: the per-form solver settings and the
other-workload summary, which records a failing workload instead of raising."""
import importlib
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    return importlib.import_module("bench")


def test_form_solver_settings():
    b = _bench()
    assert b.FORM_SOLVER["plain"] == (2, 3e-6)  # the reference's V-cycle
    assert b.FORM_SOLVER["mixed"] == b.FORM_SOLVER["checkpointed"] == (3, 3e-7)


def test_form_config_applies_and_overrides(monkeypatch):
    import torch

    b = _bench()
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = b.parse()
    a.res, a.sim_steps = 16, 4
    cfg = b.form_config(C, a, "checkpointed", torch.float32)
    assert (cfg.solver.pre_post, cfg.solver.rel_tol, cfg.recompute) == (3, 3e-7, True)
    cfg = b.form_config(C, a, "plain", torch.float32)
    assert (cfg.solver.pre_post, cfg.solver.rel_tol, cfg.backward_u) == (2, 3e-6, True)
    a.rel_tol, a.pre_post = 1e-5, 4
    cfg = b.form_config(C, a, "mixed", torch.float32)
    assert (cfg.solver.pre_post, cfg.solver.rel_tol) == (4, 1e-5)


def test_other_workloads_records_a_failure(monkeypatch):
    b = _bench()
    monkeypatch.setattr(b, "OTHER_WORKLOADS", (("no-such-workload", []),))
    out = b.other_workloads()
    assert set(out) == {"no-such-workload"} and "error" in out["no-such-workload"]
