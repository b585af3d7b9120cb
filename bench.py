#!/usr/bin/env python
"""Benchmark: forward+adjoint gradient evaluations per second, 3D 128^3.

Workload (one bench "step" = one gradient evaluation): 3D smoke shape
transition on a 128^3 MAC grid, 150 leapfrog flow-map steps, reinit every 8,
RK4, dt = 0.0085, passive density; forward simulation + adjoint backtrack,
dL/du0 of L = sum (rho(T) - rho*)^2.  Synthetic seeded inputs
(configs.shape3d_inputs): sphere -> union of two spheres, u0 ~ N(0, 0.01^2).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--form plain|mixed]
  python bench.py --impl reference ...   # the reference algorithm on the host CPU

N > 1 runs N independent replicas (one per GPU, no data-path collective; the
problem does not shard), launched by torchrun; value = N*K / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+adjoint grads/s, 3D 128³: mixed vs plain FP32 on B200 @ rel err ≤1e-4"
UNIT = "grads/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="all", choices=["plain", "mixed", "checkpointed", "both", "all"],
                    help="both: plain + checkpointed; all: plain + mixed + checkpointed (the headline form last)")
    ap.add_argument("--ckpt-dtype", default="bf16-delta", choices=["bf16", "bf16-delta", "f32"],
                    help="storage of the interval checkpoints in the checkpointed form: f32; bf16 (the 128^3 "
                         "gradient error 1.7e-4 vs FP64, over the 1e-4 bar); bf16-delta (velocity checkpoints as BF16 "
                         "differences from the previous one, the first and the passive scalar in FP32: 2.3e-6, "
                         "the default)")
    ap.add_argument("--rel-tol", type=float, default=None,
                    help="relative z.r tolerance of the FP32 projections (rTr < rel_tol * zTr0); default: the "
                         "loosest setting whose gradient is within 1e-4 of an FP64 run solved to its floor "
                         "(3D gradient 3e-6: 1e-6 and 3e-6 measure 1.3e-5, 1e-5 2.5e-4; vortex2d 1e-10, "
                         "shape2d 1e-8)")
    ap.add_argument("--pre-post", type=int, default=None,
                    help="RBGS iterations before and after each coarse correction in the FP32 forms' V-cycle "
                         "(default: the reference's 2)")
    ap.add_argument("--bottom", type=int, default=None,
                    help="bottom-level RBGS iterations of the FP32 forms' V-cycle (default: the reference's 50)")
    ap.add_argument("--no-error", action="store_true", help="skip the FP64 reference runs")
    ap.add_argument("--solver-check-every", type=int, default=0,
                    help="0: device-side PCG loop (CUDA-graph WHILE node); k: host polls every k iterations "
                         "(kernel-level profilers cannot see inside the WHILE node)")
    ap.add_argument("--res", type=int, default=128)
    ap.add_argument("--sim-steps", type=int, default=150)
    ap.add_argument("--reinit", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-other-workloads", action="store_true",
                    help="3D gradient at N=1: skip the short runs of the vortex2d, shape2d and vortex2d-batch "
                         "workloads whose summaries the line carries under other_workloads")
    ap.add_argument("--no-roofline", action="store_true",
                    help="skip the dominant-kernel roofline timing (used for profiler runs, which need W >= 1 only; "
                         "a reported bench value needs W >= 3)")
    ap.add_argument("--mixed-coarse", default="bf16", choices=["bf16", "fp32"],
                    help="storage of the MG coarse levels in the mixed form")
    ap.add_argument("--gaussians", type=int, default=3000, help="Gaussian control forces per step (shape3d-forces)")
    ap.add_argument("--workload", default="gradient",
                    choices=["gradient", "poisson", "vortex2d", "vortex2d-obstacle", "vortex2d-batch",
                             "shape2d", "shape3d-forces", "force-kernels"],
                    help="gradient: the headline 3D gradient benchmark; poisson: the mixed-precision Poisson solve "
                         "(seeded k^-5/3 divergence RHS, all-Neumann, --poisson-res^3); vortex2d: the 2D vortex "
                         "optimisation gradient dL/dtheta (256^2, 100 steps, 4 vortices); shape3d-forces: the 3D "
                         "gradient with 3000 Gaussian control forces per step (128^3, 120 steps, reinit 12)")
    ap.add_argument("--poisson-res", type=int, default=256)
    ap.add_argument("--poisson-inner-tol", type=float, default=1e-8,
                    help="relative z.r tolerance of the FP32 inner solves of the mixed Poisson solve")
    a = ap.parse_args()
    if a.rel_tol is None and a.workload not in ("gradient", "shape3d-forces"):
        a.rel_tol = {"vortex2d": 1e-10, "vortex2d-batch": 1e-10, "vortex2d-obstacle": 1e-8,
                     "shape2d": 1e-8}.get(a.workload, 3e-6)
    return a


# FP32 solver settings of the 3D gradient forms unless --rel-tol / --pre-post say otherwise:
# the plain drop-in keeps the reference's V-cycle (2 pre/post RBGS iterations) at relative
# z.r 3e-6; the mixed and checkpointed forms smooth 3 times before and after each coarse
# correction and solve to 3e-7 (1.2 PCG iterations per projection, a gradient error of 2.0e-6
# against 1.3e-5, and slightly faster).
FORM_SOLVER = {"plain": (2, 3e-6), "mixed": (3, 3e-7), "checkpointed": (3, 3e-7)}


def form_config(C, a, form, dtype):
    """plain: the reference's FP32 drop-in (backward_u=True: the adjoint re-advects
    u backwards and re-projects it); mixed: backward_u=False, the adjoint reads the
    stored trajectory (midpoint velocities in BF16, passive in FP32), BF16 MG coarse
    levels, FP64 reductions; checkpointed: the mixed form keeping only the state at
    each reinit interval's start, the adjoint replaying every interval."""
    import torch

    from dataclasses import replace

    ckpt = form == "checkpointed"
    mixed = form == "mixed" or ckpt
    store = torch.bfloat16 if (mixed and dtype == torch.float32) else None
    pp, rel = FORM_SOLVER[form]
    cfg = C.shape3d_config(res=a.res, steps=a.sim_steps, reinit_every=a.reinit, rk=4, dtype=dtype,
                           store_dtype=store, backward_u=not mixed, check_every=a.solver_check_every,
                           coarse_bf16=mixed and dtype == torch.float32 and a.mixed_coarse == "bf16",
                           rel_tol=rel if a.rel_tol is None else a.rel_tol)
    if dtype == torch.float32:
        sv = cfg.solver
        cfg = replace(cfg, solver=replace(sv, pre_post=pp if a.pre_post is None else a.pre_post,
                                          bottom=sv.bottom if a.bottom is None else a.bottom))
    # checkpointed: the mixed form with interval checkpointing (the adjoint replays each interval)
    if not ckpt:
        return cfg
    f32 = dtype == torch.float32
    cd = torch.bfloat16 if (a.ckpt_dtype == "bf16" and f32) else None
    return replace(cfg, recompute=True, ckpt_dtype=cd, ckpt_delta=a.ckpt_dtype == "bf16-delta" and f32)


def workload_name(a):
    return f"3D smoke shape transition {a.res}^3, {a.sim_steps} steps, reinit {a.reinit}, RK4, fwd+adjoint"


FORM_ORDER = {"plain": ["plain"], "mixed": ["mixed"], "checkpointed": ["checkpointed"],
              "both": ["plain", "checkpointed"], "all": ["plain", "mixed", "checkpointed"]}


def bench_forms(a):
    """The forms the GPU arm times, the headline (value) form last."""
    return FORM_ORDER[a.form]


def headline_form(a):
    return bench_forms(a)[-1]


def bench_config(a, cfg, head):
    """The `config` of the JSON line: the workload and the headline form's
    settings (the same dict on the GPU arm and the reference arm)."""
    return {"workload": workload_name(a), "form": head, "res": a.res, "sim_steps": a.sim_steps,
            "reinit_every": a.reinit, "rk": 4, "dt": cfg.dt, "backward_u": cfg.backward_u,
            "solver_rel_tol_zr": cfg.solver.rel_tol, "solver_levels": cfg.solver.levels,
            "solver_pre_post": cfg.solver.pre_post, "solver_bottom": cfg.solver.bottom,
            "inputs": "seeded: sphere r=0.15 -> union of two spheres (seed 20), u0 ~ N(0, 0.01^2) (seed 21)",
            "l2": "working set and trajectory stores exceed the 126 MB L2; no flush needed"}


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_uuid):
        self.proc = None
        self.lines = []
        self.uuid = dev_uuid

    def start(self):
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
            if self.uuid:
                cmd += ["-i", self.uuid]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                mx = float(p[1])
            except ValueError:
                continue
            for nm, v in zip(names, p[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU: the reference algorithm (oracle restatement, FP32) on the host cores
# ---------------------------------------------------------------------------
def _oracle_sim(cfg, steps, threads):
    """The FP32 oracle simulator (the reference algorithm restated in C, OpenMP)
    with the GPU form's algorithm and solver settings: backward_u, RK order,
    reinit interval and the MGPCG tolerances.  Storage precision (BF16 stores,
    BF16 coarse levels) and interval checkpointing are GPU memory layouts and
    are not modelled."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import MGParams  # noqa: E402  (checker only: CPU legs)
    from sim_oracle import OracleSim  # noqa: E402

    sc = cfg.solver
    mg = MGParams(sc.levels, sc.pre_post, sc.bottom, sc.bottom_mode, sc.max_iters, sc.abs_tol, sc.rel_tol, sc.eps)
    return OracleSim(cfg.res, cfg.dx, cfg.dt, cfg.reinit_every, steps, rk=cfg.RK_number,
                     backward_u=cfg.backward_u, prec="f32", mg=mg)


def cpu_pairs(cfg, steps, threads, inputs):
    """A `steps`-step gradient of the benchmark workload with the FP32 oracle:
    init, `steps` forward leapfrog steps (reinit every R, so whole intervals
    include their reinit work), init_gradient and `steps` adjoint steps (the
    adjoint's reinit BFECC at each interval start).  Returns (seconds for the
    init, seconds for the step pairs, loss, gradient)."""
    import numpy as np

    o = _oracle_sim(cfg, steps, threads)
    u0, rho0, rho_t = inputs
    f32 = lambda x: np.asarray(x, dtype=np.float32)
    t0 = time.perf_counter()
    o.init([f32(x) for x in u0], f32(rho0))
    t1 = time.perf_counter()
    while not o.step_midpoint():
        pass
    o.init_gradient(f32(rho_t))
    while not o.backtrack_step_midpoint():
        pass
    t2 = time.perf_counter()
    return t1 - t0, t2 - t1, o.loss, [x.copy() for x in o.adj_u]


def run_reference(a):
    """The reference arm: the reference algorithm on the host cores (the FP32
    oracle restatement; the reference's Taichi CPU backend cannot be installed
    here), same workload, form and solver settings as the GPU headline.  One
    bench step = one forward + adjoint leapfrog step pair at the benchmark size:
    the W warm-up and K timed steps run as a W-step and a K-step gradient
    (reinit every R, so their whole intervals include the reinit work), and the
    150-step gradient rate is value = 1 / (150 x seconds per pair + init)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import torch

    C = importlib.import_module("differentiable-flowmap_b200.configs")
    head = headline_form(a)
    cfg = form_config(C, a, head, torch.float32)
    threads = len(os.sched_getaffinity(0))
    inputs = C.shape3d_inputs(a.res)
    if a.warmup > 0:
        cpu_pairs(cfg, a.warmup, threads, inputs)
    t_init, t_pairs, _, _ = cpu_pairs(cfg, a.steps, threads, inputs)
    per_pair = t_pairs / a.steps
    per_grad = a.sim_steps * per_pair + t_init
    v = 1.0 / per_grad
    sample = (f"a {a.steps}-step gradient ({a.steps} forward + {a.steps} adjoint leapfrog steps, reinit every "
              f"{a.reinit} with the reinit work of its intervals) at {a.res}^3 in the {head} form's algorithm "
              f"(backward_u={cfg.backward_u}, solver rel_tol {cfg.solver.rel_tol}), after a {a.warmup}-step "
              f"warm-up gradient; {per_pair:.2f} s per step pair, scaled to {a.sim_steps} pairs + the init "
              f"projection ({t_init:.2f} s); FP32 CPU restatement of the reference algorithm in C with OpenMP "
              f"(the Taichi CPU backend is not installable here)")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": per_pair * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(a, cfg, head),
            "step_unit": "one forward + adjoint leapfrog step pair (value scaled to the 150-step gradient)",
            "ms_per_gradient": per_grad * 1e3,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_poisson(a):
    """Mixed-precision Poisson benchmark: FP32 MGPCG inner solves (FP32
    hierarchy), FP64 outer defect correction to |r|/|b| <= 1e-10, next to the
    plain FP32 MGPCG to |r|/|b| <= 1e-6; both pressures compared with an FP64
    MGPCG solve of the same system in the mean-zero gauge."""
    import numpy as np
    import torch

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    fm = importlib.import_module("differentiable-flowmap_b200")
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    n = a.poisson_res
    shape = (n, n, n)
    levels = int(np.log2(n)) - 3 + 1
    b = C.poisson_spectrum_rhs(n, seed=30)
    d_b = torch.tensor(b, device=dev)
    b64 = d_b.double()
    b64 -= b64.mean()
    bnorm2 = float((b64 * b64).sum())

    def gauge(x):
        x = x.double()
        return x - x.mean()

    # FP64 reference solve
    s64 = fm.MGPCG(shape, torch.float64, levels=levels, abs_tol=1e-26 * bnorm2, rel_tol=0.0, eps=0.0, max_iters=400,
                   check_every=4)
    x64 = torch.zeros(shape, dtype=torch.float64, device=dev)
    it64, _ = s64.solve(b64, x64)
    ref = gauge(x64)
    refn = float(ref.norm())
    del s64

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            out = fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / a.steps, out

    # plain FP32 MGPCG, |r| <= 1e-6 |b| (rTr <= 1e-12 |b|^2)
    sp = fm.MGPCG(shape, torch.float32, levels=levels, abs_tol=1e-12 * bnorm2, rel_tol=0.0, max_iters=400,
                  check_every=0)
    xp = torch.zeros(shape, device=dev)
    ms_plain, _ = timed(lambda: sp.solve(d_b, xp))
    it_plain = sp.last_iters
    err_plain = float((gauge(xp) - ref).norm()) / refn
    del sp

    # mixed: FP32 inner solves (BF16 per-level coarse grids; and with FP32 ones),
    # FP64 defect correction to 1e-10
    xm = torch.empty(shape, dtype=torch.float64, device=dev)
    work = torch.empty(shape, dtype=torch.float64, device=dev)
    mixed = {}
    for bf in (False, True):  # the headline (BF16 coarse) last
        sm = fm.MGPCG(shape, torch.float32, levels=levels, abs_tol=0.0, rel_tol=a.poisson_inner_tol, max_iters=100,
                      check_every=0, coarse_bf16=bf)
        ms_m, (xm, outer, inner, rel) = timed(lambda: sm.solve_mixed(d_b, xm, rel_tol=1e-10, work=work))
        mixed[bf] = {"ms": ms_m, "outer_corrections": outer, "inner_pcg_iters": inner, "rel_residual_fp64": rel,
                     "pressure_rel_err_vs_fp64": float((gauge(xm) - ref).norm()) / refn,
                     "coarse_storage": "bf16 (levels between the finest and the cluster-resident ones)" if bf
                     else "fp32"}
        del sm
    ms_mixed = mixed[True]["ms"]
    if rank == 0:
        line = {"metric": f"mixed-precision Poisson solve time, {n}^3 all-Neumann, |r|/|b| <= 1e-10",
                "value": ms_mixed, "unit": "ms", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": ms_mixed, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 (inner) / f64 (outer)", "data": "synthetic",
                "config": {"workload": f"Poisson {n}^3, divergence of a seeded k^-5/3 velocity (seed 30)",
                           "levels": levels, "inner_rel_tol_zr": a.poisson_inner_tol},
                "mixed": mixed[True], "mixed_fp32_coarse": mixed[False],
                "plain_fp32": {"ms": ms_plain, "pcg_iters": it_plain, "target_rel_residual": 1e-6,
                               "pressure_rel_err_vs_fp64": err_plain},
                "fp64_reference": {"pcg_iters": it64, "abs_tol_rTr": 1e-26 * bnorm2}}
        print(json.dumps(line), flush=True)
    return 0


def run_vortex2d(a):
    """2D vortex optimisation gradient: theta (4 vortices: strength, centre;
    seed 0) -> u0 -> 100 steps (256^2, dt = 0.5 dx, reinit 10, RK2, solid-style
    MGPCG) -> L = sum (omega - omega*)^2 (target: seed 1) -> adjoint -> dL/dtheta.
    One bench step = one gradient; error of dL/dtheta vs an FP64 run."""
    import numpy as np
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    vx = importlib.import_module("differentiable-flowmap_b200.vortex")

    obstacle = a.workload == "vortex2d-obstacle"
    # the reference experiment's own leaf obstacle (2D/vortex/data/leaf_mask_256_scaled.npz)
    mask = C.reference_fixtures()["leaf_mask"].astype("float32") if obstacle else None

    def problem(dtype, rel_tol, abs_tol=0.0, max_iters=400):
        cfg = C.vortex2d_config(res=256, steps=100, reinit_every=10, dtype=dtype, rel_tol=rel_tol, abs_tol=abs_tol,
                                max_iters=max_iters, check_every=0, boundary_mask=mask)
        return vx.VortexProblem(S.LFM_Diff_Simulator(config=cfg, device=dev))

    def timed(p, omt):
        for _ in range(a.warmup):
            p.gradient(theta, omt)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            loss, dth = p.gradient(theta, omt)
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / a.steps, loss, dth

    theta = C.vortex2d_theta(0)
    p32 = problem(torch.float32, a.rel_tol)
    omt = p32.final_vorticity(C.vortex2d_theta(1))
    ms_eager, loss_e, dth_e = timed(p32, omt)
    # the headline: the same gradient recorded once as a CUDA graph and replayed (both solvers run their
    # PCG loops on the device, so every projection is inside the graph)
    graphed = True
    if graphed:
        p32.capture(theta, omt)
        for _ in range(a.warmup):
            p32.graph_gradient(theta)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            loss, dth = p32.graph_gradient(theta)
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / a.steps
        if loss != loss_e or not np.array_equal(dth, dth_e):
            raise RuntimeError("graph replay differs from the eager gradient")
    else:
        ms, loss, dth = ms_eager, loss_e, dth_e
    # FP64 reference: solved to its floor (masked solves stall near rTr ~ 1e-15, so a cap of 100 iterations)
    p64 = problem(torch.float64, 1e-20, max_iters=100 if obstacle else 400)
    l64, d64 = p64.gradient(theta, omt.double())
    # the reference solver's own criterion (solid MGPCG: absolute rTr < 1e-14)
    pabs = problem(torch.float32, 0.0, abs_tol=1e-14, max_iters=100)
    ms_abs, l_abs, d_abs = timed(pabs, omt)
    name = "2D vortex dL/dtheta evaluations/s, 256^2, 100 steps, 4 vortices" + (", leaf obstacle" if obstacle else "")
    line = {"metric": name, "value": 1e3 / ms,
            "unit": "grads/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "2D vortex optimisation gradient, 256^2, dt 1/512, reinit 10, RK2, 12 parameters"
                                   + (", the reference's leaf obstacle (solid-aware MGPCG, mask kernels)" if obstacle
                                      else ""),
                       "theta_seed": 0, "target_seed": 1,
                       "obstacle_cells": int(mask.sum()) if obstacle else 0,
                       "launch": "one CUDA graph per gradient (capture_gradient)" if graphed else "eager"},
            "eager": {"grads_per_s": 1e3 / ms_eager, "ms": ms_eager},
            "loss": loss, "dtheta": [float(x) for x in dth],
            "solver": f"relative z.r {a.rel_tol:g}",
            "dtheta_rel_err_vs_fp64": float(np.linalg.norm(dth - d64) / np.linalg.norm(d64)),
            "loss_rel_err_vs_fp64": abs(loss - l64) / abs(l64),
            "reference_abs_criterion": {"solver": "absolute rTr < 1e-14, at most 100 iterations", "ms": ms_abs,
                                        "grads_per_s": 1e3 / ms_abs,
                                        "dtheta_rel_err_vs_fp64": float(np.linalg.norm(d_abs - d64) /
                                                                        np.linalg.norm(d64)),
                                        "loss_rel_err_vs_fp64": abs(l_abs - l64) / abs(l64)}}
    print(json.dumps(line), flush=True)
    return 0


def run_shape2d(a):
    """2D smoke shape transition (256^2 MAC, 200 steps, reinit 12, RK2, dt 0.01,
    MGPCG 5 levels; rho0 = three seeded rectangles, rho* = three seeded discs,
    control u0 ~ N(0, 0.01^2)): one bench step = one gradient dL/du0 of
    L = sum (rho(T) - rho*)^2 in the plain FP32 drop-in form.  value: the gradient
    replayed from one CUDA graph on device-resident inputs; e2e: the
    torch.autograd path (flowmap_loss + backward) with pinned host inputs copied
    in and the gradient and loss copied out every step."""
    import torch
    from dataclasses import replace

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    A = importlib.import_module("differentiable-flowmap_b200.autograd")
    lib = importlib.import_module("differentiable-flowmap_b200._lib")
    f32 = torch.float32
    cfg = C.shape2d_config(res=256, steps=200, reinit_every=12, rk=2, dt=0.01, dtype=f32, rel_tol=a.rel_tol,
                           check_every=0)
    sim = S.LFM_Diff_Simulator(config=cfg, device=dev)
    u0, rho0, rho_t = C.shape2d_inputs(256)
    d_u0 = [torch.tensor(x, dtype=f32, device=dev) for x in u0]
    d_r0 = torch.tensor(rho0, dtype=f32, device=dev)
    d_rt = torch.tensor(rho_t, dtype=f32, device=dev)

    def timed(fn, settle=None):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize(dev)
        if settle:
            settle()
        lib.launch_count(reset=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            out = fn()
        e1.record()
        torch.cuda.synchronize(dev)
        if settle:
            settle()  # the solver's loop bodies of the timed replays enter the launch count here
        return e0.elapsed_time(e1) / a.steps, out, lib.launch_count(reset=True)

    ms_eager, (loss, grad), _ = timed(lambda: sim.gradient(d_u0, d_r0, d_rt))
    grad = [x.clone() for x in grad]
    stats = sim.solver_stats
    graph = sim.capture_gradient(d_u0, d_r0, d_rt)

    def replay():
        graph.replay()
        return sim.adj_u

    ms, gg, launches = timed(replay, settle=graph.stats)
    launches += graph.kernels * a.steps  # kernels recorded outside the PCG loop bodies
    if any(not torch.equal(x, y) for x, y in zip(gg, grad)):
        raise RuntimeError("graph replay differs from the eager gradient")
    # end to end through torch.autograd with host buffers
    h_u0 = [torch.tensor(x, dtype=f32).pin_memory() for x in u0]
    h_r0 = torch.tensor(rho0, dtype=f32).pin_memory()
    h_rt = torch.tensor(rho_t, dtype=f32).pin_memory()
    h_g = [torch.empty(x.shape, dtype=f32).pin_memory() for x in u0]

    def e2e_step():
        u = [x.to(dev, non_blocking=True).requires_grad_(True) for x in h_u0]
        L = A.flowmap_loss(sim, u, h_r0, h_rt)
        L.backward()
        for hg, x in zip(h_g, u):
            hg.copy_(x.grad, non_blocking=True)
        return float(L)

    ms_e2e, _, _ = timed(e2e_step)
    # FP64 run with every projection solved to the FP64 floor
    c64 = C.shape2d_config(res=256, steps=200, reinit_every=12, rk=2, dt=0.01, dtype=torch.float64, rel_tol=1e-22,
                           max_iters=400, check_every=0)
    c64 = replace(c64, solver=replace(c64.solver, eps=0.0))
    s64 = S.LFM_Diff_Simulator(config=c64, device=dev)
    l64, g64 = s64.gradient([x.double() for x in d_u0], d_r0.double(), d_rt.double())
    del s64
    # the same gradient with the tightest FP32 solve that converges (relative z.r 1e-10)
    c10 = C.shape2d_config(res=256, steps=200, reinit_every=12, rk=2, dt=0.01, dtype=f32, rel_tol=1e-10,
                           max_iters=100, check_every=0)
    s10 = S.LFM_Diff_Simulator(config=c10, device=dev)
    ms10, (l10, g10), _ = timed(lambda: s10.gradient(d_u0, d_r0, d_rt))
    st10 = s10.solver_stats
    accurate = {"solver_rel_tol_zr": 1e-10, "ms": ms10, "grads_per_s": 1e3 / ms10,
                "mean_pcg_iters": st10["iterations"] / max(st10["solves"], 1),
                "grad_error_vs_fp64": {"grad_rel_l2": rel_l2(g10, g64), "loss_rel": abs(l10 - l64) / abs(l64)},
                "launch": "eager"}
    del s10
    line = {"metric": "2D shape transition dL/du0 evaluations/s, 256^2, 200 steps", "value": 1e3 / ms,
            "unit": "grads/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "2D smoke shape transition 256^2, 200 steps, reinit 12, RK2, dt 0.01, control u0",
                       "form": "plain FP32 drop-in (backward_u)", "solver_rel_tol_zr": a.rel_tol,
                       "inputs": "3 seeded rectangles (seed 10) -> 3 seeded discs (seed 11), u0 ~ N(0, 0.01^2) "
                                 "(seed 12)", "launch": "one CUDA graph per gradient (capture_gradient)",
                       "l2": "inputs (0.5 MB per field) fit in L2; the trajectory store (210 MB) does not"},
            "gpu_launches": launches, "eager": {"grads_per_s": 1e3 / ms_eager, "ms": ms_eager},
            "e2e": {"value": 1e3 / ms_e2e, "unit": "grads/s", "path": "autograd flowmap_loss + backward",
                    "h2d_bytes_per_step": sum(x.numel() * 4 for x in h_u0) + 2 * h_r0.numel() * 4,
                    "d2h_bytes_per_step": sum(x.numel() * 4 for x in h_g) + 8},
            "solver": {"mean_pcg_iters": stats["iterations"] / max(stats["solves"], 1),
                       "solves_per_grad": stats["solves"] // max(a.warmup + a.steps, 1)},
            "loss": loss, "grad_error_vs_fp64": {"grad_rel_l2": rel_l2(grad, g64), "loss_rel": abs(loss - l64) / abs(l64),
                                                 "fp64_reference": "projections to relative z.r 1e-22"},
            "accurate_solve": accurate,
            "note": ("the rectangles' discontinuous density makes the adjoint sources amplify FP32 rounding: the "
                     "gradient error vs FP64 stays near 3e-4 even with FP64 defect-corrected projections"),
            "trajectory_gb": sim.trajectory_bytes() / 1e9}
    print(json.dumps(line), flush=True)
    return 0


def run_vortex2d_batch(a):
    """16 vortex-optimisation instances (4 x 128^2, 4 x 192^2, 4 x 256^2,
    4 x 384^2; 100 steps, reinit 10, dt = 0.5 dx; control seeds 100+i, target
    seeds 200+i) advanced concurrently, one stream and host thread each; one
    bench step = one gradient of every instance.  Compared with the same
    instances run one after another.  Under torchrun the instances are split
    across the ranks by cost (greedy bin-packing on cells x steps, no collective
    in the timed loop); the time is the max over ranks."""
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    B = importlib.import_module("differentiable-flowmap_b200.batch")
    sizes, steps = B.DEFAULT_SIZES, 100
    mine = B.rank_share(sizes, steps, rank, world)
    bat = B.BatchedVortex(sizes=sizes, steps=steps, device=dev, indices=mine, rel_tol=a.rel_tol)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(concurrent, graphs=False):
        for _ in range(a.warmup):
            bat.gradients(concurrent, graphs)
        torch.cuda.synchronize(dev)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            res = bat.gradients(concurrent, graphs)
        e1.record()
        torch.cuda.synchronize(dev)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / a.steps), res

    ms_seq, seq = timed(False)
    ms_conc, conc = timed(True)
    # the same batch with every block size at the default 256, for comparison
    T = importlib.import_module("differentiable-flowmap_b200.tune")
    tuned = {n: {k: v["threads"] for k, v in t.items()} for n, t in bat.tuning.items()}
    for n in bat.tuning:
        T.reset((n, n))
    ms_default, _ = timed(True)
    for n, t in tuned.items():
        for k, th in t.items():
            T.set_threads(k, (n, n), th)
    # every instance's gradient recorded as one CUDA graph, replayed on its stream; first with every block
    # size at the default 256, then (the headline) with the tuned sizes
    for n in bat.tuning:
        T.reset((n, n))
    bat.capture()
    ms_graph_default, _ = timed(True, graphs=True)
    for n, t in tuned.items():
        for k, th in t.items():
            T.set_threads(k, (n, n), th)
    bat.capture()
    ms_graph, graph = timed(True, graphs=True)
    # the whole batch as ONE graph (a branch per instance): one launch per batch gradient
    bat.capture(single_graph=True)
    ms_one, one = timed(True, graphs=True)
    errs_one = B.gather_results({i: float(np.linalg.norm(dc - ds) / np.linalg.norm(ds))
                                 for i, (_, dc), (_, ds) in zip(mine, one, seq)})
    errs = {i: float(np.linalg.norm(dc - ds) / np.linalg.norm(ds)) for i, (_, dc), (_, ds) in zip(mine, graph, seq)}
    errs_eager = {i: float(np.linalg.norm(dc - ds) / np.linalg.norm(ds)) for i, (_, dc), (_, ds) in zip(mine, conc, seq)}
    errs_eager = B.gather_results(errs_eager)
    errs = B.gather_results(errs)
    n = len(sizes)
    if rank == 0:
        line = {"metric": "batched 2D vortex gradients/s, 16 instances (4 x 128^2, 192^2, 256^2, 384^2), 100 steps",
                "value": n * 1e3 / ms_one, "unit": "grads/s", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_one, "higher_is_better": True,
                "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": ("16 concurrent vortex instances, the batch's forward + adjoint one CUDA "
                                        "graph (a branch per instance), one graph launch per batch gradient"),
                           "sizes": list(sizes),
                           "parallelism": (f"instances split over {world} ranks by cost, no collective in the "
                                           "timed loop; time = max over ranks") if world > 1 else "single GPU",
                           "rank_shares": [B.rank_share(sizes, steps, r, world) for r in range(world)]},
                "sequential": {"grads_per_s": n * 1e3 / ms_seq, "ms_per_batch": ms_seq},
                "eager_concurrent": {"grads_per_s": n * 1e3 / ms_conc, "ms_per_batch": ms_conc,
                                     "note": "kernel launches issued from one host thread per instance",
                                     "dtheta_rel_err_vs_unbatched": [errs_eager[i] for i in range(n)]},
                "autotuned_block_sizes": {str(k): v for k, v in tuned.items()},
                "untuned_256_threads": {"grads_per_s": n * 1e3 / ms_default, "ms_per_batch": ms_default,
                                        "note": "eager concurrent"},
                "graphs_untuned_256_threads": {"grads_per_s": n * 1e3 / ms_graph_default,
                                               "ms_per_batch": ms_graph_default},
                "graph_per_instance": {"grads_per_s": n * 1e3 / ms_graph, "ms_per_batch": ms_graph,
                                       "note": "one graph per instance, replayed on its own stream",
                                       "dtheta_rel_err_vs_unbatched": [errs[i] for i in range(n)]},
                "graph_launches_per_batch": 1,
                "solver_rel_tol_zr": a.rel_tol,
                "graph_over_sequential": ms_seq / ms_one,
                "per_instance_dtheta_rel_err_vs_unbatched": [errs_one[i] for i in range(n)]}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _case11_gaussians(res, ng, steps, seed=40):
    """Seeded synthetic Gaussian parameters per step, drawn as the reference's
    3D optimiser draws radii and centres (3D/optimize_shape_G_R.py:21-53);
    strengths |s| in [0.01, 0.04] in a uniform direction."""
    import numpy as np

    dx = 1.0 / res
    rng = np.random.default_rng(seed)
    ks = np.array([1, 1, 1, 1, 2, 3, 4, 5, 6, 7, 8, 9], dtype=np.float64)
    out = []
    for _ in range(steps):
        inv_r = 1.0 / (rng.choice(ks, size=ng) * dx) ** 2
        cen = rng.uniform(0.0, 1.0, size=(ng, 3))
        v = rng.normal(size=(ng, 3))
        st = rng.uniform(5e-3, 2e-2, size=(ng, 1)) * 2.0 * v / np.linalg.norm(v, axis=1, keepdims=True)
        out.append({"c": cen.astype(np.float32), "r": inv_r.astype(np.float32), "s": st.astype(np.float32),
                    "n": ng})
    return out


def _pairs_in_support(p, res):
    """Exact count of (face, Gaussian) pairs with |X - c|^2 r < 5 (float64)."""
    import numpy as np

    dx = 1.0 / res
    pairs = 0
    for k in range(3):
        ax = [(np.arange(res + (1 if a == k else 0)) + (0.0 if a == k else 0.5)) * dx for a in range(3)]
        for I in range(p["n"]):
            rad = np.sqrt(5.0 / p["r"][I])
            sel = [np.abs(ax[a] - p["c"][I, a]) < rad for a in range(3)]
            x, y, z = (ax[a][sel[a]] - p["c"][I, a] for a in range(3))
            d2 = x[:, None, None] ** 2 + y[None, :, None] ** 2 + z[None, None, :] ** 2
            pairs += int(np.count_nonzero(d2 * p["r"][I] < 5.0))
    return pairs


def run_shape3d_forces(a):
    """3D shape transition with Gaussian control forces, the reference's case-11
    hyperparameters (3D/hyperparameters.py:268-293): 128^3, 120 steps, reinit 12,
    RK4, dt 0.0085, backward_u, 3000 Gaussians per step (seeded synthetic
    parameters, force_oracle-style draws made here with numpy).  One bench step =
    one gradient (forward with forces + adjoint with the per-step parameter sums).
    value: parameters resident on the device; e2e: numpy parameters staged per
    step as the reference's from_numpy, plus u0 / rho in and dL/du0 out."""
    import numpy as np
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    K = importlib.import_module("differentiable-flowmap_b200.kernels")
    from dataclasses import replace

    res, steps, reinit, ng = a.res, 120, 12, a.gaussians
    dx = 1.0 / res

    def config(dtype, forces=True):
        cfg = C.shape3d_config(res=res, steps=steps, reinit_every=reinit, rk=4, dtype=dtype,
                               rel_tol=(3e-6 if a.rel_tol is None else a.rel_tol) if dtype == torch.float32 else 1e-20)
        return replace(cfg, add_control_force=forces, control_num=ng)

    host = _case11_gaussians(res, ng, steps)
    devp = [{k: (torch.tensor(v, device=dev) if k != "n" else v) for k, v in p.items()} for p in host]
    u0, rho0, rho_t = C.shape3d_inputs(res)
    f32 = torch.float32
    d_u0 = [torch.tensor(x, dtype=f32, device=dev) for x in u0]
    d_r0, d_rt = torch.tensor(rho0, dtype=f32, device=dev), torch.tensor(rho_t, dtype=f32, device=dev)
    h_u0 = [torch.tensor(x, dtype=f32).pin_memory() for x in u0]
    h_r0, h_rt = torch.tensor(rho0, dtype=f32).pin_memory(), torch.tensor(rho_t, dtype=f32).pin_memory()
    h_grad = [torch.empty(x.shape, dtype=f32).pin_memory() for x in u0]

    sim = S.LFM_Diff_Simulator(config=config(f32), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(a.steps):
            out = fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / a.steps, out

    fm = importlib.import_module("differentiable-flowmap_b200")
    fm._lib.launch_count(reset=True)
    ms, (loss, grad) = timed(lambda: sim.gradient(d_u0, d_r0, d_rt, control_forces=devp))
    launches = fm._lib.launch_count(reset=True) // max(a.steps + a.warmup, 1) * a.steps

    def e2e_step():
        l, g = sim.gradient(h_u0, h_r0, h_rt, control_forces=host)
        for hg, x in zip(h_grad, g):
            hg.copy_(x, non_blocking=True)
        return float(l), g

    ms_e2e, _ = timed(e2e_step)
    nof = S.LFM_Diff_Simulator(config=config(f32, forces=False), device=dev)
    ms_nof, _ = timed(lambda: nof.gradient(d_u0, d_r0, d_rt))
    del nof

    # the two force kernels on step 0's parameters and the live adjoint velocity
    g = sim.grid
    p0 = devp[0]
    reps = 20
    e0.record()
    for _ in range(reps):
        K.gaussian_force(g, dx, p0["c"], p0["r"], p0["s"], sim.control_force)
    e1.record()
    torch.cuda.synchronize(dev)
    us_force = e0.elapsed_time(e1) * 1e3 / reps
    e0.record()
    for _ in range(reps):
        K.gaussian_force_grad(g, dx, p0["c"], p0["r"], p0["s"], sim.adj_u)
    e1.record()
    torch.cuda.synchronize(dev)
    us_grad = e0.elapsed_time(e1) * 1e3 / reps

    err = None
    if not a.no_error:
        s64 = S.LFM_Diff_Simulator(config=config(torch.float64), device=dev)
        dp64 = [{k: (v.double() if k != "n" else v) for k, v in p.items()} for p in devp]
        l64, g64 = s64.gradient([x.double() for x in d_u0], d_r0.double(), d_rt.double(), control_forces=dp64)
        num = sum(float(((x.double() - y) ** 2).sum()) for x, y in zip(grad, g64))
        den = sum(float((y ** 2).sum()) for y in g64)
        pnum = pden = 0.0
        for n in range(steps):
            for k in (0, 1):
                x, y = sim.control_force_grads[n][k], s64.control_force_grads[n][k]
                pnum += float(((x - y) ** 2).sum())
                pden += float((y ** 2).sum())
        err = {"grad_u0_rel_l2": (num / den) ** 0.5, "loss_rel": abs(float(loss) - l64) / abs(l64),
               "param_grads_rel_l2": (pnum / pden) ** 0.5 if pden > 0 else None}
        del s64

    stored = getattr(sim, "store_force", None) is not None
    nforce = steps if stored else 2 * steps
    h2d = sum(x.numel() * 4 for x in h_u0) + h_r0.numel() * 4 + h_rt.numel() * 4 + steps * ng * 7 * 4 * 2
    d2h = sum(x.numel() * 4 for x in h_grad) + 8
    line = {"metric": "3D fwd+adjoint grads/s with Gaussian control forces, 128^3, 120 steps, 3000 Gaussians/step",
            "value": 1e3 / ms, "unit": "grads/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"3D shape transition with control forces {res}^3, {steps} steps, reinit {reinit}, "
                                   f"RK4, {ng} Gaussians per step (case-11 hyperparameters)",
                       "form": "plain (backward_u)", "parameters": "seeded synthetic, strengths |s| in [0.01, 0.04]",
                       "l2": "working set and trajectory stores exceed the 126 MB L2; no flush needed"},
            "e2e": {"value": 1e3 / ms_e2e, "unit": "grads/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "without_forces": {"grads_per_s": 1e3 / ms_nof, "ms_per_grad": ms_nof},
            "force_kernels": {"k_gauss_force_us": us_force, "k_gauss_grad_us": us_grad,
                              "launches_per_grad": {"k_gauss_force": nforce, "k_gauss_grad": steps},
                              "ms_per_grad": (nforce * us_force + steps * us_grad) / 1e3,
                              "adjoint_force": "read from the forward's store" if stored else "re-evaluated"},
            "error_vs_fp64": err}
    print(json.dumps(line), flush=True)
    return 0


def run_force_kernels(a):
    """The two Gaussian-force kernels alone at --res^3 with --gaussians Gaussians
    (case-11 draws), FP32: fm_gaussian_force (every face) and
    fm_gaussian_force_grad (per-Gaussian sums against a seeded adjoint field).
    Unit of work: a (face, Gaussian) pair inside the support, counted exactly."""
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    K = importlib.import_module("differentiable-flowmap_b200.kernels")
    fm = importlib.import_module("differentiable-flowmap_b200")
    res, ng = a.res, a.gaussians
    dx = 1.0 / res
    p = _case11_gaussians(res, ng, 1)[0]
    c, r, st = (torch.tensor(p[k], device=dev) for k in ("c", "r", "s"))
    g = K.GridSpec((res, res, res))
    f = [torch.empty(g.face_shape(k), dtype=torch.float32, device=dev) for k in range(3)]
    gen = torch.Generator(device=dev).manual_seed(7)
    adj = [torch.randn(g.face_shape(k), dtype=torch.float32, device=dev, generator=gen) for k in range(3)]
    pairs = _pairs_in_support(p, res)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0.record()
        for _ in range(a.steps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) * 1e3 / a.steps

    fm._lib.launch_count(reset=True)
    us_f = timed(lambda: K.gaussian_force(g, dx, c, r, st, f))
    us_g = timed(lambda: K.gaussian_force_grad(g, dx, c, r, st, adj))
    launches = fm._lib.launch_count(reset=True)
    line = {"metric": "Gaussian control-force kernel, (face, Gaussian) pairs/s", "value": pairs / (us_f * 1e-6),
            "unit": "pairs/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": us_f / 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"fm_gaussian_force / fm_gaussian_force_grad at {res}^3, {ng} Gaussians "
                                   "(case-11 radius and centre draws, seed 40)",
                       "pairs_in_support": pairs,
                       "l2": "inputs (25 MB per field) fit in L2; the kernels are compute-bound"},
            "gpu_launches": launches,
            "k_gauss_force_us": us_f, "k_gauss_grad_us": us_g, "grad_pairs_per_s": pairs / (us_g * 1e-6)}
    print(json.dumps(line), flush=True)
    return 0


OTHER_WORKLOADS = (("vortex2d", ["--steps", "3", "--warmup", "3"]),
                   ("shape2d", ["--steps", "3", "--warmup", "3"]),
                   ("vortex2d-batch", ["--steps", "2", "--warmup", "2"]))
OTHER_KEYS = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "solver", "solver_rel_tol_zr",
              "dtheta_rel_err_vs_fp64", "grad_error_vs_fp64", "e2e", "graph_launches_per_batch",
              "per_instance_dtheta_rel_err_vs_unbatched", "clocks")


def other_workloads():
    """The other benchmark configurations, each run once as its own process on this
    GPU (`bench.py --workload W`), summarised so that one default run records them
    all: 2D vortex 256^2 (config 0), 2D shape transition 256^2 (config 1) and the
    16-instance batch (config 4)."""
    import subprocess

    out = {}
    for name, extra in OTHER_WORKLOADS:
        cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--workload", name, *extra]
        try:
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
            lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
            if p.returncode != 0 or not lines:
                out[name] = {"error": f"exit {p.returncode}: {p.stderr.strip().splitlines()[-1:]}"}
                continue
            d = json.loads(lines[-1])
            out[name] = {k: d[k] for k in OTHER_KEYS if k in d}
            out[name]["command"] = "python bench.py --workload " + name + " " + " ".join(extra)
        except Exception as e:  # recorded, never fatal to the headline line
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.workload == "poisson":
        return run_poisson(a)
    if a.workload in ("vortex2d", "vortex2d-obstacle"):
        return run_vortex2d(a)
    if a.workload == "vortex2d-batch":
        return run_vortex2d_batch(a)
    if a.workload == "shape2d":
        return run_shape2d(a)
    if a.workload == "shape3d-forces":
        return run_shape3d_forces(a)
    if a.workload == "force-kernels":
        return run_force_kernels(a)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)

    from dataclasses import replace

    fm = importlib.import_module("differentiable-flowmap_b200")
    C = importlib.import_module("differentiable-flowmap_b200.configs")
    S = importlib.import_module("differentiable-flowmap_b200.simulator")
    lib = fm._lib

    forms = bench_forms(a)
    head = headline_form(a)
    # launch shapes (gather-kernel block sizes, adjoint-source tile height) picked by the
    # project's autotuner on this grid shape; they change no result
    T = importlib.import_module("differentiable-flowmap_b200.tune")
    tuned = {k: v["threads"] for k, v in T.autotune((a.res,) * 3, rk=4, reps=5, device=dev).items()}
    sims, cfgs = {}, {}
    for f in forms:
        cfgs[f] = form_config(C, a, f, torch.float32)
        sims[f] = S.LFM_Diff_Simulator(config=cfgs[f], device=dev)
    sims_bytes = {f: x.trajectory_bytes() for f, x in sims.items()}
    sim, cfg = sims[head], cfgs[head]
    store = cfg.store_dtype
    backward_u = cfg.backward_u
    u0, rho0, rho_t = C.shape3d_inputs(a.res)
    f32 = torch.float32
    d_u0 = [torch.tensor(x, dtype=f32, device=dev) for x in u0]
    d_r0 = torch.tensor(rho0, dtype=f32, device=dev)
    d_rt = torch.tensor(rho_t, dtype=f32, device=dev)
    h_u0 = [torch.tensor(x, dtype=f32).pin_memory() for x in u0]
    h_r0 = torch.tensor(rho0, dtype=f32).pin_memory()
    h_rt = torch.tensor(rho_t, dtype=f32).pin_memory()
    h_grad = [torch.empty(x.shape, dtype=f32).pin_memory() for x in u0]
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    results = {}
    for f in forms:  # the headline form last
        s_ = sims[f]
        for _ in range(a.warmup):
            s_.gradient(d_u0, d_r0, d_rt)
        torch.cuda.synchronize(dev)
        barrier()
        if f == forms[0]:
            clocks.start()
        iters = []
        lib.launch_count(reset=True)
        torch.cuda.synchronize(dev)
        barrier()
        ev0.record(stream)
        for _ in range(a.steps):
            loss, grad = s_.gradient(d_u0, d_r0, d_rt)
            iters.append(dict(s_.solver_stats or {}))
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        launches = lib.launch_count(reset=True)
        t = torch.tensor([ev0.elapsed_time(ev1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
        results[f] = {"value": world * a.steps / (ms_max / 1e3), "ms_per_step": ms_max / a.steps,
                      "launches": launches, "iters": iters, "loss": float(loss), "grad": grad}
    clk = clocks.stop()
    value = results[head]["value"]
    ms_max = results[head]["ms_per_step"] * a.steps
    launches = results[head]["launches"]
    iters = results[head]["iters"]

    # end-to-end through the public API with host buffers
    e2e = None
    if not a.no_e2e:
        h2d = sum(x.numel() * 4 for x in h_u0) + h_r0.numel() * 4 + h_rt.numel() * 4
        d2h = sum(x.numel() * 4 for x in h_grad) + 8
        torch.cuda.synchronize(dev)
        barrier()
        ev0.record(stream)
        for _ in range(a.steps):
            loss, grad = sim.gradient(h_u0, h_r0, h_rt)
            for hg, g in zip(h_grad, grad):
                hg.copy_(g, non_blocking=True)
            _ = float(loss)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        te = torch.tensor([ev0.elapsed_time(ev1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e = {"value": world * a.steps / (float(te.item()) / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h}

    # roofline of the dominant kernel, timed live on the launching stream
    roof = None
    if rank == 0 and not a.no_roofline:
        roof = dominant_kernel_roofline(fm, sim, dev, stream)

    # gradient error of each form against an FP64 run of the same algorithm with every
    # projection solved to the FP64 floor (relative z.r 1e-22, no eps): solver truncation
    # shows up in the error instead of cancelling against an equally loose FP64 run
    errors, g64s = {}, {}
    if rank == 0 and not a.no_error:
        for f in forms:
            c64 = form_config(C, a, f, torch.float64)
            c64 = replace(c64, recompute=False, solver=replace(c64.solver, rel_tol=1e-22, abs_tol=0.0, eps=0.0,
                                                                max_iters=400))
            key = c64.backward_u
            if key not in g64s:
                s64 = S.LFM_Diff_Simulator(config=c64, device=dev)
                g64s[key] = s64.gradient([x.double() for x in d_u0], d_r0.double(), d_rt.double())
                st64 = s64.solver_stats
                del s64
                torch.cuda.empty_cache()
            l64, g64 = g64s[key]
            g32 = results[f]["grad"]
            errors[f] = {"grad_rel_l2": rel_l2(g32, g64), "loss_rel": abs(results[f]["loss"] - l64) / abs(l64),
                         "fp64_reference": "same algorithm, projections to relative z.r 1e-22"}
        if True in g64s and False in g64s:
            # the mixed forms' algorithm (backward_u off) against the plain algorithm, both FP64
            errors["algorithm_gap_fp64"] = rel_l2(g64s[False][1], g64s[True][1])
        del g64s

    def solver_stats(f):
        its = results[f]["iters"]
        solves = sum(r.get("solves", 0) for r in its)
        return {"levels": sims[f].solver.n_mg_levels, "rel_tol_zr": cfgs[f].solver.rel_tol,
                "pre_post": cfgs[f].solver.pre_post, "bottom": cfgs[f].solver.bottom,
                "mean_pcg_iters": sum(r.get("iterations", 0) for r in its) / solves if solves else None,
                "solves_per_grad": solves // max(a.steps, 1),
                "not_converged": sum(r.get("not_converged", 0) for r in its),
                "mode": "device (graph WHILE loop)" if a.solver_check_every == 0
                else f"host-checked every {a.solver_check_every} iterations"}

    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": bench_config(a, cfg, head),
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "e2e": e2e, "gpu_launches": launches, "clocks": clk, "roofline": roof,
                "forms": {f: {"value": r["value"], "ms_per_step": r["ms_per_step"], "gpu_launches": r["launches"],
                              "backward_u": cfgs[f].backward_u,
                              "velocity_store": ("interval checkpoints + a replayed f32 ring of one interval"
                                                 if cfgs[f].recompute else
                                                 "bf16" if cfgs[f].store_dtype == torch.bfloat16 else "f32"),
                              "checkpoint_dtype": (("bf16 differences of u (first checkpoint and passive in f32)"
                                                    if cfgs[f].ckpt_delta else
                                                    str(cfgs[f].ckpt_dtype or cfgs[f].dtype).replace("torch.", ""))
                                                   if cfgs[f].recompute else None),
                              "mg_coarse_storage": "bf16" if cfgs[f].solver.coarse_bf16 else "f32",
                              "trajectory_gb": sims_bytes[f] / 1e9, "solver": solver_stats(f),
                              "grad_error_vs_fp64": errors.get(f)} for f, r in results.items()},
                "algorithm_gap_fp64": errors.get("algorithm_gap_fp64"),
                "launch_shapes": {"autotuned": tuned,
                                  "note": "threads per block of the gather kernels, tile height of the adjoint-source "
                                          "stencil (tune.autotune on this grid)"}}
        for f in ("mixed", "checkpointed"):
            if "plain" in results and f in results:
                line[f"{f}_over_plain"] = results[f]["value"] / results["plain"]["value"]
        if world == 1 and not a.no_cpu_baseline:
            line["cpu_baseline"], line["parity_one_step"] = cpu_leg(a, C, S, cfg, head, dev)
        if world == 1 and not a.no_other_workloads and a.res == 128 and a.sim_steps == 150:
            line["other_workloads"] = other_workloads()
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def rel_l2(a, b):
    num = sum(float(((x.double() - y.double()) ** 2).sum()) for x, y in zip(a, b))
    den = sum(float((y.double() ** 2).sum()) for y in b)
    return (num / den) ** 0.5


def cpu_leg(a, C, S, cfg, head, dev):
    """cpu_baseline: a one-step gradient (1 forward + 1 adjoint step, the
    adjoint's reinit BFECC included) of the headline form's algorithm at the
    benchmark size with the FP32 oracle on all host threads, scaled x150 (a
    bounded sample: the reference arm times a longer one).  The same one-step
    gradient is run on the GPU and compared with it (relative L2 of dL/du0):
    implementation parity at the benchmark grid size."""
    import numpy as np
    import torch
    from dataclasses import replace

    threads = len(os.sched_getaffinity(0))
    inputs = C.shape3d_inputs(a.res)
    t_init, t_pairs, lo, go = cpu_pairs(cfg, 1, threads, inputs)
    secs = t_init + t_pairs
    one = replace(cfg, total_steps=1, recompute=False, ckpt_delta=False, store_dtype=None)
    sim1 = S.LFM_Diff_Simulator(config=one, device=dev)
    u0, rho0, rho_t = inputs
    lg, gg = sim1.gradient(u0, rho0, rho_t)
    gg = [x.double().cpu().numpy() for x in gg]
    err = float(np.sqrt(sum(((x - y) ** 2).sum() for x, y in zip(gg, go)) / sum((y.astype(np.float64) ** 2).sum()
                                                                               for y in go)))
    base = {"value": 1.0 / (secs * a.sim_steps), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"one-step gradient (1 forward + 1 adjoint step incl. the adjoint reinit) of the {head} "
                       f"form's algorithm at {a.res}^3 with the FP32 CPU restatement, {secs:.1f} s, scaled "
                       f"x{a.sim_steps} steps")}
    parity = {"case": f"one-step gradient at {a.res}^3, {head} form's algorithm, FP32 GPU vs FP32 oracle",
              "grad_rel_l2": err, "loss_rel": abs(lg - lo) / abs(lo)}
    return base, parity


def dominant_kernel_roofline(fm, sim, dev, stream):
    """Times fm_march_map (RK4 flow map + Jacobian on the three face grids and
    the centre map) on the simulator's live state with CUDA events."""
    import json as _j

    import torch

    peaks = {}
    try:
        peaks = _j.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    src = ("measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks
           else "fallback 6650 GB/s (no MEASURED_PEAKS.json on this machine)")
    g, K = sim.grid, fm.kernels
    psi, psi_f, T_f = sim.psi.clone(), [x.clone() for x in sim.psi_f], [x.clone() for x in sim.T_f]
    u = sim.u
    reps = 5
    K.march_map(g, 4, sim.dx, sim.dt, psi, psi_f, T_f, u)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        K.march_map(g, 4, sim.dx, sim.dt, psi, psi_f, T_f, u)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / reps
    ncell = g.ncell
    nface = sum(int(torch.tensor(g.face_shape(c)).prod()) for c in range(g.dim))
    # compulsory bytes: psi, T on 3 face grids r+w (2*6 floats per face node),
    # centre psi r+w (6 floats per cell), u read once (3 floats per cell)
    algo = 4 * (12 * nface + 6 * ncell + nface)
    achieved = algo / (ms / 1e3) / 1e9
    # FP32 operations of the implementation (an FMA counts 2): per face node 4 RK4
    # stages x (3 components x 195 for value + gradient + (grad u).t, plus 6 stencil
    # setups x 12) + 60 for the stage sums; per centre node 4 x (3 x 78 + 6 x 10) + 30
    flops = nface * (4 * (3 * 195 + 6 * 12) + 60) + ncell * (4 * (3 * 78 + 6 * 10) + 30)
    fp32 = fp32_peak_tflops(dev, fm)
    fp32_peak = fp32["peak"]
    fp32_achieved = flops / (ms / 1e3) / 1e12
    return {"kernel": "k_march<float,3,4> (fm_march_map)", "bound": "hbm", "achieved": achieved, "peak": hbm,
            "unit": "GB/s", "frac": achieved / hbm, "traffic": MARCH_DRAM_BYTES_PER_LAUNCH, "ms_per_launch": ms,
            "algorithmic_bytes_per_launch": algo, "peak_source": src,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch, "
                              "profiles/k_march_rk4_3d128.txt",
            "fp32": {"achieved": fp32_achieved, "peak": fp32_peak, "unit": "TFLOP/s", "frac": fp32_achieved / fp32_peak,
                     "flops_per_launch": flops,
                     "peak_source": ("measured here: the best of an FMA-chain probe (fm_fp32_fma_probe, scalar "
                                     "and paired-lane FMAs) and cuBLAS FP32 GEMM 8192^3 with TF32 off"),
                     "measured": fp32},
            "note": "gather kernel: instruction-issue bound (ncu: 527 M warp instructions per launch, issue active "
                    "66 %, L1 hit 95 %); its HBM fraction is low by construction, the fp32 entry is its bound"}


# dram bytes (read + write) of one k_march<float,3,4> launch on the 128^3
# benchmark state, from the ncu capture summarised in profiles/k_march_rk4_3d128.txt
MARCH_DRAM_BYTES_PER_LAUNCH = 371_630_592


def fp32_peak_tflops(dev, fm):
    """FP32 CUDA-core throughput measured on this GPU, TFLOP/s: an FMA-chain
    probe (scalar fmaf and paired-lane FMAs, 8 CTAs of 256 threads per SM) and
    cuBLAS SGEMM with TF32 disabled; "peak" is the best of the three."""
    import ctypes as _C

    import torch

    def best_of(fn, reps=5):
        fn()
        torch.cuda.synchronize(dev)
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize(dev)
            t = e0.elapsed_time(e1) / 1e3
            best = t if best is None else min(best, t)
        return best

    out = {}
    blocks = torch.cuda.get_device_properties(dev).multi_processor_count * 8
    iters = 65536
    buf = torch.empty(blocks * 256, dtype=torch.float32, device=dev)
    lib = fm._lib.lib()
    stream = _C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    for name, paired in (("fma_scalar", 0), ("fma_paired", 1)):
        def run(p=paired):
            fm._lib.check(lib.fm_fp32_fma_probe(p, blocks, iters, _C.c_void_p(buf.data_ptr()), stream),
                          "fm_fp32_fma_probe")
        out[name] = blocks * 256.0 * iters * 32 / best_of(run) / 1e12
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        x = torch.randn(n, n, device=dev)
        y = torch.randn(n, n, device=dev)
        out["sgemm"] = 2.0 * n ** 3 / best_of(lambda: torch.mm(x, y)) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    out["peak"] = max(out["fma_scalar"], out["fma_paired"], out["sgemm"])
    return out


if __name__ == "__main__":
    sys.exit(main())
