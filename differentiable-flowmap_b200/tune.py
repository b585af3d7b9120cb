"""Autotuner for launch shapes: the block size of the gather kernels
(advection, flow-map march, pullbacks, accumulate_init) and the tile height of
the adjoint-source stencils (nabla_u_w, nabla_scalar_adjoint).

Those kernels compute every node independently, so the threads per block and
the stencil tiles change only how the grid fills the 148 SMs (and, for the
stencil, how much of each input footprint neighbouring tiles re-read) -- which
matters for the small 2D grids of the batched vortex instances (a 128^2 face
grid is 64 blocks of 256).  ``autotune(shape)`` times each candidate on seeded
fields of that grid shape with CUDA events, keeps the fastest per kernel class
in the library's table (fm_tune_set) and returns the timings.  With
concurrency = k the candidate runs as k copies on k streams at once (each on
its own fields), which is how the kernel meets the GPU inside a batch of
concurrent instances: a launch shape that is fastest alone can lose under
contention.  Results are cached per (shape, dtype, RK order, concurrency) for
the process.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Sequence, Tuple

import torch

from . import _lib
from . import kernels as K

KINDS = {"advect_u": 0, "advect_scalar": 1, "march": 2, "pullback_u": 3, "pullback_scalar": 4, "accumulate": 5,
         "adjoint_sources": 6}
CANDIDATES = (64, 128, 256)  # threads per block of the gather kernels
TILE_CANDIDATES = {3: (4, 8), 2: (8, 16)}  # adjoint-source tile heights along i, by dimension
_cache: Dict[Tuple, Dict[str, dict]] = {}


def set_threads(kind: str, shape: Sequence[int], threads: int):
    """fm_tune_set: threads per block for kernel class ``kind`` on grid ``shape``
    (the tile height for "adjoint_sources"; 0: default)."""
    g = K.GridSpec(tuple(shape))
    _lib.check(_lib.lib().fm_tune_set(KINDS[kind], C.byref(g.c_grid()), int(threads)), "fm_tune_set")


def get_threads(kind: str, shape: Sequence[int]) -> int:
    g = K.GridSpec(tuple(shape))
    return int(_lib.lib().fm_tune_get(KINDS[kind], C.byref(g.c_grid())))


def reset(shape: Sequence[int]):
    for k in KINDS:
        set_threads(k, shape, 0)
    for key in [k for k in _cache if k[0] == tuple(shape)]:
        del _cache[key]


def _workloads(shape, dtype, rk, device):
    g = K.GridSpec(tuple(shape))
    dim = g.dim
    dx = 1.0 / shape[0]
    dt = 0.5 * dx
    gen = torch.Generator(device=device).manual_seed(11)

    def rnd(sh, scale=1.0):
        return torch.randn(sh, dtype=dtype, device=device, generator=gen) * scale

    u = [rnd(g.face_shape(c), 0.3) for c in range(dim)]
    w = [rnd(g.face_shape(c)) for c in range(dim)]
    out = [torch.empty_like(x) for x in u]
    s = rnd(tuple(shape))
    s_out = torch.empty_like(s)
    psi_c = torch.empty((dim,) + tuple(shape), dtype=dtype, device=device)
    psi_f = [torch.empty((dim,) + g.face_shape(c), dtype=dtype, device=device) for c in range(dim)]
    T_f = [torch.empty_like(x) for x in psi_f]
    K.reset_to_identity(g, dx, psi_c, psi_f, T_f)
    march_psi = [x.clone() for x in psi_f]
    march_T = [x.clone() for x in T_f]
    march_c = psi_c.clone()
    init = [x.clone() for x in w]
    return {
        "advect_u": lambda: K.advect_u_grid(g, rk, dx, dt, u, w, out),
        "advect_scalar": lambda: K.advect_scalar_grid(g, rk, dx, dt, u, s, s_out),
        "march": lambda: K.march_map(g, rk, dx, dt, march_c, march_psi, march_T, u),
        "pullback_u": lambda: K.pullback_u(g, dx, w, out, T_f, psi_f),
        "pullback_scalar": lambda: K.pullback_scalar(g, dx, s, s_out, psi_c),
        "accumulate": lambda: K.accumulate_init(g, dx, dt, w, init, T_f, psi_f),
        "adjoint_sources": lambda: K.nabla_u_w(g, dx, u, w, out),
    }


def autotune(shape: Sequence[int], dtype=torch.float32, rk: int = 2, candidates: Sequence[int] = CANDIDATES,
             reps: int = 20, device=None, concurrency: int = 1) -> Dict[str, dict]:
    """Pick and store the fastest block size per kernel class for ``shape``;
    returns {kind: {"threads": best, "us": {candidate: microseconds per launch
    round (all ``concurrency`` copies)}}}."""
    key = (tuple(shape), dtype, rk, tuple(candidates), int(concurrency))
    if key in _cache:
        return _cache[key]
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    k = max(int(concurrency), 1)
    works = [_workloads(shape, dtype, rk, dev) for _ in range(k)]
    streams = [torch.cuda.Stream(device=dev) for _ in range(k)]
    main = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def round_(kind, n):
        # n launches of `kind` on each stream, the streams running side by side
        for st, w in zip(streams, works):
            st.wait_stream(main)
            with torch.cuda.stream(st):
                for _ in range(n):
                    w[kind]()
        for st in streams:
            main.wait_stream(st)

    result = {}
    dim = len(tuple(shape))
    for kind in works[0]:
        times = {}
        cands = TILE_CANDIDATES[dim] if kind == "adjoint_sources" else candidates
        for th in cands:
            set_threads(kind, shape, th)
            round_(kind, 3)
            torch.cuda.synchronize(dev)
            e0.record(main)
            round_(kind, reps)
            e1.record(main)
            torch.cuda.synchronize(dev)
            times[th] = e0.elapsed_time(e1) * 1e3 / reps
        best = min(cands, key=lambda t: (times[t], -t))
        set_threads(kind, shape, best)
        result[kind] = {"threads": best, "us": times}
    _cache[key] = result
    return result
