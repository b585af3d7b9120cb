"""Many vortex-optimisation instances of uneven grid sizes advanced together.

Each instance owns its simulator, solver handle and CUDA stream; one host
thread per instance issues its gradient (forward + adjoint), so the GPU
interleaves the instances' small kernels (a single 2D instance of these sizes
leaves most of the 148 SMs idle).  Every projection runs on the device (CUDA-
graph WHILE loop), so an instance's step never waits for the host; the only
host synchronisations per gradient are the loss read at the seed and the
solver statistics at the end, each on the instance's own stream.  All kernels
and reductions are deterministic, so every instance's result equals its
unbatched run bit for bit.
"""
from __future__ import annotations

import threading
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from . import kernels as K
from .configs import vortex2d_config, vortex2d_theta
from .simulator import LFM_Diff_Simulator
from .vortex import VortexProblem


@dataclass
class VortexInstance:
    res: int
    theta: np.ndarray
    omega_target: Optional[torch.Tensor] = None
    problem: Optional[VortexProblem] = None
    stream: Optional[torch.cuda.Stream] = None
    loss: Optional[float] = None
    dtheta: Optional[np.ndarray] = None


DEFAULT_SIZES = (128,) * 4 + (192,) * 4 + (256,) * 4 + (384,) * 4


def instance_cost(res: int, steps: int) -> int:
    """Work of one 2D instance's gradient: cells x steps (every kernel is per cell)."""
    return res * res * steps


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Instances across ``world`` ranks by greedy bin-packing: the costliest
    first (ties by index), each to the least-loaded rank (ties to the lowest).
    Deterministic; every instance lands on exactly one rank; each rank's list
    is in ascending instance order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]


def rank_share(sizes: Sequence[int], steps: int, rank: int, world: int) -> List[int]:
    """The global instance indices rank ``rank`` of ``world`` advances."""
    return partition([instance_cost(n, steps) for n in sizes], world)[rank]


def gather_results(local: dict, group=None) -> dict:
    """Merge every rank's {instance index: result} (torch.distributed
    all_gather_object; called after the timed region)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return dict(local)
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local, group=group)
    out = {}
    for p in parts:
        overlap = set(out) & set(p)
        if overlap:
            raise RuntimeError(f"instances {sorted(overlap)} reported by two ranks")
        out.update(p)
    return out


class BatchedVortex:
    """16-instance batch: 4 x 128^2, 4 x 192^2, 4 x 256^2, 4 x 384^2 vortex
    optimisations.  ``indices`` selects the global instances this process
    advances (a rank's share); seeds follow the global index, so results do not
    depend on the partition.  ``autotune`` picks the gather kernels' block
    sizes per instance shape first (tune.py)."""

    def __init__(self, sizes: Sequence[int] = DEFAULT_SIZES, steps: int = 100,
                 reinit_every: int = 10, dtype=torch.float32, rel_tol: float = 1e-6, control_seed0: int = 100,
                 target_seed0: int = 200, device=None, indices: Optional[Sequence[int]] = None,
                 autotune: bool = True):
        _lib.lib()  # load the library once, before any worker thread
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.instances: List[VortexInstance] = []
        self.indices = list(range(len(sizes))) if indices is None else list(indices)
        # block sizes of the gather kernels per instance shape (tune.py); results do not change
        self.tuning = {}
        if autotune:
            from . import tune

            # each shape timed as it runs here: as many concurrent copies as the
            # batch has instances
            with torch.cuda.device(self.device):
                for n in sorted({sizes[i] for i in self.indices}):
                    self.tuning[n] = tune.autotune((n, n), dtype, rk=2, device=self.device,
                                                   concurrency=len(self.indices))
        for i in self.indices:
            n = sizes[i]
            cfg = vortex2d_config(res=n, steps=steps, reinit_every=reinit_every, dtype=dtype, rel_tol=rel_tol)
            stream = torch.cuda.Stream(device=self.device)
            with torch.cuda.stream(stream):
                prob = VortexProblem(LFM_Diff_Simulator(config=cfg, device=self.device))
                omt = prob.final_vorticity(vortex2d_theta(target_seed0 + i))
            self.instances.append(VortexInstance(n, vortex2d_theta(control_seed0 + i), omt, prob, stream))
        torch.cuda.synchronize(self.device)

    def capture(self, single_graph: bool = False):
        """Record every instance's gradient as a CUDA graph (untimed setup; runs one
        eager gradient per instance first).  single_graph=False: one graph per
        instance, replayed on its own stream.  single_graph=True: ONE graph for the
        whole batch, each instance's forward + adjoint a branch forked from the
        capturing stream onto the instance's stream and joined back, so a batch
        gradient is one graph launch; the branches have no dependencies between
        them and run concurrently."""
        self.batch_graph = None
        if not single_graph:
            for inst in self.instances:
                with torch.cuda.device(self.device), torch.cuda.stream(inst.stream):
                    inst.problem.capture(inst.theta, inst.omega_target)
            torch.cuda.synchronize(self.device)
            self.captured = True
            return
        with torch.cuda.device(self.device):
            for inst in self.instances:
                with torch.cuda.stream(inst.stream):
                    inst.problem.prepare_record(inst.theta, inst.omega_target)
            torch.cuda.synchronize(self.device)
            main = torch.cuda.Stream(device=self.device)
            graph = torch.cuda.CUDAGraph()
            recorded = []
            with torch.cuda.graph(graph, stream=main, capture_error_mode="thread_local"):
                # every fork before any join: a branch forked after an earlier branch's
                # join would depend on that branch and run after it
                for inst in self.instances:
                    inst.stream.wait_stream(main)
                for inst in self.instances:
                    with torch.cuda.stream(inst.stream):
                        recorded.append(inst.problem.record())
                for inst in self.instances:
                    main.wait_stream(inst.stream)
        self.batch_graph = graph
        self.batch_roles = [r[0] for r in recorded]
        self.batch_loss = [r[1] for r in recorded]
        self.batch_kernels = sum(r[2] for r in recorded)
        self.captured = True

    def _run(self, inst: VortexInstance):
        with torch.cuda.device(self.device), torch.cuda.stream(inst.stream):
            inst.loss, inst.dtheta = inst.problem.gradient(inst.theta, inst.omega_target)

    def gradients(self, concurrent: bool = True, graphs: bool = False):
        """One gradient per instance; concurrent=False runs them one after another.
        graphs=True replays the captured graphs (capture() first): one graph
        launch per instance on its stream, all issued from this thread, or, after
        capture(single_graph=True), one graph launch for the whole batch; then the
        losses and dL/dtheta are read back instance by instance."""
        if graphs and getattr(self, "batch_graph", None) is not None:
            # the whole batch as one graph launch on the current stream
            with torch.cuda.device(self.device):
                for inst in self.instances:
                    K.vortex_velocity_2d(inst.problem.grid, inst.problem.dx, inst.theta, inst.problem._u0[0],
                                         inst.problem._u0[1])
                self.batch_graph.replay()
                for inst, roles, loss in zip(self.instances, self.batch_roles, self.batch_loss):
                    for k, v in roles.items():
                        setattr(inst.problem.sim, k, v)
                    inst.loss = float(loss.item())
                    inst.problem.loss = inst.loss
                    inst.dtheta = inst.problem.calculate_dtheta(inst.theta)
        elif graphs:
            if not getattr(self, "captured", False):
                raise RuntimeError("gradients(graphs=True): call capture() first")
            with torch.cuda.device(self.device):
                for inst in self.instances:
                    with torch.cuda.stream(inst.stream):
                        inst.problem.launch_gradient(inst.theta)
                        if not concurrent:
                            inst.loss, inst.dtheta = inst.problem.finish_gradient(inst.theta)
                if concurrent:
                    for inst in self.instances:
                        with torch.cuda.stream(inst.stream):
                            inst.loss, inst.dtheta = inst.problem.finish_gradient(inst.theta)
        elif not concurrent:
            for inst in self.instances:
                self._run(inst)
        else:
            errors = []

            def work(inst):
                try:
                    self._run(inst)
                except BaseException as e:  # re-raised on the caller's thread
                    errors.append(e)

            threads = [threading.Thread(target=work, args=(inst,)) for inst in self.instances]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
            if errors:
                raise errors[0]
        torch.cuda.synchronize(self.device)
        return [(inst.loss, inst.dtheta) for inst in self.instances]
