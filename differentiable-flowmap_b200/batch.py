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


class BatchedVortex:
    """16-instance batch of BASELINE config 4: 4 x 128^2, 4 x 192^2, 4 x 256^2, 4 x 384^2."""

    def __init__(self, sizes: Sequence[int] = (128,) * 4 + (192,) * 4 + (256,) * 4 + (384,) * 4, steps: int = 100,
                 reinit_every: int = 10, dtype=torch.float32, rel_tol: float = 1e-6, control_seed0: int = 100,
                 target_seed0: int = 200, device=None):
        _lib.lib()  # load the library once, before any worker thread
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.instances: List[VortexInstance] = []
        for i, n in enumerate(sizes):
            cfg = vortex2d_config(res=n, steps=steps, reinit_every=reinit_every, dtype=dtype, rel_tol=rel_tol)
            stream = torch.cuda.Stream(device=self.device)
            with torch.cuda.stream(stream):
                prob = VortexProblem(LFM_Diff_Simulator(config=cfg, device=self.device))
                omt = prob.final_vorticity(vortex2d_theta(target_seed0 + i))
            self.instances.append(VortexInstance(n, vortex2d_theta(control_seed0 + i), omt, prob, stream))
        torch.cuda.synchronize(self.device)

    def _run(self, inst: VortexInstance):
        with torch.cuda.device(self.device), torch.cuda.stream(inst.stream):
            inst.loss, inst.dtheta = inst.problem.gradient(inst.theta, inst.omega_target)

    def gradients(self, concurrent: bool = True):
        """One gradient per instance; concurrent=False runs them one after another."""
        if not concurrent:
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
