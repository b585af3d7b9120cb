"""B200-native (sm_100a) leapfrog flow-map fluid step, adjoint and MGPCG.

Import with ``importlib.import_module("differentiable-flowmap_b200")`` (the
directory name is not a Python identifier).  All compute runs in
libflowmap_sm100.so through its C ABI (include/flowmap_sm100.h); there is no
CPU fallback.
"""
from . import _lib, kernels
from ._lib import FlowmapError, NotConvergedError
from .kernels import GridSpec
from .mgpcg import MGPCG, MGPCG_2, MGPCG_2_solid, MGPCG_3

__all__ = ["FlowmapError", "NotConvergedError", "GridSpec", "MGPCG", "MGPCG_2", "MGPCG_2_solid", "MGPCG_3",
           "kernels", "_lib"]
