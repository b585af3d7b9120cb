"""ctypes binding of libflowmap_sm100.so (the C ABI in include/flowmap_sm100.h).

The product path has no fallback: if the library is missing or CUDA is not
available, every call raises ``FlowmapError``.
"""
from __future__ import annotations

import ctypes as C
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libflowmap_sm100.so")
HEADER_PATH = os.path.join(_HERE, "..", "include", "flowmap_sm100.h")

FM_F32, FM_F64 = 0, 1
FM_OK = 0
FM_ERR_CUDA = 6
STATUS = {
    0: "FM_OK",
    1: "FM_ERR_SHAPE",
    2: "FM_ERR_ARG",
    3: "FM_ERR_NOT_CONVERGED",
    4: "FM_ERR_NONFINITE",
    5: "FM_ERR_TIMEOUT",
    6: "FM_ERR_CUDA",
    7: "FM_ERR_DTYPE",
    8: "FM_ERR_CAPACITY",
}


class FlowmapError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)}")


class NotConvergedError(FlowmapError):
    pass


class Grid(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int * 3)]


class MGParams(C.Structure):
    _fields_ = [
        ("levels", C.c_int),
        ("pre_post", C.c_int),
        ("bottom", C.c_int),
        ("bottom_mode", C.c_int),
        ("max_iters", C.c_int),
        ("abs_tol", C.c_double),
        ("rel_tol", C.c_double),
        ("eps", C.c_double),
        ("check_every", C.c_int),
        ("coarse_bf16", C.c_int),
    ]


class MGStats(C.Structure):
    _fields_ = [
        ("solves", C.c_longlong),
        ("iterations", C.c_longlong),
        ("not_converged", C.c_longlong),
        ("nonfinite", C.c_longlong),
        ("last_iters", C.c_int),
        ("max_iters_seen", C.c_int),
        ("last_rtr", C.c_double),
    ]


P, D, I, L = C.c_void_p, C.c_double, C.c_int, C.c_long
GP = C.POINTER(Grid)

# signature table: name -> argtypes (restype int)
SIGNATURES = {
    "fm_abi_version": [],
    "fm_advect_u_grid": [GP, I, I, D, D] + [P] * 9 + [P],
    "fm_advect_scalar_grid": [GP, I, I, D, D] + [P] * 5 + [P],
    "fm_rk_grid": [GP, I, I, D, D, I, P, P, P, P, P, P],
    "fm_march_map": [GP, I, I, D, D] + [P] * 7 + [P] * 3 + [P],
    "fm_pullback_u": [GP, I, D] + [P] * 12 + [D, D] + [P] * 3 + [P],
    "fm_pullback_scalar": [GP, I, D, P, P, P, D, D, P, P],
    "fm_advect_scalar_grid_adj": [GP, I, I, D, D] + [P] * 9 + [P],
    "fm_advect_u_grid_adj": [GP, I, I, D, D] + [P] * 15 + [P],
    "fm_pullback_u_adj": [GP, I, D] + [P] * 9 + [D, D] + [P] * 15 + [P],
    "fm_pullback_scalar_adj": [GP, I, D, P, P, D, D, P, P, P, P, P],
    "fm_rk_grid_adj": [GP, I, I, D, D, I] + [P] * 12 + [P],
    "fm_accumulate_init": [GP, I, D, D, I, I] + [P] * 12 + [P] * 6 + [P],
    "fm_accumulate_init_pair": [GP, I, D, D, I, I] + [P] * 12 + [P] * 6 + [P] * 3 + [D, P],
    "fm_nabla_u_w": [GP, I, I, D] + [P] * 9 + [P],
    "fm_nabla_scalar_adjoint": [GP, I, D, P, P, P, P, P, P],
    "fm_reset_to_identity": [GP, I, D] + [P] * 7 + [P],
    "fm_add_fields": [I, L, P, P, P, D, P],
    "fm_mgpcg_create": [GP, I, C.POINTER(MGParams), C.POINTER(P)],
    "fm_mgpcg_destroy": [P],
    "fm_project": [P, P, P, P, P, P, C.POINTER(I), C.POINTER(D)],
    "fm_mgpcg_solve": [P, P, P, P, C.POINTER(I), C.POINTER(D)],
    "fm_laplacian": [GP, I, P, P, P],
    "fm_mgpcg_stats": [P, P, I, C.POINTER(MGStats)],
    "fm_project_noalloc": [GP, I, C.POINTER(MGParams), P, P, P, P, C.POINTER(I), C.POINTER(D)],
    "fm_convert": [L, I, P, I, P, P],
    "fm_advect_u_grid_pair": [GP, I, I, D, D] + [P] * 15 + [P],
    "fm_advect_scalar_grid_pair": [GP, I, I, D, D] + [P] * 7 + [P],
    "fm_mg_vcycle": [P, P, P, P],
    "fm_mgpcg_solve_dc": [P, I, P, P, P, D, I, P, C.POINTER(I), C.POINTER(I), C.POINTER(D)],
    "fm_project_dc": [P, P, P, P, P, D, I, P, P],
    "fm_clamp_extrema": [GP, I, I, P, P, P, P],
    "fm_tune_set": [I, GP, I],
    "fm_tune_get": [I, GP],
    "fm_solid_create": [GP, I, C.POINTER(MGParams), P, C.POINTER(P)],
    "fm_solid_destroy": [P],
    "fm_solid_set_mask": [P, P, P],
    "fm_solid_vcycle": [P, P, P, P],
    "fm_solid_solve": [P, P, P, P, C.POINTER(I), C.POINTER(D)],
    "fm_solid_project": [P, P, P, P, P, P, C.POINTER(I), C.POINTER(D)],
    "fm_solid_stats": [P, P, I, C.POINTER(MGStats)],
    "fm_mask_velocity": [GP, I, P, P, P, P, P, P],
    "fm_mask_passive": [GP, I, P, P, I, P],
    "fm_viscous_force_2d": [GP, I, D, D, P, P, P, P, P, P, P, P, P],
    "fm_gaussian_force": [GP, I, D, I, P, P, P, P, P, P, P],
    "fm_gaussian_force_grad": [GP, I, D, I, P, P, P, P, P, P, P, P, P, P, P],
    "fm_vortex_velocity_2d": [GP, I, D, I, C.POINTER(D), P, P, P],
    "fm_vortex_velocity_grad_2d": [GP, I, D, I, C.POINTER(D), P, P, P, P, P],
    "fm_vorticity_2d": [GP, I, D, P, P, P, P],
    "fm_vorticity_loss_2d": [GP, I, D, P, P, P, P, P, P, P, P, P],
}
RESTYPES = {"fm_launch_count": C.c_longlong}
SIGNATURES["fm_launch_count"] = [I]
SIGNATURES["fm_last_cuda_error"] = [C.c_char_p, I]
SIGNATURES["fm_fp32_fma_probe"] = [I, I, I, P, P]
SIGNATURES["fm_set_pdl"] = [I]

_lib = None


def lib() -> C.CDLL:
    """Load the CUDA library (raises FlowmapError-free OSError if absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python differentiable-flowmap_b200/build.py` "
                "(the flow-map package has no CPU fallback)")
        l = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(l, name)
            f.argtypes = args
            f.restype = RESTYPES.get(name, C.c_int)
        l.fm_status_string.argtypes = [C.c_int]
        l.fm_status_string.restype = C.c_char_p
        _lib = l
    return _lib


def launch_count(reset: bool = False) -> int:
    """Kernels launched by libflowmap_sm100.so so far (graph launches included)."""
    return int(lib().fm_launch_count(1 if reset else 0))


def set_pdl(enable: bool) -> bool:
    """Programmatic dependent launch for the solver kernels; returns the previous setting."""
    return bool(lib().fm_set_pdl(1 if enable else 0))


def last_cuda_error():
    """(code, name) of the CUDA error behind the library's last FM_ERR_CUDA."""
    buf = C.create_string_buffer(64)
    code = lib().fm_last_cuda_error(buf, 64)
    return code, buf.value.decode()


def check(status: int, where: str):
    if status != FM_OK:
        if status == 3:
            raise NotConvergedError(status, where)
        if status == FM_ERR_CUDA:
            code, name = last_cuda_error()
            if code:
                where = f"{where} ({name} = {code})"
        raise FlowmapError(status, where)


FM_BF16 = 2


def dtype_code(t: torch.dtype, storage: bool = False) -> int:
    """FM_F32/FM_F64 for compute entry points; FM_BF16 too for storage (fm_convert)."""
    if t == torch.float32:
        return FM_F32
    if t == torch.float64:
        return FM_F64
    if storage and t == torch.bfloat16:
        return FM_BF16
    raise FlowmapError(7, f"dtype {t}")


def ptr(t):
    """Device pointer of a contiguous CUDA tensor (None passes NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise FlowmapError(2, "tensor is not on a CUDA device (no CPU fallback)")
    if not t.is_contiguous():
        raise FlowmapError(2, "tensor must be contiguous")
    return t.data_ptr()


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def header_symbols(path: str = HEADER_PATH):
    """Function names declared in include/flowmap_sm100.h."""
    import re

    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fm_[a-z0-9_]+)\s*\(", txt)))
