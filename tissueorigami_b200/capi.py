"""ctypes binding of the C ABI declared in ``include/tf_b200.h``.

This is the Python face of the drop-in boundary: every call goes straight to
``_lib/libtf_b200.so``. There is no CPU fallback - if the library or a CUDA device is missing,
``load()`` raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

TF_OK = 0
TF_NEWTON_NOT_CONVERGED = 1
TF_KRYLOV_MAX_ITERS = 2
TF_KRYLOV_BREAKDOWN = 3
TF_NONFINITE = 4
TF_ELEMENT_INVERTED = 5
TF_ERR_ARGUMENT = -1
TF_ERR_CUDA = -2
TF_ERR_OUT_OF_MEMORY = -3
TF_ERR_STATE = -4
TF_ERR_UNSUPPORTED = -5
TF_ERR_TOO_LARGE = -6
TF_NOALLOC_MAX_NODES = 16384

TF_PRECOND_BLOCK_JACOBI = 0
TF_PRECOND_ILU0 = 1
TF_PRECOND_TWO_LEVEL = 2
TF_PRECOND_MULTILEVEL = 3
TF_KRYLOV_AUTO = 0
TF_KRYLOV_BICGSTAB = 1
TF_KRYLOV_CG = 2
TF_SCATTER_AUTO = 0
TF_SCATTER_ATOMIC = 1
TF_SCATTER_COLOURED = 2
TF_SCATTER_STAGED = 3

STATUS_NAMES = {
    0: "ok", 1: "newton_not_converged", 2: "krylov_max_iters", 3: "krylov_breakdown",
    4: "nonfinite", 5: "element_inverted", -1: "argument", -2: "cuda", -3: "out_of_memory",
    -4: "state", -5: "unsupported", -6: "too_large",
}

# Every entry point include/tf_b200.h declares (checked by the CPU test suite).
EXPORTS = [
    "tf_default_params", "tf_version", "tf_create", "tf_destroy", "tf_set_material",
    "tf_set_inv_fg", "tf_set_boundary", "tf_set_viscosity_surface", "tf_newton_step",
    "tf_newton_step_device", "tf_get_pattern", "tf_assemble", "tf_solve", "tf_set_growth",
    "tf_get_growth", "tf_time_step", "tf_time_step_device", "tf_get_schedule", "tf_autotune",
    "tf_time_kernels", "tf_last_error", "tf_solve_bsr_noalloc", "tf_batch_create",
    "tf_get_tissue_stats", "tf_get_n_tissues", "tf_adjoint_forward", "tf_adjoint_backward",
    "tf_solve_direct", "tf_get_preconditioner", "tf_get_smoother_block", "tf_measure_fp64", "tf_invert_dense", "tf_set_packing", "tf_detect_packing",
    "tf_get_packing", "tf_set_lumen", "tf_get_lumen",
    "tf_set_grid_growth", "tf_set_time", "tf_get_time", "tf_set_external_force", "tf_newton_iteration",
    "tf_get_krylov_method",
]


class MeshDesc(ctypes.Structure):
    _fields_ = [("n_nodes", ctypes.c_int32), ("n_elems", ctypes.c_int32),
                ("conn", ctypes.POINTER(ctypes.c_int32)), ("xref", ctypes.POINTER(ctypes.c_double))]


class Params(ctypes.Structure):
    _fields_ = [("max_newton_iters", ctypes.c_int32), ("newton_tol", ctypes.c_double),
                ("krylov_max_iters", ctypes.c_int32), ("krylov_rtol", ctypes.c_double),
                ("precond", ctypes.c_int32), ("scatter", ctypes.c_int32),
                ("elems_per_block", ctypes.c_int32), ("device", ctypes.c_int32),
                ("use_graphs", ctypes.c_int32), ("persistent", ctypes.c_int32),
                ("smoother_nodes", ctypes.c_int32), ("krylov_refine", ctypes.c_int32),
                ("krylov_method", ctypes.c_int32), ("krylov_warm_start", ctypes.c_int32)]


class GridGrowth(ctypes.Structure):
    _fields_ = [("t0", ctypes.c_double), ("t1", ctypes.c_double), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
                ("rates", ctypes.POINTER(ctypes.c_double)), ("angles", ctypes.POINTER(ctypes.c_double)),
                ("z_min", ctypes.c_double), ("z_max", ctypes.c_double), ("flags", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class StepStats(ctypes.Structure):
    _fields_ = [("newton_iters", ctypes.c_int32), ("krylov_iters_total", ctypes.c_int32),
                ("krylov_iters_max", ctypes.c_int32), ("status", ctypes.c_int32),
                ("du_norm", ctypes.c_double * 32), ("krylov_rel_res", ctypes.c_double * 32),
                ("ms_assemble", ctypes.c_double), ("ms_solve", ctypes.c_double),
                ("ms_total", ctypes.c_double), ("gpu_launches", ctypes.c_int64),
                ("ms_solve_kernel", ctypes.c_double), ("solve_launches", ctypes.c_int32),
                ("krylov_method", ctypes.c_int32), ("krylov_iters_cg", ctypes.c_int32)]

    def as_dict(self):
        n = min(self.newton_iters, 32)
        return {"newton_iters": self.newton_iters, "krylov_iters_total": self.krylov_iters_total,
                "krylov_iters_max": self.krylov_iters_max, "status": self.status,
                "du_norm": list(self.du_norm[:n]), "krylov_rel_res": list(self.krylov_rel_res[:n]),
                "ms_assemble": self.ms_assemble, "ms_solve": self.ms_solve, "ms_total": self.ms_total,
                "gpu_launches": int(self.gpu_launches), "ms_solve_kernel": self.ms_solve_kernel,
                "solve_launches": int(self.solve_launches), "krylov_method": int(self.krylov_method),
                "krylov_iters_cg": int(self.krylov_iters_cg)}


_lib = None

_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int32)
_U = ctypes.POINTER(ctypes.c_uint8)


def lib_path() -> str:
    return _build.LIB_PATH


def load(build_if_missing: bool = True):
    """Load the CUDA library (building it first when missing); raises if that is impossible."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB_PATH
    if not os.path.exists(path):
        if not build_if_missing:
            raise RuntimeError(f"tissueorigami_b200 CUDA library missing: {path}")
        _build.build()
    L = ctypes.CDLL(path)
    c_int, c_double = ctypes.c_int32, ctypes.c_double
    L.tf_default_params.argtypes = [ctypes.POINTER(Params)]
    L.tf_default_params.restype = None
    L.tf_version.restype = ctypes.c_char_p
    L.tf_create.argtypes = [ctypes.POINTER(MeshDesc), ctypes.POINTER(Params), ctypes.POINTER(_P)]
    L.tf_destroy.argtypes = [_P]
    L.tf_destroy.restype = None
    L.tf_set_material.argtypes = [_P, _D, _D, _D]
    L.tf_set_inv_fg.argtypes = [_P, _D]
    L.tf_set_boundary.argtypes = [_P, _U, _D, _I, c_int]
    L.tf_set_viscosity_surface.argtypes = [_P, _D]
    L.tf_newton_step.argtypes = [_P, _D, c_double, _D, ctypes.POINTER(StepStats)]
    L.tf_newton_step_device.argtypes = [_P, _P, c_double, _P, ctypes.POINTER(StepStats)]
    L.tf_get_pattern.argtypes = [_P, _I, _I, _I]
    L.tf_assemble.argtypes = [_P, _D, _D, c_double, _D, _D]
    L.tf_solve.argtypes = [_P, _D, _D, _D, _I, _D]
    L.tf_set_growth.argtypes = [_P, _D, _D, _D, _U, _U]
    L.tf_get_growth.argtypes = [_P, _D, _D]
    L.tf_time_step.argtypes = [_P, _D, c_double, _D, ctypes.POINTER(StepStats)]
    L.tf_time_step_device.argtypes = [_P, _P, c_double, _P, ctypes.POINTER(StepStats)]
    L.tf_get_schedule.argtypes = [_P, _I, _I, _I]
    L.tf_get_preconditioner.argtypes = [_P, _I, _I, _I]
    L.tf_get_smoother_block.argtypes = [_P, _I]
    L.tf_autotune.argtypes = [_P, _D, c_double]
    L.tf_time_kernels.argtypes = [_P, c_int, _D, _D]
    L.tf_batch_create.argtypes = [c_int, ctypes.POINTER(MeshDesc), ctypes.POINTER(Params), ctypes.POINTER(_P)]
    L.tf_get_tissue_stats.argtypes = [_P, _I, _I, _I]
    L.tf_get_n_tissues.argtypes = [_P]
    L.tf_adjoint_forward.argtypes = [_P, _D, c_int, c_double, c_int, _D, ctypes.POINTER(StepStats)]
    L.tf_adjoint_backward.argtypes = [_P, _D, _D, _D, ctypes.POINTER(StepStats)]
    L.tf_solve_direct.argtypes = [_P, _D, _D, _D, _D, _I]
    L.tf_solve_bsr_noalloc.argtypes = [c_int, _P, _P, _P, _P, _P, c_double, c_int, _P, _I, _D]
    L.tf_measure_fp64.argtypes = [c_int, _D]
    L.tf_invert_dense.argtypes = [c_int, c_int, c_int, c_int, _D, _I]
    L.tf_set_packing.argtypes = [_P, c_int, _I]
    L.tf_detect_packing.argtypes = [_P, _D, _I]
    L.tf_get_packing.argtypes = [_P, c_int, _I, _I, _D, _D, _D]
    L.tf_set_lumen.argtypes = [_P, c_int, _I, c_double, c_double, _D]
    L.tf_get_lumen.argtypes = [_P, _D, _D, _D]
    L.tf_set_grid_growth.argtypes = [_P, c_int, ctypes.POINTER(GridGrowth), c_int, _D, _D, _I]
    L.tf_set_time.argtypes = [_P, c_double]
    L.tf_set_external_force.argtypes = [_P, _D]
    L.tf_get_krylov_method.argtypes = [_P, _I]
    L.tf_newton_iteration.argtypes = [_P, _D, _D, c_double, _D, _I, _D]
    L.tf_get_time.argtypes = [_P, _D]
    L.tf_last_error.argtypes = [_P]
    L.tf_last_error.restype = ctypes.c_char_p
    for name in EXPORTS:
        fn = getattr(L, name)
        if fn.restype is ctypes.c_int:  # default restype
            fn.restype = c_int
    _lib = L
    return L


def default_params() -> Params:
    p = Params()
    load().tf_default_params(ctypes.byref(p))
    return p


def dptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, "float64 C-contiguous array expected"
    return a.ctypes.data_as(_D)


def iptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous, "int32 C-contiguous array expected"
    return a.ctypes.data_as(_I)


def uptr(a):
    if a is None:
        return None
    assert a.dtype == np.uint8 and a.flags.c_contiguous, "uint8 C-contiguous array expected"
    return a.ctypes.data_as(_U)


class TFError(RuntimeError):
    def __init__(self, code, where, detail=""):
        super().__init__(f"{where} failed: {STATUS_NAMES.get(code, code)} ({code}) {detail}")
        self.code = code


def check(code, where, ctx=None):
    """Raise on errors (< 0); pass numerical outcomes (>= 0) back to the caller."""
    if code < 0:
        detail = ""
        if ctx or where in ("tf_create", "tf_batch_create"):
            msg = load().tf_last_error(ctx if ctx else None)
            detail = msg.decode() if msg else ""
        raise TFError(code, where, detail)
    return code
