"""ctypes binding of the C ABI in include/helm_b200.h (libhelm_b200.so, built in-tree).

There is no fallback: if the library is missing or cannot be loaded, every
entry point raises.  Build it with ``python -m mpi_b200.build``.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhelm_b200.so")

HELM_OK = 0
HELM_ERR_INVALID = 1
HELM_ERR_NOT_POW2 = 2
HELM_ERR_SINGULAR = 3
HELM_ERR_OOM = 4
HELM_ERR_CUDA = 5
HELM_ERR_UNSUPPORTED = 6
HELM_ERR_NO_DEVICE = 7

HELM_FP64 = 0
HELM_FP32 = 1
HELM_FP32_REFINE = 2

HELM_METHOD_AUTO = 0
HELM_METHOD_LU = 1
HELM_METHOD_FDM = 2

# Every symbol the header declares (tests check the library exports them all).
EXPORTS = (
    "helm2d_plan_create", "helm3d_plan_create", "helm_plan_set_layout", "helm_plan_set_io_bytes",
    "helm_plan_set_refine_sweeps", "helm_solve", "helm_solve_adjoint", "helm_plan_get_grid",
    "helm_plan_info", "helm_plan_destroy", "helm_status_string", "helm_last_error",
    "helm_plan_set_stage_timing", "helm_plan_stage_times", "helm_fd3d_plan_create",
    "helm2d_batch_create", "helm_batch_offsets", "helm_batch_info", "helm_batch_set_graph",
    "helm_batch_solve", "helm_batch_destroy", "helm_plan_get_launch_variants", "helm_plan_set_launch_variants",
    "helm2d_periodic_plan_create", "helm3d_periodic_plan_create", "helm_gll_derivative", "helm_fourier_derivative",
    "helm_write_tecplot", "helm_write_vtk", "helm_solve_adjoint_misfit", "helm_solve_static_scratch",
    "helm_plan_kernels", "helm_debug_fail_alloc", "helm_plan_device_status", "helm_plan_set_operator_callback",
    "helm_gll_grid", "helm_lu_factor", "helm_lu_solve", "helm_max_abs_diff", "helm_batch_device_status",
    "helm_plan_set_derivative_variant", "helm_plan_get_derivative_variant",
)

# operator callback of helm_plan_set_operator_callback: void op(int iw, int jw, double* op, int ld, void* user)
OPERATOR_FN = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                               ctypes.c_void_p)

# exact-solution callback of helm_write_tecplot: double exact(double x, double y, double z)
EXACT_FN = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double)


class HelmError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        lib = _lib
        msg = lib.helm_status_string(status).decode() if lib else str(status)
        last = lib.helm_last_error().decode() if lib else ""
        super().__init__(f"{where}: {msg} ({status})" + (f" [{last}]" if last else ""))


class robin_t(ctypes.Structure):
    _fields_ = [("alphal", ctypes.c_double), ("betal", ctypes.c_double),
                ("alphar", ctypes.c_double), ("betar", ctypes.c_double)]


_lib = None


def lib() -> ctypes.CDLL:
    """Load libhelm_b200.so (raises when it is absent: no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m mpi_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    i, d, ll, vp = ctypes.c_int, ctypes.c_double, ctypes.c_longlong, ctypes.c_void_p
    P = ctypes.POINTER
    L.helm2d_plan_create.argtypes = [i, i, i, d, d, d, d, P(robin_t), d, i, i, P(vp)]
    L.helm3d_plan_create.argtypes = [i, i, i, i, d, d, d, d, d, d, P(robin_t), d, i, i, P(vp)]
    L.helm_fd3d_plan_create.argtypes = [i, i, i, d, d, d, d, d, d, P(robin_t), d, i, P(vp)]
    L.helm_gll_derivative.argtypes = [vp, i, vp, vp, vp]
    L.helm_write_tecplot.argtypes = [vp, vp, EXACT_FN, ctypes.c_char_p]
    L.helm_write_vtk.argtypes = [vp, vp, ctypes.c_char_p]
    L.helm_solve_adjoint_misfit.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
    L.helm_fourier_derivative.argtypes = [vp, i, i, vp, vp, vp]
    L.helm2d_periodic_plan_create.argtypes = [i, i, i, d, d, d, d, d, i, i, P(vp)]
    L.helm3d_periodic_plan_create.argtypes = [i, i, i, i, d, d, d, d, d, d, d, i, i, P(vp)]
    L.helm_plan_set_layout.argtypes = [vp, ll, ll, ll]
    L.helm_plan_set_io_bytes.argtypes = [vp, i]
    L.helm_plan_set_refine_sweeps.argtypes = [vp, i]
    L.helm_solve.argtypes = [vp, vp, vp, vp, vp, vp]
    L.helm_solve_adjoint.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
    L.helm_plan_get_grid.argtypes = [vp, vp, vp, vp]
    L.helm_plan_info.argtypes = [vp, P(i), P(i), P(i), P(ll)]
    L.helm_plan_destroy.argtypes = [vp]
    L.helm_plan_set_stage_timing.argtypes = [vp, i]
    L.helm_plan_stage_times.argtypes = [vp, P(ctypes.c_float)]
    L.helm_plan_device_status.argtypes = [vp, P(ctypes.c_int), ctypes.c_int]
    L.helm_plan_set_operator_callback.argtypes = [vp, OPERATOR_FN, vp]
    L.helm_gll_grid.argtypes = [i, i, d, vp, vp, vp]
    L.helm_lu_factor.argtypes = [i, vp, vp, vp]
    L.helm_lu_solve.argtypes = [i, vp, vp, vp]
    L.helm_max_abs_diff.argtypes = [vp, vp, vp, vp, vp]
    L.helm_batch_device_status.argtypes = [vp, P(ctypes.c_int), ctypes.c_int]
    L.helm2d_batch_create.argtypes = [i, P(i), P(i), P(d), d, d, d, d, i, P(vp)]
    L.helm_batch_offsets.argtypes = [vp, P(ll), P(ll)]
    L.helm_batch_info.argtypes = [vp, P(i), P(i), P(ll)]
    L.helm_batch_set_graph.argtypes = [vp, i]
    L.helm_batch_solve.argtypes = [vp, vp, vp, vp]
    L.helm_batch_destroy.argtypes = [vp]
    L.helm_plan_get_launch_variants.argtypes = [vp, P(i), P(i)]
    L.helm_plan_set_launch_variants.argtypes = [vp, P(i), i]
    L.helm_plan_set_derivative_variant.argtypes = [vp, i]
    L.helm_plan_get_derivative_variant.argtypes = [vp, P(i)]
    L.helm_status_string.argtypes = [i]
    L.helm_status_string.restype = ctypes.c_char_p
    L.helm_last_error.argtypes = []
    L.helm_last_error.restype = ctypes.c_char_p
    L.helm_debug_fail_alloc.argtypes = [ctypes.c_longlong]
    L.helm_plan_kernels.argtypes = [ctypes.c_void_p]
    L.helm_plan_kernels.restype = ctypes.c_char_p
    for name in EXPORTS:
        f = getattr(L, name)
        if f.restype is None or f.restype is ctypes.c_int:
            if name not in ("helm_status_string", "helm_last_error", "helm_plan_kernels"):
                f.restype = ctypes.c_int
    _lib = L
    return L


def check(status: int, where: str) -> None:
    if status != HELM_OK:
        raise HelmError(status, where)
