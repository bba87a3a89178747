"""ctypes binding of libfeatb200.so (the C ABI declared in include/featb200.h).

The library is built in-tree by ``feat3.doxytest_b200/build.py``; importing this module without it
raises immediately: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfeatb200.so")

FB_OK = 0
SOLVER_STATUS = {0: "undefined", 1: "progress", 2: "success", 3: "aborted", 4: "diverged", 5: "max_iter",
                 6: "stagnated"}
PREC = {"f64": 0, "f32": 1, "f32_bf16": 2}
ORDER = {"native": 0, "rcm": 1}


class FeatB200Error(RuntimeError):
    pass


class CsrHost(C.Structure):
    _fields_ = [("rows", C.c_uint64), ("columns", C.c_uint64), ("used_elements", C.c_uint64),
                ("row_ptr", C.c_void_p), ("col_ind", C.c_void_p), ("val", C.c_void_p)]


class SolverConfig(C.Structure):
    _fields_ = [("precision", C.c_int), ("ordering", C.c_int), ("omega", C.c_double),
                ("smooth_steps", C.c_int), ("tol_rel", C.c_double), ("tol_abs", C.c_double),
                ("max_iter", C.c_int), ("min_iter", C.c_int), ("use_graph", C.c_int),
                ("rows_per_block", C.c_int), ("tail_rows", C.c_int), ("tma_rows", C.c_int),
                ("cluster_rows", C.c_int), ("cycle", C.c_int), ("tma_window", C.c_int),
                ("diagonal", C.c_int), ("pdl", C.c_int),
                ("adapt_cgc", C.c_int), ("fused", C.c_int), ("smoother", C.c_int),
                ("smoother_omega", C.c_double), ("sweep_colouring", C.c_int),
                ("streamed", C.c_int)]


class StoragePlan(C.Structure):
    _fields_ = [("kind", C.c_int), ("narrow", C.c_int), ("width", C.c_uint32), ("diagonals", C.c_uint32),
                ("entries", C.c_uint64)]


class SolveInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("def_init", C.c_double),
                ("def_final", C.c_double), ("solve_ms", C.c_double), ("kernel_launches", C.c_uint64),
                ("bytes_moved", C.c_double)]


P = C.c_void_p
U64 = C.c_uint64
D = C.c_double
F = C.c_float
I = C.c_int

# name -> (restype, argtypes); every function returns fb_status unless stated
_PROTOS = {
    "fb_last_error": (C.c_char_p, []),
    "fb_version": (C.c_char_p, []),
    "fb_kernel_launch_count": (U64, []),
    "fb_apply_csr_f64_u64": (I, [P, D, P, D, P, P, P, P, U64, U64, U64, I, P]),
    "fb_apply_csr_f64_u32": (I, [P, D, P, D, P, P, P, P, U64, U64, U64, I, P]),
    "fb_apply_csr_f32_u64": (I, [P, F, P, F, P, P, P, P, U64, U64, U64, I, P]),
    "fb_apply_csr_f32_u32": (I, [P, F, P, F, P, P, P, P, U64, U64, U64, I, P]),
    "fb_axpy_f64": (I, [P, D, P, P, U64, P]),
    "fb_axpy_f32": (I, [P, F, P, P, U64, P]),
    "fb_dot_f64": (I, [P, P, P, U64, P]),
    "fb_dot_f32": (I, [P, P, P, U64, P]),
    "fb_dot_f64_noalloc": (I, [P, P, P, U64, P]),
    "fb_solver_set_iteration_limits": (I, [P, I, I]),
    "fb_q1_pattern_3d": (I, [I, P, P, P]),
    "fb_q1_assemble_3d": (I, [I, I, P, P, P, P, P]),
    "fb_q1_prolongation_3d": (I, [I, C.POINTER(C.c_uint64), P, P, P, P]),
    "fb_set_memory_f64": (I, [P, D, U64, P]),
    "fb_set_memory_f32": (I, [P, F, U64, P]),
    "fb_set_memory_u64": (I, [P, U64, U64, P]),
    "fb_set_memory_u32": (I, [P, C.c_uint32, U64, P]),
    "fb_scale_rows_csr_f64_u64": (I, [P, P, P, P, U64, P]),
    "fb_norm2_f64": (I, [P, P, U64, P]),
    "fb_norm2_f32": (I, [P, P, U64, P]),
    "fb_component_product_f64": (I, [P, P, P, U64, P]),
    "fb_component_product_f32": (I, [P, P, P, U64, P]),
    "fb_component_invert_f64": (I, [P, P, D, U64, P]),
    "fb_component_invert_f32": (I, [P, P, F, U64, P]),
    "fb_scale_f64": (I, [P, P, D, U64, P]),
    "fb_scale_f32": (I, [P, P, F, U64, P]),
    "fb_unit_filter_rhs_f64_u64": (I, [P, P, P, U64, P]),
    "fb_unit_filter_def_f64_u64": (I, [P, P, U64, P]),
    "fb_unit_filter_rhs_f32_u32": (I, [P, P, P, U64, P]),
    "fb_unit_filter_def_f32_u32": (I, [P, P, U64, P]),
    "fb_diagonal_csr_u64": (I, [P, P, P, U64, P]),
    "fb_convert_f64_to_f32": (I, [P, P, U64, P]),
    "fb_convert_f32_to_f64": (I, [P, P, U64, P]),
    "fb_hierarchy_create": (I, [C.POINTER(P), I]),
    "fb_hierarchy_set_level": (I, [P, I, C.POINTER(CsrHost), P, P, U64, C.POINTER(CsrHost),
                                   C.POINTER(CsrHost)]),
    "fb_hierarchy_destroy": (None, [P]),
    "fb_solver_config_default": (None, [C.POINTER(SolverConfig)]),
    "fb_solver_create": (I, [C.POINTER(P), P, C.POINTER(SolverConfig)]),
    "fb_solver_destroy": (None, [P]),
    "fb_solver_solve": (I, [P, P, P, C.POINTER(SolveInfo)]),
    "fb_solver_solve_device": (I, [P, P, P, P, C.POINTER(SolveInfo)]),
    "fb_solver_vcycle": (I, [P, P, P]),
    "fb_solver_level_info": (I, [P, P]),
    "fb_multigrid_cycle_events": (I, [I, I, I, P, P, U64, C.POINTER(C.c_uint64)]),
    "fb_matrix_storage_plan": (I, [C.POINTER(CsrHost), P, U64, I, I, C.POINTER(StoragePlan)]),
    "fb_solver_update_matrix": (I, [P, I, P, P]),
    "fb_solver_set_tolerances": (I, [P, D, D]),
    "fb_q1_pattern_2d": (I, [I, P, P, P]),
    "fb_q1_assemble_2d": (I, [I, I, P, P, D, I, P, P, P, P, P]),
    "fb_q1_sample_2d": (I, [I, I, P, P, D, I, P, P, P, P]),
    "fb_q1_prolongation_2d": (I, [I, C.POINTER(C.c_uint64), P, P, P, P]),
    "fb_unet_create": (I, [C.POINTER(P), I, I]),
    "fb_unet_destroy": (None, [P]),
    "fb_unet_num_params": (I, [P, C.POINTER(C.c_uint64)]),
    "fb_unet_set_params": (I, [P, P]),
    "fb_unet_get_params": (I, [P, P]),
    "fb_unet_get_grads": (I, [P, P]),
    "fb_unet_forward": (I, [P, P, P, I, P]),
    "fb_unet_backward": (I, [P, P, I, I, P]),
    "fb_unet_adam": (I, [P, C.c_float, C.c_float, C.c_float, C.c_float, I, P]),
    "fb_unet_mse": (I, [P, P, P, C.c_uint64, P, P, P]),
    "fb_solver_time_kernel": (I, [P, I, I, I, C.POINTER(D), C.POINTER(D)]),
    "fb_msolver_create": (I, [C.POINTER(P), P, C.POINTER(SolverConfig), I]),
    "fb_msolver_destroy": (None, [P]),
    "fb_msolver_solve": (I, [P, P, P, P]),
    "fb_msolver_solve_device": (I, [P, P, P, P, P]),
    "fb_batch_create": (I, [C.POINTER(P), I, C.POINTER(P), C.POINTER(SolverConfig)]),
    "fb_batch_destroy": (None, [P]),
    "fb_batch_sizes": (I, [P, P]),
    "fb_batch_solve": (I, [P, P, P, P]),
    "fb_batch_solve_device": (I, [P, P, P, P, P]),
    "fb_batch_rows_per_block": (I, [P, P, C.POINTER(I)]),
}

_lib = None


def lib():
    """The loaded library; raises FeatB200Error when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FeatB200Error(
                f"featb200: {LIB_PATH} is missing; build it with `python feat3.doxytest_b200/build.py` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return sorted(_PROTOS)


def check(status, what="featb200"):
    if status != FB_OK:
        msg = lib().fb_last_error().decode(errors="replace")
        raise FeatB200Error(f"{what} failed with status {status}: {msg}")


def launch_count():
    return int(lib().fb_kernel_launch_count())
