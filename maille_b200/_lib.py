"""ctypes binding of the C ABI declared in include/maille_gpu.h (libmaille_gpu.so, in-tree).

The library is the product: there is no Python or CPU fallback. Loading fails loudly when the
shared library is missing, and every compute call reports the library's status codes.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmaille_gpu.so")

MAILLE_OK, MAILLE_SINGULAR, MAILLE_NOT_CONVERGED, MAILLE_INVALID_INPUT, MAILLE_CUDA_ERROR, \
    MAILLE_CANCELLED = range(6)
MAILLE_FP64, MAILLE_MIXED = 0, 1
MAILLE_NOALLOC_MAX_BLOCK_ROWS = 1 << 26
MAILLE_ORDER_AUTO, MAILLE_ORDER_MULTICOLOR, MAILLE_ORDER_RCM, MAILLE_ORDER_MULTICOLOR_BFS = 0, 1, 2, 3
MAILLE_ORDER_MULTICOLOR_ITERATED = 4

_d = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)
_i32 = ctypes.POINTER(ctypes.c_int32)
_u8 = ctypes.POINTER(ctypes.c_uint8)


class ElasticProblem(ctypes.Structure):
    _fields_ = [
        ("n_nodes", ctypes.c_int64), ("coords", _d), ("nodes_per_elem", ctypes.c_int32),
        ("n_elems", ctypes.c_int64), ("conn", _i64), ("young", _d), ("poisson", _d),
        ("fixed", _u8), ("imposed", _d), ("f", _d), ("rel_tol", ctypes.c_double),
        ("max_iter", ctypes.c_int32), ("precision", ctypes.c_int32), ("ordering", ctypes.c_int32),
        ("device", ctypes.c_int32),
    ]


class ElasticResult(ctypes.Structure):
    _fields_ = [
        ("u", _d), ("reactions", _d), ("gauss_stress", _d), ("von_mises", _d),
        ("iterations", ctypes.c_int32), ("outer_iterations", ctypes.c_int32),
        ("final_rel_residual", ctypes.c_double), ("shift", ctypes.c_double),
        ("free_dofs", ctypes.c_int64), ("block_rows", ctypes.c_int64), ("blocks", ctypes.c_int64),
        ("levels", ctypes.c_int32), ("ms_setup", ctypes.c_double), ("ms_upload", ctypes.c_double),
        ("ms_assembly", ctypes.c_double), ("ms_factor", ctypes.c_double),
        ("ms_solve", ctypes.c_double), ("ms_post", ctypes.c_double),
        ("ms_download", ctypes.c_double), ("ms_element", ctypes.c_double),
        ("ms_ordering", ctypes.c_double), ("ms_symbolic", ctypes.c_double),
        ("ms_buffers", ctypes.c_double),
    ]


MAILLE_BATCH_MAX_RHS = 8


class BatchProblem(ctypes.Structure):
    _fields_ = [
        ("n_instances", ctypes.c_int32), ("nodes_per_elem", ctypes.c_int32),
        ("n_rhs", ctypes.c_int32), ("node_offset", _i64), ("elem_offset", _i64),
        ("coords", _d), ("conn", _i64), ("young", _d), ("poisson", _d), ("fixed", _u8),
        ("imposed", _d), ("f", _d), ("rel_tol", ctypes.c_double), ("max_iter", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("device", ctypes.c_int32),
    ]


class BatchResult(ctypes.Structure):
    _fields_ = [
        ("u", _d), ("iterations", _i32), ("rel_residual", _d), ("status", _i32),
        ("max_iterations", ctypes.c_int32), ("levels", ctypes.c_int32),
        ("free_dofs", ctypes.c_int64), ("block_rows", ctypes.c_int64), ("blocks", ctypes.c_int64),
        ("lanes_per_row", ctypes.c_int32), ("rhs_per_lane", ctypes.c_int32),
        ("threads", ctypes.c_int32), ("task_slices", ctypes.c_int32), ("autotuned", ctypes.c_int32),
        ("ms_setup", ctypes.c_double), ("ms_upload", ctypes.c_double),
        ("ms_assembly", ctypes.c_double), ("ms_factor", ctypes.c_double),
        ("ms_tune", ctypes.c_double), ("ms_solve", ctypes.c_double),
        ("ms_download", ctypes.c_double),
    ]


class LargeStrainProblem(ctypes.Structure):
    _fields_ = [
        ("n_nodes", ctypes.c_int64), ("coords", _d), ("n_elems", ctypes.c_int64), ("conn", _i64),
        ("young", _d), ("poisson", _d), ("fixed", _u8), ("imposed", _d), ("f", _d),
        ("increments", ctypes.c_int32), ("newton_tol", ctypes.c_double),
        ("newton_max_iter", ctypes.c_int32), ("rel_tol", ctypes.c_double),
        ("max_iter", ctypes.c_int32), ("precision", ctypes.c_int32), ("device", ctypes.c_int32),
    ]


class LargeStrainResult(ctypes.Structure):
    _fields_ = [
        ("u", _d), ("reactions", _d), ("newton_iterations", _i32), ("cuts", _i32),
        ("newton_total", ctypes.c_int64), ("pcg_total", ctypes.c_int64), ("ms_total", ctypes.c_double),
    ]


class ThermalProblem(ctypes.Structure):
    _fields_ = [
        ("n_nodes", ctypes.c_int64), ("coords", _d), ("nodes_per_elem", ctypes.c_int32),
        ("n_elems", ctypes.c_int64), ("conn", _i64), ("conductivity", _d), ("rho_c", _d),
        ("fixed", _u8), ("imposed", _d), ("f", _d), ("n_convection", ctypes.c_int64),
        ("conv_elem", _i64), ("conv_face", _i32), ("conv_film", _d), ("initial", _d),
        ("time_step", ctypes.c_double), ("theta", ctypes.c_double), ("increments", ctypes.c_int32),
        ("rel_tol", ctypes.c_double), ("max_iter", ctypes.c_int32), ("ordering", ctypes.c_int32),
        ("device", ctypes.c_int32), ("precision", ctypes.c_int32),
    ]


class ThermalResult(ctypes.Structure):
    _fields_ = [
        ("temperatures", _d), ("reactions", _d), ("heat_fluxes", _d), ("iterations", _i32),
        ("iterations_total", ctypes.c_int64), ("max_rel_residual", ctypes.c_double),
        ("shift", ctypes.c_double), ("free_nodes", ctypes.c_int64), ("nonzeros", ctypes.c_int64),
        ("levels", ctypes.c_int32), ("ms_setup", ctypes.c_double), ("ms_upload", ctypes.c_double),
        ("ms_assembly", ctypes.c_double), ("ms_factor", ctypes.c_double), ("ms_steps", ctypes.c_double),
        ("ms_download", ctypes.c_double),
    ]


# every symbol include/maille_gpu.h declares, with its ctypes signature
SIGNATURES = {
    "maille_gpu_last_error": ([], ctypes.c_char_p),
    "maille_gpu_version": ([], ctypes.c_char_p),
    "maille_gpu_device_count": ([], ctypes.c_int32),
    "maille_gpu_elastic_solve": ([ctypes.POINTER(ElasticProblem), ctypes.POINTER(ElasticResult)],
                                 ctypes.c_int32),
    "maille_gpu_create": ([ctypes.POINTER(ElasticProblem), ctypes.POINTER(ctypes.c_void_p)],
                          ctypes.c_int32),
    "maille_gpu_solve": ([ctypes.c_void_p, _d, ctypes.POINTER(ElasticResult)], ctypes.c_int32),
    "maille_gpu_backward": ([ctypes.c_void_p, _d, _d, _d], ctypes.c_int32),
    "maille_gpu_solve_device": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int32),
    "maille_gpu_cancel": ([ctypes.c_void_p, ctypes.c_int32], None),
    "maille_gpu_stream": ([ctypes.c_void_p], ctypes.c_void_p),
    "maille_gpu_destroy": ([ctypes.c_void_p], None),
    "maille_gpu_refactor": ([ctypes.c_void_p, _d, _d], ctypes.c_int32),
    "maille_gpu_multiply": ([ctypes.c_void_p, _d, _d], ctypes.c_int32),
    "maille_gpu_nodal_stresses": ([ctypes.c_void_p, _d, _d], ctypes.c_int32),
    "maille_gpu_trim_memory": ([ctypes.c_int32], ctypes.c_int32),
    "maille_gpu_wait_selftest": ([ctypes.c_int32, ctypes.c_int32, _i32], ctypes.c_int32),
    "maille_gpu_spmv_device": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32], ctypes.c_int32),
    "maille_gpu_kernel_launches": ([], ctypes.c_int64),
    "maille_gpu_bsr3_spmv_dot_noalloc": ([ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                                         ctypes.c_int32),
    "maille_gpu_face_pressure_loads": ([ctypes.c_int64, _d, ctypes.c_int32, ctypes.c_int64, _i64,
                                        ctypes.c_int64, _i64, _i32, _d, _d], ctypes.c_int32),
    "maille_gpu_batched_solve": ([ctypes.POINTER(BatchProblem), ctypes.POINTER(BatchResult)],
                                 ctypes.c_int32),
    "maille_gpu_batch_create": ([ctypes.POINTER(BatchProblem), ctypes.POINTER(ctypes.c_void_p)],
                                ctypes.c_int32),
    "maille_gpu_batch_solve": ([ctypes.c_void_p, _d, ctypes.POINTER(BatchResult)], ctypes.c_int32),
    "maille_gpu_batch_refactor": ([ctypes.c_void_p, _d, _d], ctypes.c_int32),
    "maille_gpu_batch_cancel": ([ctypes.c_void_p, ctypes.c_int32], None),
    "maille_gpu_batch_stream": ([ctypes.c_void_p], ctypes.c_void_p),
    "maille_gpu_batch_destroy": ([ctypes.c_void_p], None),
    "maille_gpu_large_strain_create": ([ctypes.POINTER(LargeStrainProblem), ctypes.POINTER(ctypes.c_void_p)],
                                       ctypes.c_int32),
    "maille_gpu_large_strain_run": ([ctypes.c_void_p, ctypes.POINTER(LargeStrainResult)], ctypes.c_int32),
    "maille_gpu_large_strain_backward": ([ctypes.c_void_p, _d, _d, _d], ctypes.c_int32),
    "maille_gpu_large_strain_set_materials": ([ctypes.c_void_p, _d, _d], ctypes.c_int32),
    "maille_gpu_large_strain_cancel": ([ctypes.c_void_p, ctypes.c_int32], None),
    "maille_gpu_large_strain_destroy": ([ctypes.c_void_p], None),
    "maille_gpu_thermal_transient": ([ctypes.POINTER(ThermalProblem), ctypes.POINTER(ThermalResult)],
                                     ctypes.c_int32),
    "maille_gpu_thermal_cancel": ([ctypes.c_int32, ctypes.c_int32], ctypes.c_int32),
    "maille_gpu_thermal_loads": ([ctypes.c_int64, _d, ctypes.c_int32, ctypes.c_int64, _i64, ctypes.c_int64,
                                  _i64, _d, ctypes.c_int64, _i64, _i32, _d, _d, _d], ctypes.c_int32),
}

_lib = None


def load():
    """Loads libmaille_gpu.so (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m maille_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def last_error() -> str:
    return load().maille_gpu_last_error().decode()


def ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None
