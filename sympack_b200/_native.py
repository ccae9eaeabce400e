"""ctypes binding of the C ABI declared in ``include/sympack_b200.h``.

The shared library is built in-tree (``sympack_b200/_lib/libsympack_b200.so``) by
``sympack_b200.build``; importing this module builds it first when it is missing
or stale and nvcc is available.  There is no CPU fallback: if the library
cannot be loaded, every solver call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from . import build as _build

SPB_OK = 0
SPB_ERR_INVALID = -1
SPB_ERR_NOT_SPD = -2
SPB_ERR_OOM = -3
SPB_ERR_CUDA = -4
SPB_ERR_STATE = -5
SPB_ERR_STRUCTURE = -6
SPB_ERR_TIMEOUT = -7
SPB_ERR_NOT_CONVERGED = -8

ORDERINGS = {"MMD": 0, "NATURAL": 1, "USER": 2, "RCM": 3, "AMD": 4}
PRECISIONS = {"FP64": 0, "FP32_IR": 1}
DECOMPOSITIONS = {"LL": 0, "LDL": 1}


class spb_options(C.Structure):
    _fields_ = [
        ("ordering", C.c_int),
        ("nrelax0", C.c_int),
        ("nrelax1", C.c_int),
        ("nrelax2", C.c_int),
        ("max_snode", C.c_int),
        ("zrelax0", C.c_double),
        ("zrelax1", C.c_double),
        ("zrelax2", C.c_double),
        ("user_perm", C.POINTER(C.c_int32)),
        ("device", C.c_int),
        ("precision", C.c_int),
        ("ir_tolerance", C.c_double),
        ("ir_max_iter", C.c_int),
        ("verbose", C.c_int),
        ("plan_small_max_w", C.c_int),
        ("plan_big_tile_rows", C.c_int),
        ("fp32_engine", C.c_int),
        ("decomposition", C.c_int),
        ("plan_outer_nb", C.c_int),
        ("plan_dense_min_w", C.c_int),
        ("plan_solve_chunk", C.c_int),
        ("plan_solve_tiles", C.c_int),
        ("factor_schedule", C.c_int),
    ]


class spb_info(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("nsuper", C.c_int32),
        ("nlevels", C.c_int32),
        ("max_width", C.c_int32),
        ("nnz_a", C.c_int64),
        ("nnz_l", C.c_int64),
        ("lindx_size", C.c_int64),
        ("arena_bytes", C.c_int64),
        ("device_bytes", C.c_int64),
        ("flops_stat", C.c_double),
        ("flops_exec", C.c_double),
        ("ncells", C.c_int32),
        ("nblocks", C.c_int32),
        ("ir_iterations", C.c_int32),
        ("factor_launches", C.c_int32),
        ("backward_error", C.c_double),
        ("dense_root_width", C.c_int32),
        ("pad_", C.c_int32),
        ("inverse_bytes", C.c_int64),
        ("factor_sched_us", C.c_double),
        ("factor_tasks", C.c_int32),
        ("pad2_", C.c_int32),
    ]


KIND_NAMES = ["assemble", "factor_small", "potrf_diag", "trsm_rows", "gemm_simt", "gemm_dmma",
              "solve_forward", "solve_backward", "solve_inverse"]


class spb_profile(C.Structure):
    _fields_ = [
        ("ms", C.c_double * 9),
        ("flops", C.c_double * 9),
        ("bytes", C.c_double * 9),
        ("launches", C.c_int32 * 9),
    ]


# (name, restype, argtypes) of every exported entry point
_P = C.c_void_p
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)
_DP = C.POINTER(C.c_double)
SIGNATURES = [
    ("spb_default_options", None, [C.POINTER(spb_options)]),
    ("spb_create", C.c_int, [C.POINTER(spb_options), C.POINTER(_P)]),
    ("spb_destroy", None, [_P]),
    ("spb_last_error", C.c_char_p, [_P]),
    ("spb_symbolic", C.c_int, [_P, C.c_int32, _I64P, _I32P]),
    ("spb_symbolic_batch", C.c_int, [_P, C.c_int32, _I32P, C.c_int32, _I64P, _I32P]),
    ("spb_symbolic_from", C.c_int, [_P, _P]),
    ("spb_predict_device_bytes", C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_int64)]),
    ("spb_replan", C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32]),
    ("spb_get_solve_trace", C.c_int, [_P, C.c_int32, C.POINTER(C.c_uint64), C.c_int64, C.POINTER(C.c_int64)]),
    ("spb_distribute", C.c_int, [_P, _DP]),
    ("spb_distribute_device", C.c_int, [_P, _P]),
    ("spb_factorize", C.c_int, [_P]),
    ("spb_solve", C.c_int, [_P, _DP, C.c_int32, C.c_int64]),
    ("spb_get_solution", C.c_int, [_P, _DP, C.c_int32, C.c_int64]),
    ("spb_solve_device", C.c_int, [_P, _P, _P, C.c_int32, C.c_int64]),
    ("spb_solve_device_noalloc", C.c_int, [_P, _P, _P, C.c_int32, C.c_int64]),
    ("spb_get_info", C.c_int, [_P, C.POINTER(spb_info)]),
    ("spb_get_ordering", C.c_int, [_P, _I32P, _I32P]),
    ("spb_get_mmd_invp", C.c_int, [_P, _I32P]),
    ("spb_get_etree", C.c_int, [_P, _I32P]),
    ("spb_get_colcounts", C.c_int, [_P, _I32P, _I32P]),
    ("spb_get_supernodes", C.c_int, [_P, _I32P, _I32P]),
    ("spb_get_structure", C.c_int, [_P, _I64P, _I32P]),
    ("spb_get_cells", C.c_int, [_P, _I32P, _I32P, _I32P, _I32P, _I32P, _I32P, _I32P]),
    ("spb_get_factor", C.c_int, [_P, _DP]),
    ("spb_get_status", C.c_int, [_P, _I32P, _I32P, _I32P]),
    ("spb_set_wait_limit", C.c_int, [_P, C.c_int64]),
    ("spb_debug_stall", C.c_int, [_P, C.c_int32]),
    ("spb_debug_stall_factor", C.c_int, [_P, C.c_int32]),
    ("spb_set_factor_trace", C.c_int, [_P, C.c_int32]),
    ("spb_get_factor_trace", C.c_int, [_P, C.POINTER(C.c_uint64), C.c_int64, C.POINTER(C.c_int64), _I32P]),
    ("spb_reorder_factor_from_trace", C.c_int, [_P]),
    ("spb_clear_status", C.c_int, [_P]),
    ("spb_set_stream", C.c_int, [_P, _P]),
    ("spb_set_profiling", C.c_int, [_P, C.c_int]),
    ("spb_get_profile", C.c_int, [_P, C.POINTER(spb_profile)]),
    ("spb_rb_info", C.c_int, [C.c_char_p, _I32P, _I64P]),
    ("spb_rb_read", C.c_int, [C.c_char_p, _I64P, _I32P, _DP]),
    ("spb_rb_write", C.c_int, [C.c_char_p, C.c_char_p, C.c_int32, _I64P, _I32P, _DP]),
]

_lib = None


def lib_path() -> Path:
    return _build.LIB


def load() -> C.CDLL:
    """Load (building if needed) the native library; raises if it cannot."""
    global _lib
    if _lib is not None:
        return _lib
    if _build.needs_build():
        if os.environ.get("SPB_NO_BUILD"):
            raise RuntimeError(f"native library missing or stale: {_build.LIB}")
        _build.build()
    lib = C.CDLL(str(_build.LIB))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return [name for name, _, _ in SIGNATURES]
