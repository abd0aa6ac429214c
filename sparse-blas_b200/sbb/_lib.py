"""Loader for libsbb.so (the CUDA product) and libsbbgen.so (generators).

There is no fallback: if the shared library is missing or fails to load, this
raises.  Build it with ``make -C sparse-blas_b200`` (or
``__graft_entry__.build()``).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsbb.so")
GEN_PATH = os.path.join(HERE, "libsbbgen.so")

_lib = None
_gen = None

vp = C.c_void_p
dp = C.POINTER(C.c_double)


class Config(C.Structure):
    """sbb_config (include/sbb_spmv.h)."""
    _fields_ = [("kernel", C.c_int), ("vector_width", C.c_int),
                ("items_per_thread", C.c_int), ("persistent", C.c_int),
                ("tile_sigma", C.c_int)]


class PlanInfo(C.Structure):
    """sbb_plan_info (include/sbb_spmv.h)."""
    _fields_ = [("kernel", C.c_int), ("vector_width", C.c_int),
                ("items_per_thread", C.c_int), ("persistent", C.c_int),
                ("tile_sigma", C.c_int), ("tiles", C.c_int),
                ("max_row_len", C.c_int), ("empty_rows", C.c_int),
                ("scratch_bytes", C.c_size_t)]


class GenParams(C.Structure):
    """sbbgen_params (csrc/gen/generators.cpp)."""
    _fields_ = [("seed", C.c_ulonglong), ("family", C.c_int), ("m", C.c_int), ("n", C.c_int),
                ("expo", C.c_double), ("lmin", C.c_double), ("lmax", C.c_double),
                ("p", C.c_double), ("hw", C.c_int), ("block", C.c_int), ("r", C.c_double),
                ("mu", C.c_double), ("sigma", C.c_double), ("ndense", C.c_int),
                ("dense_lo", C.c_double), ("dense_hi", C.c_double), ("dense_expo", C.c_double),
                ("p_empty", C.c_double), ("unit_values", C.c_int)]


class BatchItem(C.Structure):
    """sbb_batch_item (include/sbb_spmv.h)."""
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("nnz", C.c_int), ("rowptr", vp), ("col", vp),
                ("val", vp), ("x", vp), ("y", vp), ("alpha", C.c_double), ("beta", C.c_double),
                ("cls", C.c_int)]


# Every symbol include/sbb_spmv.h declares, with its ctypes signature.
SIGNATURES = {
    "spMV_mgpu_baseline": (C.c_int, [C.c_int, C.c_int, C.c_longlong, dp, vp, vp, vp, vp, dp, vp,
                                     C.c_int]),
    "spMV_mgpu_v1": (C.c_int, [C.c_int, C.c_int, C.c_longlong, dp, vp, vp, vp, vp, dp, vp,
                               C.c_int, C.c_int]),
    "spMV_mgpu_v2": (C.c_int, [C.c_int, C.c_int, C.c_longlong, dp, vp, vp, vp, vp, dp, vp,
                               C.c_int, C.c_int, C.c_longlong, C.c_int]),
    "csr5_kernel": (C.c_int, [C.c_int, C.c_int, C.c_int, dp, vp, vp, vp, vp, dp, vp]),
    "get_row_from_index": (C.c_int, [C.c_int, vp, C.c_longlong]),
    "get_time": (C.c_double, []),
    "get_gpu_availble_mem": (C.c_double, [C.c_int]),
    "sbb_plan_create": (C.c_int, [C.POINTER(vp), C.c_int, C.c_int, C.c_int, vp, vp, vp,
                                  C.POINTER(Config), vp]),
    "sbb_plan_create_f32": (C.c_int, [C.POINTER(vp), C.c_int, C.c_int, C.c_int, vp, vp, vp,
                                      C.POINTER(Config), vp]),
    "sbb_plan_create_f32_lanes": (C.c_int, [C.POINTER(vp), C.c_int, C.c_int, C.c_int, vp, vp,
                                            vp, C.POINTER(Config), vp]),
    "sbb_spmv": (C.c_int, [vp, C.c_double, vp, C.c_double, vp, vp]),
    "sbb_spmv_f32": (C.c_int, [vp, C.c_double, vp, C.c_double, vp, vp]),
    "sbb_spmv_timed": (C.c_int, [vp, C.c_double, vp, C.c_double, vp, vp, vp, vp]),
    "sbb_plan_launches": (C.c_int, [vp]),
    "sbb_plan_check": (C.c_int, [vp]),
    "sbb_plan_info_get": (C.c_int, [vp, C.POINTER(PlanInfo)]),
    "sbb_plan_partition": (C.c_int, [vp, vp, vp, C.c_int]),
    "sbb_plan_destroy": (C.c_int, [vp]),
    "sbb_batch_create": (C.c_int, [C.POINTER(vp), C.POINTER(BatchItem), C.c_int, vp]),
    "sbb_batch_run": (C.c_int, [vp, vp]),
    "sbb_batch_run_graph": (C.c_int, [vp, vp]),
    "sbb_batch_run_each": (C.c_int, [vp, vp]),
    "sbb_batch_launches": (C.c_int, [vp, C.c_int]),
    "sbb_batch_check": (C.c_int, [vp]),
    "sbb_batch_destroy": (C.c_int, [vp]),
    "sbb_tune_classes": (C.c_int, [C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, C.c_double,
                                   C.c_double, C.c_int, C.POINTER(C.c_float), vp]),
    "sbb_features": (C.c_int, [C.c_int, C.c_int, C.c_int, vp, vp, vp, vp]),
    "sbb_mlp_forward": (C.c_int, [vp, vp, C.c_int, vp, vp]),
    "sbb_mlp_grad": (C.c_int, [vp, vp, vp, vp, C.c_int, vp, vp, vp]),
    "sbb_mlp_train": (C.c_int, [vp, vp, vp, vp, C.c_int, C.c_int, C.c_float, C.c_float, vp, vp]),
    "sbb_mlp_select": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, vp, C.POINTER(C.c_int), vp]),
    "sbb_mm_load": (C.c_int, [C.c_char_p, C.c_double, C.POINTER(vp), C.POINTER(C.c_int),
                              C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    "sbb_mm_copy": (C.c_int, [vp, vp, vp, vp]),
    "sbb_mm_free": (None, [vp]),
    "sbb_spmv_merge_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, vp, vp, vp, C.c_double, vp,
                                         C.c_double, vp, vp]),
    "sbb_last_error": (C.c_char_p, []),
    "sbb_last_call_phases": (C.c_int, [dp, C.c_int]),
    "sbb_test_hook": (C.c_int, [C.c_int, C.c_longlong]),
}

# sbb_test_hook selectors (include/sbb_spmv.h)
TEST_RESET, TEST_FAIL_ALLOC, TEST_FREE_BYTES, TEST_WAIT_BUDGET = 0, 1, 2, 3


def lib():
    """libsbb.so with argtypes set; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libsbb.so not built at {LIB_PATH}; run make -C sparse-blas_b200")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().sbb_last_error().decode(errors="replace")


def gen():
    global _gen
    if _gen is None:
        if not os.path.exists(GEN_PATH):
            raise RuntimeError(f"libsbbgen.so not built at {GEN_PATH}")
        G = C.CDLL(GEN_PATH)
        G.sbbgen_rowptr.argtypes = [C.POINTER(GenParams), vp]
        G.sbbgen_rowptr.restype = C.c_longlong
        G.sbbgen_fill.argtypes = [C.POINTER(GenParams), vp, vp, vp]
        G.sbbgen_fill.restype = None
        G.sbbgen_uniform.argtypes = [C.c_ulonglong, C.c_longlong, C.c_double, C.c_double, vp]
        G.sbbgen_uniform.restype = None
        G.sbbgen_threads.restype = C.c_int
        _gen = G
    return _gen
