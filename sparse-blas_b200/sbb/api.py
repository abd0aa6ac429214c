"""The reference's entry points, called from Python with host (numpy) arrays.

Same names, argument order, meaning and return codes as
SparseBLAS/include/spmv_kernel.h:9-34 of JieyangChen7/Sparse-BLAS: ``alpha``
and ``beta`` are scalars (passed to the C ABI by pointer), ``y`` is updated in
place, the return value is 0 on success, -1 on a bad argument / not enough
device memory / device error, 1 on an allocation failure.  ``ngpu`` is
accepted and pinned to 1.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import lib


def _arr(a, dt, name):
    if not isinstance(a, np.ndarray) or a.dtype != dt or not a.flags["C_CONTIGUOUS"]:
        raise TypeError(f"{name} must be a C-contiguous numpy array of {np.dtype(dt).name}")
    return a.ctypes.data_as(C.c_void_p)


def _common(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y):
    a = C.c_double(float(alpha))
    b = C.c_double(float(beta))
    return [int(m), int(n), int(nnz), C.byref(a), _arr(csrVal, np.float64, "csrVal"),
            _arr(csrRowPtr, np.int64, "csrRowPtr"), _arr(csrColIndex, np.int32, "csrColIndex"),
            _arr(x, np.float64, "x"), C.byref(b), _arr(y, np.float64, "y")], (a, b)


def spMV_mgpu_baseline(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y, ngpu=1):
    args, keep = _common(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y)
    return lib().spMV_mgpu_baseline(*args, int(ngpu))


def spMV_mgpu_v1(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y, ngpu=1,
                 kernel=1):
    args, keep = _common(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y)
    return lib().spMV_mgpu_v1(*args, int(ngpu), int(kernel))


def spMV_mgpu_v2(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y, ngpu=1,
                 kernel=1, nb=None, q=1):
    args, keep = _common(m, n, nnz, alpha, csrVal, csrRowPtr, csrColIndex, x, beta, y)
    return lib().spMV_mgpu_v2(*args, int(ngpu), int(kernel), int(nnz if nb is None else nb),
                              int(q))


def get_row_from_index(n, a, idx):
    return lib().get_row_from_index(int(n), _arr(a, np.int64, "a"), int(idx))


def get_time():
    return lib().get_time()


def get_gpu_availble_mem(ngpu=1):
    return lib().get_gpu_availble_mem(int(ngpu))
