"""ctypes front end of the CPU oracle (liboracle.so) and of oracle/_ref/libref.so.

TEST INFRASTRUCTURE ONLY.  The tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module as the checker; the
product (the ``sbb`` package and libsbb.so) never does.

``liboracle.so`` restates the reference's path in C (see sbb_oracle.c for the
file:line each function follows).  ``_ref/libref.so`` is the reference's own
host drivers (SparseBLAS/src/dspmv_mgpu_{baseline,v1,v2}.cu, spmv_helper.cu)
compiled unchanged against CPU stand-ins for the CUDA runtime and the removed
legacy cuSPARSE csrmv (ref_shim.cpp); it exists only where the reference
sources were present at build time.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


class Slice(C.Structure):
    """orc_slice: one GPU's (v1/baseline) or one task's (v2) share."""
    _fields_ = [("start_idx", C.c_longlong), ("end_idx", C.c_longlong),
                ("start_row", C.c_int), ("end_row", C.c_int),
                ("start_flag", C.c_int), ("end_flag", C.c_int),
                ("y2", C.c_double)]

    def as_tuple(self):
        return (self.start_idx, self.end_idx, self.start_row, self.end_row,
                bool(self.start_flag), bool(self.end_flag))


def build(ref: bool = False) -> None:
    """liboracle.so; with ref, also _ref/libref.so from the reference sources
    named by REF or SBB_REFERENCE_SRC in the environment."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_get_row_from_index.argtypes = [C.c_int, i64p, C.c_longlong]
        L.orc_get_row_from_index.restype = C.c_int
        L.orc_v1_partition.argtypes = [C.c_int, C.c_longlong, i64p, C.c_int, C.POINTER(Slice)]
        L.orc_baseline_partition.argtypes = [C.c_int, i64p, C.c_int, C.POINTER(Slice)]
        L.orc_v2_num_tasks.argtypes = [C.c_longlong, C.c_longlong]
        L.orc_v2_num_tasks.restype = C.c_int
        L.orc_v2_tasks.argtypes = [C.c_int, C.c_longlong, i64p, f64p, C.c_longlong, C.c_int,
                                   C.POINTER(Slice)]
        common = [C.c_int, C.c_int, C.c_longlong, C.c_double, f64p, i64p, i32p, f64p,
                  C.c_double, f64p]
        L.orc_dropin_baseline.argtypes = common + [C.c_int]
        L.orc_dropin_v1.argtypes = common + [C.c_int, C.c_int]
        L.orc_dropin_v2.argtypes = common + [C.c_int, C.c_longlong, C.c_int]
        for f in (L.orc_dropin_baseline, L.orc_dropin_v1, L.orc_dropin_v2):
            f.restype = C.c_int
        L.orc_spmv_host.argtypes = [C.c_int, i64p, i32p, f64p, f64p, C.c_double, C.c_double,
                                    f64p, C.c_int]
        L.orc_spmv_host_f32.argtypes = [C.c_int, i32p, i32p, f32p, f32p, C.c_double,
                                        C.c_double, f64p, C.c_int]
        L.orc_spmv_dd.argtypes = [C.c_int, i64p, i32p, f64p, f64p, C.c_double, C.c_double,
                                  f64p, f64p, f64p]
        L.orc_merge_path_split.argtypes = [C.c_int, i32p, C.c_longlong, C.c_int, i32p, i32p]
        L.orc_csr5_sigma.argtypes = [C.c_int, C.c_longlong]
        L.orc_csr5_sigma.restype = C.c_int
        _LIB = L
    return _LIB


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref.so"))


def ref():
    """The reference's own drivers (CPU stand-ins for CUDA/cuSPARSE)."""
    global _REF
    if _REF is None:
        R = C.CDLL(os.path.join(HERE, "_ref", "libref.so"))
        R.ref_get_row_from_index.argtypes = [C.c_int, i64p, C.c_longlong]
        R.ref_get_row_from_index.restype = C.c_int
        R.ref_set_free_bytes.argtypes = [C.c_ulonglong]
        dptr = C.POINTER(C.c_double)
        common = [C.c_int, C.c_int, C.c_longlong, dptr, f64p, i64p, i32p, f64p, dptr, f64p]
        R.ref_spMV_mgpu_baseline.argtypes = common + [C.c_int]
        R.ref_spMV_mgpu_baseline.restype = C.c_int
        R.ref_spMV_mgpu_v1.argtypes = common + [C.c_int, C.c_int]
        R.ref_spMV_mgpu_v1.restype = C.c_int
        R.ref_spMV_mgpu_v2.argtypes = common + [C.c_int, C.c_int, C.c_longlong, C.c_int]
        R.ref_spMV_mgpu_v2.restype = None
        _REF = R
    return _REF


# ---------------------------------------------------------------- helpers

def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def get_row_from_index(rowptr, idx: int) -> int:
    rp = _c(rowptr, np.int64)
    return lib().orc_get_row_from_index(len(rp) - 1, rp, idx)


def v1_partition(rowptr, nnz: int, P: int):
    rp = _c(rowptr, np.int64)
    out = (Slice * P)()
    lib().orc_v1_partition(len(rp) - 1, nnz, rp, P, out)
    return [s.as_tuple() for s in out]


def baseline_partition(rowptr, P: int):
    rp = _c(rowptr, np.int64)
    out = (Slice * P)()
    lib().orc_baseline_partition(len(rp) - 1, rp, P, out)
    return [s.as_tuple() for s in out]


def v2_tasks(rowptr, nnz: int, y, nb: int):
    rp = _c(rowptr, np.int64)
    T = lib().orc_v2_num_tasks(nnz, nb)
    out = (Slice * T)()
    lib().orc_v2_tasks(len(rp) - 1, nnz, rp, _c(y, np.float64), nb, T, out)
    return [s.as_tuple() + (s.y2,) for s in out]


def dropin(version: str, m, n, nnz, alpha, val, rowptr, col, x, beta, y, ngpu=1,
           kernel=1, nb=None, q=1):
    """Oracle result of spMV_mgpu_{baseline,v1,v2}; returns (rc, y_out)."""
    yo = _c(y, np.float64).copy()
    args = (m, n, nnz, float(alpha), _c(val, np.float64), _c(rowptr, np.int64),
            _c(col, np.int32), _c(x, np.float64), float(beta), yo)
    L = lib()
    if version == "baseline":
        rc = L.orc_dropin_baseline(*args, ngpu)
    elif version == "v1":
        rc = L.orc_dropin_v1(*args, ngpu, kernel)
    elif version == "v2":
        rc = L.orc_dropin_v2(*args, kernel, nnz if nb is None else nb, q)
    else:
        raise ValueError(version)
    return rc, yo


def ref_dropin(version: str, m, n, nnz, alpha, val, rowptr, col, x, beta, y, ngpu=1,
               kernel=1, nb=None, q=1):
    """The reference's own driver on the CPU stand-ins; returns (rc, y_out)."""
    yo = _c(y, np.float64).copy()
    a = C.c_double(alpha)
    b = C.c_double(beta)
    args = (m, n, nnz, C.byref(a), _c(val, np.float64), _c(rowptr, np.int64),
            _c(col, np.int32), _c(x, np.float64), C.byref(b), yo)
    R = ref()
    if version == "baseline":
        rc = R.ref_spMV_mgpu_baseline(*args, ngpu)
    elif version == "v1":
        rc = R.ref_spMV_mgpu_v1(*args, ngpu, kernel)
    elif version == "v2":
        R.ref_spMV_mgpu_v2(*args, ngpu, kernel, nnz if nb is None else nb, q)
        rc = 0
    else:
        raise ValueError(version)
    return rc, yo


def spmv_host(rowptr, col, val, x, alpha, beta, y, nthreads=1):
    """The reference's host loop (main.cu:350-356) with +beta*y; returns y_out."""
    yo = _c(y, np.float64).copy()
    rp = _c(rowptr, np.int64)
    lib().orc_spmv_host(len(rp) - 1, rp, _c(col, np.int32), _c(val, np.float64),
                        _c(x, np.float64), float(alpha), float(beta), yo, nthreads)
    return yo


def spmv_host_f32(rowptr32, col, val32, x32, alpha, beta, y, nthreads=1):
    yo = _c(y, np.float64).copy()
    rp = _c(rowptr32, np.int32)
    lib().orc_spmv_host_f32(len(rp) - 1, rp, _c(col, np.int32), _c(val32, np.float32),
                            _c(x32, np.float32), float(alpha), float(beta), yo, nthreads)
    return yo


def spmv_dd(rowptr, col, val, x, alpha, beta, y):
    """Accurate (double-double) y and the per-row error scale."""
    rp = _c(rowptr, np.int64)
    m = len(rp) - 1
    yo = np.empty(m, np.float64)
    sc = np.empty(m, np.float64)
    lib().orc_spmv_dd(m, rp, _c(col, np.int32), _c(val, np.float64), _c(x, np.float64),
                      float(alpha), float(beta), _c(y, np.float64), yo, sc)
    return yo, sc


def rel_err(y, y_ref, scale):
    """Per-row error |y - y_ref| / scale (scale 0 rows must match exactly)."""
    y = np.asarray(y, np.float64)
    d = np.abs(y - y_ref)
    out = np.zeros_like(d)
    nz = scale > 0
    out[nz] = d[nz] / scale[nz]
    out[~nz] = np.where(d[~nz] == 0, 0.0, np.inf)
    return out


def merge_path_split(rowptr32, items_per_part: int, P: int):
    rp = _c(rowptr32, np.int32)
    rows = np.empty(P + 1, np.int32)
    nzs = np.empty(P + 1, np.int32)
    lib().orc_merge_path_split(len(rp) - 1, rp, items_per_part, P, rows, nzs)
    return rows, nzs


def csr5_sigma(m: int, nnz: int) -> int:
    return lib().orc_csr5_sigma(m, nnz)
