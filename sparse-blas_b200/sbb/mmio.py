"""Matrix Market files: read (through libsbb's reader) and write.

``read`` returns canonical CSR (rows and columns sorted, duplicates summed,
symmetric storage expanded) whatever the entry order of the file; the
reference's test driver used the file's COO order as CSR, which is right only
for files sorted by row (SparseBLAS/test/dspmv_test.cu:228-251, 305-306).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import last_error, lib
from .gen import Csr


class MatrixMarketError(RuntimeError):
    pass


def read(path, pattern_value: float = 1.0) -> Csr:
    """The matrix of a Matrix Market coordinate file (real / integer /
    pattern; general / symmetric / skew-symmetric) as CSR; entries of a
    pattern file get ``pattern_value``."""
    h = C.c_void_p()
    m, n, nnz = C.c_int(), C.c_int(), C.c_longlong()
    rc = lib().sbb_mm_load(os.fsencode(os.fspath(path)), float(pattern_value), C.byref(h),
                           C.byref(m), C.byref(n), C.byref(nnz))
    if rc != 0:
        raise MatrixMarketError(last_error())
    try:
        rowptr = np.empty(m.value + 1, np.int64)
        col = np.empty(nnz.value, np.int32)
        val = np.empty(nnz.value, np.float64)
        rc = lib().sbb_mm_copy(h, rowptr.ctypes.data_as(C.c_void_p),
                               col.ctypes.data_as(C.c_void_p), val.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise MatrixMarketError(last_error())
    finally:
        lib().sbb_mm_free(h)
    return Csr(m.value, n.value, rowptr, col, val, os.path.basename(os.fspath(path)))


def write(path, A: Csr, symmetry: str = "general", comment: str = "") -> None:
    """Writes A as a real coordinate file (1-based, one entry per line, in
    row order).  symmetry="symmetric" writes the lower triangle only (A must
    be symmetric)."""
    rows = np.repeat(np.arange(A.m, dtype=np.int64), np.diff(A.rowptr))
    cols = A.col.astype(np.int64)
    vals = A.val
    if symmetry == "symmetric":
        keep = cols <= rows
        rows, cols, vals = rows[keep], cols[keep], vals[keep]
    elif symmetry != "general":
        raise ValueError("symmetry must be 'general' or 'symmetric'")
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real {symmetry}\n")
        for line in comment.splitlines():
            f.write(f"% {line}\n")
        f.write(f"{A.m} {A.n} {len(vals)}\n")
        for r, c, v in zip((rows + 1).tolist(), (cols + 1).tolist(), vals.tolist()):
            f.write(f"{r} {c} {v!r}\n")
