"""cuSPARSE SpMV as a runtime comparator for the GPU tests (test code only).

The reference's kernels 1 and 2 call the legacy ``cusparseDcsrmv`` and
``cusparseDcsrmv_mp`` (SparseBLAS src/dspmv_mgpu_baseline.cu:163-167,
src/dspmv_mgpu_v1.cu:200-210, src/dspmv_mgpu_v2.cu:351-361), which cuSPARSE
dropped in CUDA 11.  Their successor is the generic ``cusparseSpMV``: ``CUSPARSE_SPMV_CSR_ALG1`` (row
based, deterministic) stands in for csrmv and ``CUSPARSE_SPMV_CSR_ALG2``
(load-balanced by nnz) for csrmv_mp.  The library's results are only compared
with; nothing in the product calls it.

Bound through ctypes on device pointers of torch CUDA tensors; the handle is
the one loaded with torch (libcusparse.so.12).
"""
from __future__ import annotations

import ctypes as C
import glob
import os

# cusparse.h / library_types.h enumerators used here
_OP_N = 0
_BASE_ZERO = 0
_INDEX_32I, _INDEX_64I = 2, 3
_R_32F, _R_64F = 0, 1
ALGS = {"alg1": 2, "alg2": 3, "default": 0}

_lib = None
_handle = None


def _load():
    global _lib
    if _lib is not None:
        return _lib
    import torch  # loads torch's CUDA libraries, cuSPARSE among them
    names = ["libcusparse.so.12"]
    names += glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cusparse",
                                    "lib", "libcusparse.so.12"))
    names += ["/usr/local/cuda/lib64/libcusparse.so.12"]
    err = None
    for nm in names:
        try:
            _lib = C.CDLL(nm)
            break
        except OSError as e:
            err = e
    if _lib is None:
        raise OSError(f"libcusparse not found: {err}")
    vp, i64 = C.c_void_p, C.c_int64
    sig = {
        "cusparseCreate": [C.POINTER(vp)],
        "cusparseSetStream": [vp, vp],
        "cusparseCreateCsr": [C.POINTER(vp), i64, i64, i64, vp, vp, vp, C.c_int, C.c_int, C.c_int,
                              C.c_int],
        "cusparseCreateDnVec": [C.POINTER(vp), i64, vp, C.c_int],
        "cusparseSpMV_bufferSize": [vp, C.c_int, vp, vp, vp, vp, vp, C.c_int, C.c_int,
                                    C.POINTER(C.c_size_t)],
        "cusparseSpMV": [vp, C.c_int, vp, vp, vp, vp, vp, C.c_int, C.c_int, vp],
        "cusparseDestroySpMat": [vp],
        "cusparseDestroyDnVec": [vp],
    }
    for name, args in sig.items():
        f = getattr(_lib, name)
        f.argtypes = args
        f.restype = C.c_int
    return _lib


def available():
    try:
        _load()
        return True
    except OSError:
        return False


def _ok(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} returned cuSPARSE status {rc}")


def _get_handle():
    global _handle
    lib = _load()
    if _handle is None:
        h = C.c_void_p()
        _ok(lib.cusparseCreate(C.byref(h)), "cusparseCreate")
        _handle = h
    return _handle


class SpMV:
    """y = alpha*A*x + beta*y by cusparseSpMV on CUDA tensors.

    rowptr, col: int32 (or both int64) [m+1], [nnz]; val: float64 or float32
    [nnz]; the vectors x and y have val's type.  Descriptors and the work
    buffer are made once, so ``run`` can be timed."""

    def __init__(self, m, n, rowptr, col, val, x, y, alg="alg1", stream=None):
        import torch
        lib = _load()
        self.lib, self.h = lib, _get_handle()
        self.keep = (rowptr, col, val, x, y)
        self.dt = _R_64F if val.dtype == torch.float64 else _R_32F
        ctype = C.c_double if self.dt == _R_64F else C.c_float
        self.alg = ALGS[alg]
        self.stream = stream or torch.cuda.current_stream()
        self.A, self.X, self.Y = C.c_void_p(), C.c_void_p(), C.c_void_p()
        if rowptr.dtype != col.dtype:  # cuSPARSE takes one index width for both
            raise ValueError("row offsets and column indices must have the same integer type")
        rp_t = _INDEX_64I if rowptr.dtype == torch.int64 else _INDEX_32I
        _ok(lib.cusparseCreateCsr(C.byref(self.A), m, n, col.numel(), C.c_void_p(rowptr.data_ptr()),
                                  C.c_void_p(col.data_ptr()), C.c_void_p(val.data_ptr()), rp_t,
                                  _INDEX_32I, _BASE_ZERO, self.dt), "cusparseCreateCsr")
        _ok(lib.cusparseCreateDnVec(C.byref(self.X), n, C.c_void_p(x.data_ptr()), self.dt),
            "cusparseCreateDnVec")
        _ok(lib.cusparseCreateDnVec(C.byref(self.Y), m, C.c_void_p(y.data_ptr()), self.dt),
            "cusparseCreateDnVec")
        self._ctype = ctype
        a, b = ctype(1.0), ctype(0.0)
        size = C.c_size_t(0)
        _ok(lib.cusparseSpMV_bufferSize(self.h, _OP_N, C.byref(a), self.A, self.X, C.byref(b),
                                        self.Y, self.dt, self.alg, C.byref(size)),
            "cusparseSpMV_bufferSize")
        self.buf = torch.empty(max(int(size.value), 16), dtype=torch.uint8, device=val.device)

    def run(self, alpha, beta):
        lib = self.lib
        _ok(lib.cusparseSetStream(self.h, C.c_void_p(self.stream.cuda_stream)), "cusparseSetStream")
        a, b = self._ctype(alpha), self._ctype(beta)
        _ok(lib.cusparseSpMV(self.h, _OP_N, C.byref(a), self.A, self.X, C.byref(b), self.Y,
                             self.dt, self.alg, C.c_void_p(self.buf.data_ptr())), "cusparseSpMV")

    def close(self):
        if self.A:
            self.lib.cusparseDestroySpMat(self.A)
            self.lib.cusparseDestroyDnVec(self.X)
            self.lib.cusparseDestroyDnVec(self.Y)
            self.A = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def spmv(m, n, rowptr, col, val, x, y, alpha, beta, alg="alg1"):
    """One cusparseSpMV into y (in place) on the current stream."""
    op = SpMV(m, n, rowptr, col, val, x, y, alg)
    op.run(alpha, beta)
    import torch
    torch.cuda.current_stream().synchronize()
    op.close()
    return y
