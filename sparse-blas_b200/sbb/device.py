"""Device API over torch CUDA tensors: plans built once, SpMV launched many times.

torch is used only for device memory and streams; every launch goes through
libsbb.so.
"""
from __future__ import annotations

import ctypes as C

from ._lib import Config, PlanInfo, last_error, lib

KERNELS = {"auto": 0, "vector": 1, "merge": 2, "tiled": 3, "learned": 4, "rows": 5}


class SbbError(RuntimeError):
    pass


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _stream(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class Plan:
    """A reusable SpMV plan for one CSR matrix resident on the GPU.

    rowptr/col are int32 CUDA tensors, val float64 (or float32 with f32=True).
    f32_lanes=True (with f32=True) builds the FP32-storage form whose lane
    runs of at most 8 products are summed in FP32 (sbb_plan_create_f32_lanes;
    tiled kernel only).  The tensors are kept alive by the plan.
    """

    def __init__(self, rowptr, col, val, n, kernel="auto", vector_width=0,
                 items_per_thread=0, persistent=0, tile_sigma=0, f32=False, stream=None,
                 f32_lanes=False):
        import torch
        assert rowptr.dtype == torch.int32 and col.dtype == torch.int32
        assert val.dtype == (torch.float32 if f32 else torch.float64)
        self.m = rowptr.numel() - 1
        self.n = int(n)
        self.nnz = col.numel()
        self.f32 = f32
        self._keep = (rowptr, col, val)
        cfg = Config(KERNELS[kernel] if isinstance(kernel, str) else int(kernel),
                     vector_width, items_per_thread, persistent, tile_sigma)
        h = C.c_void_p()
        assert f32 or not f32_lanes
        create = (lib().sbb_plan_create_f32_lanes if f32_lanes else
                  lib().sbb_plan_create_f32 if f32 else lib().sbb_plan_create)
        rc = create(C.byref(h), self.m, self.n, self.nnz, _ptr(rowptr), _ptr(col), _ptr(val),
                    C.byref(cfg), _stream(stream))
        if rc != 0:
            raise SbbError(f"sbb_plan_create failed ({rc}): {last_error()}")
        self.h = h

    def spmv(self, x, y, alpha=1.0, beta=0.0, stream=None):
        f = lib().sbb_spmv_f32 if self.f32 else lib().sbb_spmv
        rc = f(self.h, float(alpha), _ptr(x), float(beta), _ptr(y), _stream(stream))
        if rc != 0:
            raise SbbError(f"sbb_spmv failed ({rc}): {last_error()}")

    def check(self):
        rc = lib().sbb_plan_check(self.h)
        if rc != 0:
            raise SbbError(f"device check failed ({rc}): {last_error()}")

    def info(self):
        i = PlanInfo()
        lib().sbb_plan_info_get(self.h, C.byref(i))
        return {f: getattr(i, f) for f, _ in PlanInfo._fields_}

    def partition(self):
        import numpy as np
        info = self.info()
        cnt = info["tiles"] + 1
        rows = np.empty(cnt, np.int32)
        nzs = np.empty(cnt, np.int32)
        rc = lib().sbb_plan_partition(self.h, rows.ctypes.data_as(C.c_void_p),
                                      nzs.ctypes.data_as(C.c_void_p), cnt)
        if rc < 0:
            raise SbbError(last_error())
        return rows, nzs

    def close(self):
        if getattr(self, "h", None):
            lib().sbb_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
