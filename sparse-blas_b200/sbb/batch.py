"""Batched SpMV (one persistent launch for many matrices) and the autotuner.

Classes (``include/sbb_spmv.h``, SBB_NUM_CLASSES = 6): 0..3 vector CSR with
4, 8, 16, 32 lanes per row, 4 merge path (6 items per lane), 5 CSR5-style
tiles of 32 x 4 nnz.  Every class computes the same SpMV; the tuner times all
six on a matrix as plain launches and keeps the fastest.
"""
from __future__ import annotations

import ctypes as C

from ._lib import BatchItem, last_error, lib

NUM_CLASSES = 6
CLASS_NAMES = ["vector4", "vector8", "vector16", "vector32", "merge6", "tiled4"]


class BatchError(RuntimeError):
    pass


def _stream(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class Batch:
    """mats: list of dicts with torch CUDA tensors rowptr (int32), col (int32),
    val (float64), x, y (float64), ints m, n and floats alpha, beta; classes:
    one class per matrix.  The tensors must outlive the batch (it keeps a
    reference to the list)."""

    def __init__(self, mats, classes, stream=None):
        assert len(mats) == len(classes)
        self._keep = mats
        arr = (BatchItem * max(len(mats), 1))()
        for i, (d, c) in enumerate(zip(mats, classes)):
            arr[i] = BatchItem(d["m"], d["n"], d["col"].numel(), d["rowptr"].data_ptr(),
                               d["col"].data_ptr(), d["val"].data_ptr(), d["x"].data_ptr(),
                               d["y"].data_ptr(), float(d.get("alpha", 1.0)),
                               float(d.get("beta", 0.0)), int(c))
        h = C.c_void_p()
        rc = lib().sbb_batch_create(C.byref(h), arr, len(mats), _stream(stream))
        if rc != 0:
            raise BatchError(f"sbb_batch_create failed ({rc}): {last_error()}")
        self.h = h

    def run(self, stream=None):
        self._ok(lib().sbb_batch_run(self.h, _stream(stream)))

    def run_graph(self, stream=None):
        self._ok(lib().sbb_batch_run_graph(self.h, _stream(stream)))

    def run_each(self, stream=None):
        self._ok(lib().sbb_batch_run_each(self.h, _stream(stream)))

    def launches(self, per_matrix=False):
        return lib().sbb_batch_launches(self.h, 1 if per_matrix else 0)

    def check(self):
        self._ok(lib().sbb_batch_check(self.h))

    def _ok(self, rc):
        if rc != 0:
            raise BatchError(f"batch call failed ({rc}): {last_error()}")

    def close(self):
        if getattr(self, "h", None):
            lib().sbb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tune(d, reps=5, stream=None):
    """Mean ms of each class on matrix d (dict as in Batch); d['y'] is overwritten."""
    ms = (C.c_float * NUM_CLASSES)()
    rc = lib().sbb_tune_classes(d["m"], d["n"], d["col"].numel(), C.c_void_p(d["rowptr"].data_ptr()),
                                C.c_void_p(d["col"].data_ptr()), C.c_void_p(d["val"].data_ptr()),
                                C.c_void_p(d["x"].data_ptr()), C.c_void_p(d["y"].data_ptr()),
                                float(d.get("alpha", 1.0)), float(d.get("beta", 0.0)), reps, ms,
                                _stream(stream))
    if rc != 0:
        raise BatchError(f"sbb_tune_classes failed ({rc}): {last_error()}")
    return [float(v) for v in ms]
