"""CPU: the C-ABI library loads and exports every symbol include/*.h declares.

No compute call is made here (there is no GPU); only the host-only helpers
(get_row_from_index, get_time) are called.
"""
import ctypes as C
import glob
import os
import re

import numpy as np

from helpers import golden_grfi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w ]*?[\s\*]+([A-Za-z_]\w*)\s*\(", text,
                             flags=re.M):
            if m.group(1) not in ("if", "while", "return", "sizeof"):
                names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    from sbb._lib import LIB_PATH, SIGNATURES
    lib = C.CDLL(LIB_PATH)
    names = declared_functions()
    assert {"spMV_mgpu_baseline", "spMV_mgpu_v1", "spMV_mgpu_v2", "csr5_kernel",
            "get_row_from_index", "get_time", "get_gpu_availble_mem"} <= names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # the Python bindings cover the same set
    assert names <= set(SIGNATURES) | {n for n in names if n.startswith("sbb_") and hasattr(lib, n)}


def test_cxx_linkage_shims_exported():
    """The reference's header declares C++ linkage; those mangled names exist too."""
    from sbb._lib import LIB_PATH
    lib = C.CDLL(LIB_PATH)
    for mangled in ("_Z18spMV_mgpu_baselineiixPdS_PxPiS_S_S_i",
                    "_Z12spMV_mgpu_v1iixPdS_PxPiS_S_S_ii",
                    "_Z12spMV_mgpu_v2iixPdS_PxPiS_S_S_iixi",
                    "_Z11csr5_kerneliiiPdS_PiS0_S_S_S_",
                    "_Z18get_row_from_indexiPxx", "_Z8get_timev", "_Z20get_gpu_availble_memi"):
        assert hasattr(lib, mangled), mangled


def test_get_row_from_index_matches_reference_answers():
    from sbb import api
    n = 0
    for m, rp, idx, row in golden_grfi():
        assert api.get_row_from_index(m, rp, idx) == row
        n += 1
    assert n > 500


def test_get_time_is_seconds():
    from sbb import api
    t0 = api.get_time()
    t1 = api.get_time()
    assert 1.5e9 < t0 <= t1 < 1e11


def test_bad_arguments_rejected_before_any_device_work():
    """Argument checks are host-side: they return -1 without touching a GPU."""
    from sbb import api
    rp = np.array([0, 1], np.int64)
    col = np.zeros(1, np.int32)
    val = np.ones(1)
    x = np.ones(1)
    y = np.zeros(1)
    assert api.spMV_mgpu_v1(1, 1, 1, 1.0, val, rp, col, x, 0.0, y, ngpu=0, kernel=1) == -1
    assert api.spMV_mgpu_v1(1, 1, 1, 1.0, val, rp, col, x, 0.0, y, ngpu=1, kernel=4) == -1
    assert api.spMV_mgpu_v2(1, 1, 1, 1.0, val, rp, col, x, 0.0, y, ngpu=1, kernel=1, nb=0,
                            q=1) == -1
    assert api.spMV_mgpu_v2(1, 1, 1, 1.0, val, rp, col, x, 0.0, y, ngpu=1, kernel=1, nb=1,
                            q=0) == -1
    bad_rp = np.array([0, 2], np.int64)  # rowptr[m] != nnz
    assert api.spMV_mgpu_baseline(1, 1, 1, 1.0, val, bad_rp, col, x, 0.0, y, ngpu=1) == -1


def test_nnz_beyond_int32_rejected_on_the_host():
    """One GPU takes at most 2^31 - 1 nnz, the reference's own limit (it
    casts each device's nnz to int, src/dspmv_mgpu_v1.cu:119): larger calls
    return -1 before any array is read or any device work starts."""
    from sbb import api
    rp = np.array([0, 1], np.int64)
    col = np.zeros(1, np.int32)
    val = np.ones(1)
    x = np.ones(1)
    y = np.zeros(1)
    for nnz in (2 ** 31, 2 ** 40):
        assert api.spMV_mgpu_baseline(1, 1, nnz, 1.0, val, rp, col, x, 0.0, y, ngpu=1) == -1
        for k in (1, 2, 3):
            assert api.spMV_mgpu_v1(1, 1, nnz, 1.0, val, rp, col, x, 0.0, y, ngpu=1,
                                    kernel=k) == -1
            assert api.spMV_mgpu_v2(1, 1, nnz, 1.0, val, rp, col, x, 0.0, y, ngpu=1, kernel=k,
                                    nb=1 << 20, q=1) == -1
    assert np.array_equal(y, np.zeros(1))


def test_overlapping_x_and_y_rejected_on_the_host():
    """x must not overlap y (the kernels read x while they write y): the
    no-allocation entry point and batch creation refuse such calls before any
    device work (the pointers here are never dereferenced)."""
    import ctypes as C
    from sbb._lib import BatchItem, last_error, lib
    base = 1 << 32
    p = lambda off: C.c_void_p(base + off)  # noqa: E731
    m, n = 100, 100
    # y starts inside x
    rc = lib().sbb_spmv_merge_noalloc(m, n, 10, p(0), p(1 << 20), p(2 << 20), 1.0, p(0), 0.0,
                                      p(8 * 50), None)
    assert rc == -1 and "overlap" in last_error()

    def items(*specs):
        arr = (BatchItem * len(specs))()
        for it, (xo, yo) in zip(arr, specs):
            it.m, it.n, it.nnz = m, n, 10
            it.rowptr, it.col, it.val = base + (3 << 20), base + (4 << 20), base + (5 << 20)
            it.x, it.y = base + xo, base + yo
            it.alpha, it.beta, it.cls = 1.0, 0.0, 0
        return arr

    h = C.c_void_p()
    # two y arrays overlapping
    arr = items((0, 8 << 20), (1 << 16, (8 << 20) + 8 * 99))
    assert lib().sbb_batch_create(C.byref(h), arr, 2, None) == -1
    assert "y arrays overlap" in last_error()
    # item 1's x overlapping item 0's y (a shared x is allowed)
    arr = items((0, 8 << 20), ((8 << 20) + 8 * 10, 9 << 20), (0, 10 << 20))
    assert lib().sbb_batch_create(C.byref(h), arr, 3, None) == -1
    assert "item 1's x overlaps" in last_error()


def test_batch_and_tuner_reject_bad_arguments_on_the_host():
    from sbb._lib import lib
    assert lib().sbb_batch_create(None, None, 0, None) == -1
    h = C.c_void_p()
    assert lib().sbb_batch_create(C.byref(h), None, -1, None) == -1
    assert lib().sbb_tune_classes(1, 1, 1, None, None, None, None, None, 1.0, 0.0, 3, None,
                                  None) == -1
    assert lib().sbb_batch_run(None, None) == -1
    assert lib().sbb_batch_destroy(None) == 0


def test_test_hook_selectors():
    """sbb_test_hook is host-only: it arms and disarms without a GPU and
    refuses an unknown selector."""
    from sbb._lib import TEST_FAIL_ALLOC, TEST_RESET, TEST_WAIT_BUDGET, lib
    L = lib()
    assert L.sbb_test_hook(99, 0) == -1
    assert L.sbb_test_hook(TEST_FAIL_ALLOC, -1) == -1
    assert L.sbb_test_hook(TEST_WAIT_BUDGET, 0) == 0
    assert L.sbb_test_hook(TEST_RESET, 0) == 0
