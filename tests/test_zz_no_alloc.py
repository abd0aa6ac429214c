"""GPU: the entry point for callers that cannot allocate device memory.

sbb_spmv_merge_noalloc runs the merge-path SpMV with its scratch in a fixed
__device__ array of the library instead of cudaMalloc'ed buffers, for code
that must not call the device allocator (memory-capped processes, callbacks,
frameworks that own all device memory).  It is checked here, through the
C ABI, against the accurate CPU oracle and against the existing plan-based
entry point (sbb_spmv with a merge-path plan), within the FP64 tolerance the
other tests use, on two calls in a row, because the shared scratch keeps the
previous call's contents.  A second test checks the one property the entry
point exists for: after a warm-up call, further calls change neither the
device's free memory nor the use of the default stream-ordered memory pool.
This file is collected last so a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from helpers import TOL_FP64, max_scaled_err, rand_csr

pytestmark = pytest.mark.gpu


def _dev(a, torch, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0", dtype)


def _noalloc(L, m, n, nnz, rp, col, val, x, y, alpha, beta):
    return L.sbb_spmv_merge_noalloc(m, n, nnz, C.c_void_p(rp.data_ptr()), C.c_void_p(col.data_ptr()),
                                    C.c_void_p(val.data_ptr()), alpha, C.c_void_p(x.data_ptr()),
                                    beta, C.c_void_p(y.data_ptr()), None)


@pytest.mark.parametrize("case", ["uniform", "empty_rows", "long_rows", "c1", "beta0",
                                  "empty_tail"])
def test_noalloc_matches_oracle_and_plan_entry_point(cuda, case):
    import torch
    from sbb import gen
    from sbb._lib import lib, last_error
    from sbb.device import Plan
    if case == "c1":
        A = gen.c1()
        rp, col, val = A.rowptr, A.col, A.val
        x, y = gen.uniform_vec(11, A.n), gen.uniform_vec(12, A.m)
    elif case == "uniform":
        rp, col, val, x, y = rand_csr(31, 20000, 15000, 0, 30)
    elif case == "empty_rows":
        rp, col, val, x, y = rand_csr(32, 9000, 7000, 0, 12, p_empty=0.5)
    elif case == "long_rows":
        rp, col, val, x, y = rand_csr(33, 3000, 300000, 0, 8,
                                      long_rows=[(0, 200000), (1500, 60000), (2999, 5000)])
    elif case == "beta0":
        rp, col, val, x, y = rand_csr(34, 12000, 9000, 0, 20, p_empty=0.1)
    else:  # the last 700 rows empty: the final segments cover rows without nnz
        rp, col, val, x, y = rand_csr(35, 6000, 5000, 1, 16)
        nz_keep = int(rp[5300])
        rp = np.concatenate([rp[:5301], np.full(700, nz_keep, rp.dtype)])
        col, val = col[:nz_keep], val[:nz_keep]
    m, n, nnz = len(rp) - 1, len(x), int(rp[-1])
    alpha, beta = 1.25, (0.0 if case == "beta0" else -0.5)
    drp, dcol, dval, dx = _dev(rp.astype(np.int32), torch), _dev(col, torch), _dev(val, torch), _dev(x, torch)
    y0 = _dev(y, torch)

    P = Plan(drp, dcol, dval, n, kernel="merge", items_per_thread=12)
    y_plan = y0.clone()
    P.spmv(dx, y_plan, alpha, beta)
    torch.cuda.synchronize()
    P.check()
    P.close()
    y_plan = y_plan.cpu().numpy()
    y_ref, scale = O.spmv_dd(rp, col, val, x, alpha, beta, y)

    L = lib()
    for call in range(2):  # two calls in a row share (and reuse) the scratch
        y_na = y0.clone()
        rc = _noalloc(L, m, n, nnz, drp, dcol, dval, dx, y_na, alpha, beta)
        assert rc == 0, last_error()
        torch.cuda.synchronize()
        y_na = y_na.cpu().numpy()
        err = max_scaled_err(y_na, y_ref, scale)
        assert err <= TOL_FP64, (call, "vs oracle", err)
        err = max_scaled_err(y_na, y_plan, scale)
        assert err <= TOL_FP64, (call, "vs plan entry point", err)


def _pool_bytes(driver):
    """(used, reserved) bytes of device 0's default stream-ordered memory pool."""
    err, pool = driver.cuDeviceGetDefaultMemPool(0)
    assert err == driver.CUresult.CUDA_SUCCESS, err
    out = []
    for attr in (driver.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                 driver.CUmemPool_attribute.CU_MEMPOOL_ATTR_RESERVED_MEM_HIGH,
                 driver.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_CURRENT,
                 driver.CUmemPool_attribute.CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT):
        err, v = driver.cuMemPoolGetAttribute(pool, attr)
        assert err == driver.CUresult.CUDA_SUCCESS, err
        out.append(int(v))
    return pool, out


def test_noalloc_calls_allocate_nothing(cuda):
    """Neither cudaMalloc (device free memory) nor the stream-ordered pool
    (its use and reservation, including their high-water marks, reset just
    before the calls) moves while the entry point runs."""
    import torch
    from cuda.bindings import driver
    from sbb._lib import lib, last_error
    rp, col, val, x, y = rand_csr(36, 50000, 40000, 0, 24, p_empty=0.05)
    m, n, nnz = len(rp) - 1, len(x), int(rp[-1])
    drp, dcol, dval, dx = _dev(rp.astype(np.int32), torch), _dev(col, torch), _dev(val, torch), _dev(x, torch)
    ys = [_dev(y, torch) for _ in range(4)]  # every tensor exists before the measured calls
    L = lib()
    assert _noalloc(L, m, n, nnz, drp, dcol, dval, dx, ys[0], 1.0, 0.5) == 0, last_error()
    torch.cuda.synchronize()  # warm-up: modules loaded, scratch address looked up
    assert driver.cuInit(0)[0] == driver.CUresult.CUDA_SUCCESS
    pool, _ = _pool_bytes(driver)
    for attr in (driver.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                 driver.CUmemPool_attribute.CU_MEMPOOL_ATTR_RESERVED_MEM_HIGH):
        err, = driver.cuMemPoolSetAttribute(pool, attr, driver.cuuint64_t(0))
        assert err == driver.CUresult.CUDA_SUCCESS, err
    _, before = _pool_bytes(driver)
    free_before = torch.cuda.mem_get_info(0)[0]
    for i in range(1, 4):
        rc = _noalloc(L, m, n, nnz, drp, dcol, dval, dx, ys[i], 1.0, 0.5)
        assert rc == 0, last_error()
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info(0)[0]
    _, after = _pool_bytes(driver)
    assert free_after == free_before, (free_before, free_after)
    assert after == before, (before, after)
    for i in range(1, 4):  # and the calls did their work
        assert torch.equal(ys[i], ys[0])


def test_noalloc_rejects_inputs_beyond_its_capacity(cuda):
    import torch
    from sbb._lib import lib, last_error
    L = lib()
    small = torch.zeros(8, dtype=torch.int32, device="cuda:0")
    vals = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    # m + nnz above the fixed scratch capacity is refused on the host,
    # before any device work
    rc = L.sbb_spmv_merge_noalloc(60_000_000, 10, 60_000_000, C.c_void_p(small.data_ptr()),
                                  C.c_void_p(small.data_ptr()), C.c_void_p(vals.data_ptr()), 1.0,
                                  C.c_void_p(vals.data_ptr()), 0.0, C.c_void_p(vals.data_ptr()), None)
    assert rc == -1
    assert "capacity" in last_error()
