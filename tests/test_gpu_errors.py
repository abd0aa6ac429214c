"""GPU: the error paths of the reference's contract, made to happen on the host.

The reference returns 1 when a device allocation fails
(SparseBLAS/src/dspmv_mgpu_baseline.cu:99-135) and -1 when its memory
pre-check (0.8 x free memory, SparseBLAS/src/dspmv_mgpu_v1.cu:104-116) or a
kernel fails.  On a healthy B200 with test-sized inputs none of that happens,
so these tests arm the library's test hooks (sbb_test_hook): a failing
allocation, a shrunken free-memory figure, and a zero poll budget for the
first tile-copy wait of the tiled kernel, which then takes its timeout path
(lets its copies land, raises the timeout status, stops).  No GPU is faulted:
every failure is a host-side decision or a bounded wait giving up.  After
each injected failure the hooks are disarmed and the same call must succeed
with the oracle's result, so no failure leaves state behind.
"""
import numpy as np
import pytest

import oracle as O
from helpers import TOL_FP64, max_scaled_err, rand_csr

pytestmark = pytest.mark.gpu


@pytest.fixture
def hooks(cuda):
    from sbb._lib import TEST_RESET, lib
    L = lib()
    L.sbb_test_hook(TEST_RESET, 0)
    yield L
    L.sbb_test_hook(TEST_RESET, 0)


def _case(seed=41, m=20000, n=18000, lmax=24):
    rp, col, val, x, y = rand_csr(seed, m, n, 0, lmax, p_empty=0.05)
    return rp, col, val, x, y


def _call(version, rp, col, val, x, y, alpha=1.5, beta=-0.5, kernel=2):
    from sbb import api
    m, n, nnz = len(rp) - 1, len(x), int(rp[-1])
    yy = y.copy()
    if version == "baseline":
        rc = api.spMV_mgpu_baseline(m, n, nnz, alpha, val, rp, col, x, beta, yy, 1)
    elif version == "v1":
        rc = api.spMV_mgpu_v1(m, n, nnz, alpha, val, rp, col, x, beta, yy, 1, kernel)
    else:
        rc = api.spMV_mgpu_v2(m, n, nnz, alpha, val, rp, col, x, beta, yy, 1, kernel, 4096, 2)
    return rc, yy


def _check_ok(version, rp, col, val, x, y, kernel=2):
    rc, yy = _call(version, rp, col, val, x, y, kernel=kernel)
    assert rc == 0
    m, n, nnz = len(rp) - 1, len(x), int(rp[-1])
    # kernel 3 honours alpha and beta here (the reference's CSR5 drops them),
    # so its expected result is that of the other kernels on the same split
    rc_o, y_o = O.dropin(version, m, n, nnz, 1.5, val, rp, col, x, -0.5, y, ngpu=1,
                         kernel=2 if kernel == 3 else kernel, nb=4096, q=2)
    assert rc_o == 0
    _, scale = O.spmv_dd(rp, col, val, x, 1.5, -0.5, y)
    assert max_scaled_err(yy, y_o, scale) <= TOL_FP64


@pytest.mark.parametrize("version", ["baseline", "v1", "v2"])
@pytest.mark.parametrize("k", [1, 2, 4, 7, 9])
def test_allocation_failure_returns_1(hooks, version, k):
    """The k-th device allocation of the call fails: the call returns 1 (the
    reference's code for a failed cudaMalloc) with y untouched, and the next
    call, with the hook disarmed, is correct."""
    from sbb._lib import TEST_FAIL_ALLOC, TEST_RESET
    rp, col, val, x, y = _case()
    assert hooks.sbb_test_hook(TEST_FAIL_ALLOC, k) == 0
    rc, yy = _call(version, rp, col, val, x, y)
    hooks.sbb_test_hook(TEST_RESET, 0)
    if rc == 0:
        # the call made fewer than k allocations: nothing failed, result right
        pytest.skip(f"{version} makes fewer than {k} allocations")
    assert rc == 1, rc
    assert np.array_equal(yy, y)
    _check_ok(version, rp, col, val, x, y)


def test_allocation_failure_in_plan_build_returns_nomem(hooks):
    """The device API: a failing allocation while a plan is built gives
    SBB_ERR_NOMEM, for each kernel's plan."""
    import torch
    from sbb._lib import TEST_FAIL_ALLOC, TEST_RESET
    from sbb.device import Plan, SbbError
    rp, col, val, x, y = _case()
    d = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0", dt)  # noqa: E731
    drp, dcol, dval = d(rp.astype(np.int32)), d(col), d(val)
    for kernel in ("merge", "tiled"):
        hooks.sbb_test_hook(TEST_FAIL_ALLOC, 2)
        with pytest.raises(SbbError, match=r"\(-4\)"):
            Plan(drp, dcol, dval, len(x), kernel=kernel)
        hooks.sbb_test_hook(TEST_RESET, 0)
        P = Plan(drp, dcol, dval, len(x), kernel=kernel)
        yd = d(y)
        P.spmv(d(x), yd, 1.5, -0.5)
        torch.cuda.synchronize()
        P.check()
        P.close()
        y_ref, scale = O.spmv_dd(rp, col, val, x, 1.5, -0.5, y)
        assert max_scaled_err(yd.cpu().numpy(), y_ref, scale) <= TOL_FP64


@pytest.mark.parametrize("version", ["baseline", "v1", "v2"])
def test_memory_precheck_returns_minus_1(hooks, version):
    """With the free memory the pre-check sees shrunk below what the call
    needs, the call returns -1 before touching the device or y."""
    from sbb._lib import TEST_FREE_BYTES, TEST_RESET
    rp, col, val, x, y = _case()
    assert hooks.sbb_test_hook(TEST_FREE_BYTES, 4096) == 0
    rc, yy = _call(version, rp, col, val, x, y)
    hooks.sbb_test_hook(TEST_RESET, 0)
    assert rc == -1, rc
    assert np.array_equal(yy, y)
    _check_ok(version, rp, col, val, x, y)


@pytest.mark.parametrize("form", ["fp64", "f32", "f32_lanes"])
def test_tiled_wait_timeout_reports_status(hooks, form):
    """A zero poll budget for the first tile-copy wait of the first warp: the
    kernel gives up that wait, lets its copies in flight land, raises the
    timeout status and stops; sbb_plan_check reports SBB_ERR_INPUT with the
    timeout message, and the context stays usable.  fp64: 32 x 4 tiles, a
    two-tile ring; f32 / f32_lanes: the FP32-storage 32 x 8 tiles, a
    three-tile ring with the x gathers one tile ahead."""
    import torch
    from helpers import TOL_FP32
    from sbb._lib import TEST_RESET, TEST_WAIT_BUDGET
    from sbb.device import Plan, SbbError
    rp, col, val, x, y = _case(seed=42, m=60000, n=50000, lmax=40)
    d = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0", dt)  # noqa: E731
    f32 = form != "fp64"
    drp, dcol = d(rp.astype(np.int32)), d(col)
    dval = d(val.astype(np.float32)) if f32 else d(val)
    dx = d(x.astype(np.float32)) if f32 else d(x)
    kw = dict(kernel="tiled", tile_sigma=8 if f32 else 4, f32=f32,
              f32_lanes=form == "f32_lanes")
    P = Plan(drp, dcol, dval, len(x), **kw)
    assert hooks.sbb_test_hook(TEST_WAIT_BUDGET, 0) == 0
    yd = d(y)
    P.spmv(dx, yd, 1.5, -0.5)
    torch.cuda.synchronize()
    hooks.sbb_test_hook(TEST_RESET, 0)
    with pytest.raises(SbbError, match="bounded wait"):
        P.check()
    P.close()
    # a fresh plan on the same context computes the right result
    P = Plan(drp, dcol, dval, len(x), **kw)
    yd = d(y)
    P.spmv(dx, yd, 1.5, -0.5)
    torch.cuda.synchronize()
    P.check()
    P.close()
    y_ref, scale = O.spmv_dd(rp, col, val, x, 1.5, -0.5, y)
    assert max_scaled_err(yd.cpu().numpy(), y_ref, scale) <= (TOL_FP32 if f32 else TOL_FP64)


def test_dropin_kernel3_timeout_returns_minus_1(hooks):
    """The same timeout through spMV_mgpu_v1 with kernel 3: -1, then a clean
    call gives the reference's result."""
    from sbb._lib import TEST_RESET, TEST_WAIT_BUDGET
    rp, col, val, x, y = _case(seed=43, m=60000, n=50000, lmax=40)
    assert hooks.sbb_test_hook(TEST_WAIT_BUDGET, 0) == 0
    rc, _ = _call("v1", rp, col, val, x, y, kernel=3)
    hooks.sbb_test_hook(TEST_RESET, 0)
    assert rc == -1, rc
    _check_ok("v1", rp, col, val, x, y, kernel=3)
