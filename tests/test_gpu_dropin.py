"""GPU: the drop-in entry points against the reference's own outputs.

Golden fixtures hold the reference drivers' results (tests/golden).  The GPU
sums in a different order than the reference's csrmv, so FP values are
compared per row within TOL_FP64 of |alpha|*sum|a_ij x_j| + |beta*y_i|
(the error metric); return codes and which rows are written must match
exactly.  The GPU count is pinned to 1, so fixtures made with ngpu > 1 are
compared with the oracle's ngpu = 1 result.  Kernel 3: the reference's CSR5
drops alpha and beta; this library honours them, so kernel-3 fixtures are
compared with the reference where alpha = 1, beta = 0 and with the oracle's
kernel-1 semantics elsewhere.
"""
import numpy as np
import pytest

import oracle as O
from helpers import TOL_FP64, golden_cases, max_scaled_err, rand_csr

pytestmark = pytest.mark.gpu

CASES = golden_cases()


def _scale(c, rowptr=None):
    rp = c["rowptr"] if rowptr is None else rowptr
    _, sc = O.spmv_dd(rp, c["col"], c["val"], c["x"], c["alpha"], c["beta"], c["y"])
    return sc


def _call(api, c, kernel=None, ngpu=None):
    y = c["y"].copy()
    args = (c["m"], c["n"], c["nnz"], c["alpha"], c["val"], c["rowptr"], c["col"], c["x"],
            c["beta"], y)
    ng = c["ngpu"] if ngpu is None else ngpu
    k = c["kernel"] if kernel is None else kernel
    if c["version"] == "baseline":
        rc = api.spMV_mgpu_baseline(*args, ngpu=ng)
    elif c["version"] == "v1":
        rc = api.spMV_mgpu_v1(*args, ngpu=ng, kernel=k)
    else:
        rc = api.spMV_mgpu_v2(*args, ngpu=ng, kernel=k, nb=c["nb"], q=c["q"])
    return rc, y


def _expected(c):
    """The reference's result for this call on one GPU, with this library's kernel-3 semantics."""
    if c["ngpu"] == 1 and (c["kernel"] != 3 or (c["alpha"] == 1.0 and c["beta"] == 0.0)):
        return c["rc"], c["y_ref"]
    k = 1 if c["kernel"] == 3 else c["kernel"]
    return O.dropin(c["version"], c["m"], c["n"], c["nnz"], c["alpha"], c["val"], c["rowptr"],
                    c["col"], c["x"], c["beta"], c["y"], ngpu=1, kernel=k,
                    nb=c["nb"] or None, q=c["q"])


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_dropin_matches_reference(cuda, c):
    from sbb import api
    rc_ref, y_ref = _expected(c)
    rc, y = _call(api, c)
    assert rc == rc_ref
    untouched = y_ref == c["y"]
    # rows the reference leaves alone must be left alone bit for bit
    assert np.array_equal(y[untouched & (y_ref == c["y"])], c["y"][untouched])
    err = max_scaled_err(y, y_ref, _scale(c))
    assert err <= TOL_FP64, err


@pytest.mark.parametrize("kernel", [1, 2, 3])
@pytest.mark.parametrize("version", ["v1", "v2"])
def test_dropin_random_with_empty_rows(cuda, kernel, version):
    from sbb import api
    for seed in range(4):
        m, n = 3000 + 17 * seed, 2500
        rp, col, val, x, y = rand_csr(100 + seed, m, n, 0, 40, p_empty=0.25,
                                      long_rows=[(5, 2400), (m - 3, 2000)])
        nnz = int(rp[-1])
        alpha, beta = 0.8, (0.0 if seed % 2 else -0.6)
        nb = max(1, nnz // (1 + 3 * seed)) if version == "v2" else None
        rc_ref, y_ref = O.dropin(version, m, n, nnz, alpha, val, rp, col, x, beta, y, ngpu=1,
                                 kernel=1 if kernel == 3 else kernel, nb=nb, q=2)
        yy = y.copy()
        if version == "v1":
            rc = api.spMV_mgpu_v1(m, n, nnz, alpha, val, rp, col, x, beta, yy, ngpu=4,
                                  kernel=kernel)
        else:
            rc = api.spMV_mgpu_v2(m, n, nnz, alpha, val, rp, col, x, beta, yy, ngpu=2,
                                  kernel=kernel, nb=nb, q=2)
        assert rc == rc_ref == 0
        _, sc = O.spmv_dd(rp, col, val, x, alpha, beta, y)
        assert max_scaled_err(yy, y_ref, sc) <= TOL_FP64


def _dropin_case(seed, version, kernel):
    """A drop-in call on a seeded matrix with empty and long rows, with the
    oracle driver's result and the row scale (computed here, on the calling
    thread)."""
    m, n = 2000 + 37 * seed, 1800
    rp, col, val, x, y = rand_csr(500 + seed, m, n, 0, 30, p_empty=0.2,
                                  long_rows=[(4, 1700), (m - 2, 900)])
    nnz = int(rp[-1])
    alpha, beta = 1.0 - 0.1 * seed, (0.0 if seed % 2 else 0.7)
    nb = max(1, nnz // 5) if version == "v2" else None
    rc_ref, y_ref = O.dropin(version, m, n, nnz, alpha, val, rp, col, x, beta, y, ngpu=1,
                             kernel=1 if kernel in (0, 3) else kernel, nb=nb, q=2)
    assert rc_ref == 0
    _, sc = O.spmv_dd(rp, col, val, x, alpha, beta, y)
    return dict(version=version, kernel=kernel, args=(m, n, nnz, alpha, val, rp, col, x, beta),
                y=y, nb=nb, y_ref=y_ref, sc=sc)


def _dropin_call(c):
    """Runs case c through the drop-in API; returns (rc, max scaled error)."""
    from sbb import api
    yy = c["y"].copy()
    m, n, nnz, alpha, val, rp, col, x, beta = c["args"]
    if c["version"] == "baseline":
        rc = api.spMV_mgpu_baseline(m, n, nnz, alpha, val, rp, col, x, beta, yy, ngpu=1)
    elif c["version"] == "v1":
        rc = api.spMV_mgpu_v1(m, n, nnz, alpha, val, rp, col, x, beta, yy, ngpu=1,
                              kernel=c["kernel"])
    else:
        rc = api.spMV_mgpu_v2(m, n, nnz, alpha, val, rp, col, x, beta, yy, ngpu=1,
                              kernel=c["kernel"], nb=c["nb"], q=2)
    return rc, max_scaled_err(yy, c["y_ref"], c["sc"])


CONCURRENT_CALLS = [("baseline", 0), ("v1", 1), ("v1", 2), ("v1", 3), ("v2", 1), ("v2", 2),
                    ("v2", 3)]


def test_dropin_concurrent_callers(cuda):
    """Drop-in calls from 8 host threads at once (ctypes releases the GIL,
    so the calls overlap): each thread has its own streams and status words
    and every result matches the oracle's driver."""
    from concurrent.futures import ThreadPoolExecutor
    cases = [_dropin_case(seed, v, k) for seed in range(8) for v, k in CONCURRENT_CALLS]
    with ThreadPoolExecutor(max_workers=8) as ex:
        results = list(ex.map(_dropin_call, cases * 2))
    for c, (rc, err) in zip(cases * 2, results):
        assert rc == 0 and err <= TOL_FP64, (c["version"], c["kernel"], err)


def test_dropin_short_lived_threads(cuda):
    """Threads that make one call each and end: each ends with its streams
    and pinned status words released, and 80 of them in turn keep working
    (no per-thread resources pile up to a failure)."""
    import threading
    cases = [_dropin_case(s, v, k) for s in range(2) for v, k in CONCURRENT_CALLS]
    errors = []

    def one(i):
        try:
            rc, err = _dropin_call(cases[i % len(cases)])
            if rc != 0 or err > TOL_FP64:
                errors.append((i, rc, err))
        except Exception as e:  # reported below
            errors.append((i, repr(e)))

    for wave in range(10):
        ts = [threading.Thread(target=one, args=(wave * 8 + j,)) for j in range(8)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
    assert not errors, errors


def test_dropin_rejects_bad_columns(cuda):
    from sbb import api
    rp, col, val, x, y = rand_csr(1, 50, 40, 1, 5)
    col = col.copy()
    col[7] = 40  # == n: out of range
    yy = y.copy()
    rc = api.spMV_mgpu_v1(50, 40, int(rp[-1]), 1.0, val, rp, col, x, 0.0, yy, ngpu=1, kernel=2)
    assert rc == -1


def test_dropin_rejects_non_monotone_rowptr(cuda):
    from sbb import api
    rp, col, val, x, y = rand_csr(2, 50, 40, 1, 5)
    rp = rp.copy()
    rp[10], rp[11] = rp[11], rp[10]
    if rp[10] == rp[11]:
        rp[10] += 1
    yy = y.copy()
    rc = api.spMV_mgpu_v1(50, 40, int(rp[-1]), 1.0, val, rp, col, x, 0.0, yy, ngpu=1, kernel=1)
    assert rc == -1
    assert np.array_equal(yy, y)


def test_dropin_tiny_and_empty(cuda):
    from sbb import api
    # one row, one nnz
    rp = np.array([0, 1], np.int64)
    col = np.array([0], np.int32)
    val = np.array([2.0])
    x = np.array([3.0])
    y = np.array([1.0])
    for k in (1, 2, 3):
        yy = y.copy()
        assert api.spMV_mgpu_v1(1, 1, 1, 1.0, val, rp, col, x, 0.5, yy, ngpu=1, kernel=k) == 0
        assert yy[0] == 6.5
    # nnz == 0, m == 1: the single row gets beta*y
    rp0 = np.zeros(2, np.int64)
    yy = np.array([4.0])
    assert api.spMV_mgpu_v1(1, 1, 0, 1.0, np.zeros(1), rp0, np.zeros(1, np.int32), x, 0.5, yy,
                            ngpu=1, kernel=1) == 0
    assert yy[0] == 2.0
    # nnz == 0, m >= 2: the partition covers no row (reference: no row written / abort)
    rp0 = np.zeros(6, np.int64)
    yy = np.arange(5, dtype=np.float64)
    assert api.spMV_mgpu_v1(5, 1, 0, 1.0, np.zeros(1), rp0, np.zeros(1, np.int32), x, 0.5, yy,
                            ngpu=1, kernel=2) == 0
    assert np.array_equal(yy, np.arange(5, dtype=np.float64))


@pytest.mark.parametrize("version,kernel", [("baseline", 0), ("v1", 1), ("v1", 2), ("v1", 3),
                                            ("v2", 2), ("v2", 3)])
def test_dropin_large_call_chunked(cuda, version, kernel):
    """Calls with >= 8M nnz copy, compute and copy back in row chunks on two
    streams; results must match the oracle's drivers like small calls do
    (empty rows, beta != 0, several v2 tasks)."""
    from sbb import api, gen
    A = gen.uniform(41, 450_000, 300_000, 0, 46, p_empty=0.1)
    m, n, nnz = A.m, A.n, A.nnz
    assert nnz >= 8 << 20
    x = gen.uniform_vec(42, n)
    y = gen.uniform_vec(43, m)
    alpha, beta = 0.9, -0.7
    nb = nnz // 3 + 1
    kk = 1 if kernel == 3 else max(kernel, 1)
    rc_ref, y_ref = O.dropin(version, m, n, nnz, alpha, A.val, A.rowptr, A.col, x, beta, y,
                             ngpu=1, kernel=kk, nb=nb, q=2)
    yy = y.copy()
    if version == "baseline":
        rc = api.spMV_mgpu_baseline(m, n, nnz, alpha, A.val, A.rowptr, A.col, x, beta, yy, ngpu=1)
    elif version == "v1":
        rc = api.spMV_mgpu_v1(m, n, nnz, alpha, A.val, A.rowptr, A.col, x, beta, yy, ngpu=2,
                              kernel=kernel)
    else:
        rc = api.spMV_mgpu_v2(m, n, nnz, alpha, A.val, A.rowptr, A.col, x, beta, yy, ngpu=2,
                              kernel=kernel, nb=nb, q=2)
    assert rc == rc_ref == 0
    _, sc = O.spmv_dd(A.rowptr, A.col, A.val, x, alpha, beta, y)
    assert max_scaled_err(yy, y_ref, sc) <= TOL_FP64
    untouched = y_ref == y
    assert np.array_equal(yy[untouched], y[untouched])


@pytest.mark.parametrize("nb_div,q", [(400, 1), (400, 4), (3, 2), (1, 8)])
def test_v2_task_queue_matches_oracle(cuda, nb_div, q):
    """spMV_mgpu_v2 with kernel 2: the tasks run as the merge kernel's device
    work queue (q CTAs per SM, items of nb nnz up to the cap); every nb and q
    gives the oracle driver's result, and a repeated call the same bits."""
    from sbb import api
    rp, col, val, x, y = rand_csr(12, 150000, 120000, 0, 24)
    m, n, nnz = len(rp) - 1, len(x), int(rp[-1])
    nb = max(1, nnz // nb_div)
    rc_ref, y_ref = O.dropin("v2", m, n, nnz, 1.3, val, rp, col, x, -0.6, y, ngpu=1, kernel=2,
                             nb=nb, q=q)
    assert rc_ref == 0
    _, sc = O.spmv_dd(rp, col, val, x, 1.3, -0.6, y)
    outs = []
    for _ in range(2):
        yy = y.copy()
        assert api.spMV_mgpu_v2(m, n, nnz, 1.3, val, rp, col, x, -0.6, yy, ngpu=1, kernel=2,
                                nb=nb, q=q) == 0
        outs.append(yy)
    assert max_scaled_err(outs[0], y_ref, sc) <= TOL_FP64
    assert np.array_equal(outs[0], outs[1])


def test_last_call_phases(cuda):
    """sbb_last_call_phases: nothing before a thread's first call, then five
    non-negative phases of the last call that add up to at most its wall
    time."""
    import ctypes as C
    import threading
    import time
    from sbb import api
    from sbb._lib import lib
    got = {}

    def worker():
        ph = (C.c_double * 5)()
        got["before"] = lib().sbb_last_call_phases(ph, 5)
        rp, col, val, x, y = rand_csr(13, 3000, 2500, 0, 16)
        m, n, nnz = len(rp) - 1, len(x), int(rp[-1])
        t0 = time.perf_counter()
        got["rc"] = api.spMV_mgpu_v1(m, n, nnz, 1.0, val, rp, col, x, 0.5, y.copy(), ngpu=1, kernel=2)
        got["wall_ms"] = (time.perf_counter() - t0) * 1e3
        got["n"] = lib().sbb_last_call_phases(ph, 5)
        got["ph"] = list(ph)
        got["n2"] = lib().sbb_last_call_phases(ph, 2)

    th = threading.Thread(target=worker)
    th.start()
    th.join()
    assert got["before"] == 0 and got["rc"] == 0 and got["n"] == 5 and got["n2"] == 2
    assert all(v >= 0.0 for v in got["ph"]) and sum(got["ph"]) <= got["wall_ms"] + 1e-6


def test_v1_merge_same_bits_as_merge_plan(cuda):
    """A host-pointer call with kernel 2 builds its carry runs on the device
    (no host synchronisation) and still sums every run as the plan API's
    merge plan does: warp sums for runs of at most 1,024 carries, block trees
    for longer ones, so y is the same bit for bit."""
    import torch
    from sbb import api
    from sbb.device import Plan
    rp, col, val, x, y = rand_csr(14, 3000, 300000, 0, 8, long_rows=[(5, 220000), (77, 20000)])
    m, n, nnz = len(rp) - 1, len(x), int(rp[-1])
    yy = y.copy()
    assert api.spMV_mgpu_v1(m, n, nnz, 0.8, val, rp, col, x, 0.3, yy, ngpu=1, kernel=2) == 0
    d = torch.device("cuda:0")
    P = Plan(torch.from_numpy(rp.astype(np.int32)).to(d), torch.from_numpy(col).to(d),
             torch.from_numpy(val).to(d), n, kernel="merge")
    yd = torch.from_numpy(y).to(d)
    P.spmv(torch.from_numpy(x).to(d), yd, 0.8, 0.3)
    torch.cuda.synchronize()
    P.check()
    P.close()
    assert np.array_equal(yy, yd.cpu().numpy())
