"""GPU: the plain path against cuSPARSE's SpMV on the same inputs.

The reference computes kernels 1 and 2 with cuSPARSE's csrmv and csrmv_mp;
their successor ``cusparseSpMV`` (CSR ALG1 and ALG2, ``cusparse_ref.py``)
runs here beside this library's kernels as a runtime comparator.
Bar, per row: |y - y_cusparse| <= 1e-12 * (|alpha| * sum_j |a_ij x_j| +
|beta * y_i|).  Each comparison first holds cuSPARSE itself to the same bar
against the double-double oracle, so a failure says which side is off.
The reference test's own check (test/dspmv_test.cu:268-279: x = 1, y = 0,
every version against cuSPARSE at absolute 1e-3) runs on every drop-in
entry point and kernel as well.
"""
import numpy as np
import pytest

import cusparse_ref as CS
import oracle as O
from helpers import TOL_FP64, max_scaled_err, rand_csr

MATS = {
    "uniform": lambda: rand_csr(1, 5000, 4000, 0, 30),
    "empty_rows": lambda: rand_csr(2, 4000, 3000, 0, 12, p_empty=0.6),
    "long_rows": lambda: rand_csr(3, 2000, 200000, 0, 8,
                                  long_rows=[(0, 150000), (999, 70000), (1999, 9000)]),
    "wide": lambda: rand_csr(5, 300, 100000, 100, 2000),
    "tall": lambda: rand_csr(6, 100000, 500, 0, 3),
}
PLANS = [dict(kernel="vector", vector_width=8), dict(kernel="merge"), dict(kernel="tiled"),
         dict(kernel="tiled", tile_sigma=4), dict(kernel="auto")]


def test_comparator_library_loads():
    """cuSPARSE's SpMV entry points resolve (no device needed)."""
    if not CS.available():
        pytest.skip("libcusparse not present")
    lib = CS._load()
    for name in ("cusparseCreateCsr", "cusparseSpMV", "cusparseSpMV_bufferSize"):
        assert getattr(lib, name) is not None


def _dev(rp, col, val, x, y):
    """Device copies; row offsets as int32, the width of the column indices
    (cuSPARSE takes one index width for both)."""
    import torch
    d = torch.device("cuda:0")
    return (torch.from_numpy(np.asarray(rp)).to(d, torch.int32), torch.from_numpy(col).to(d),
            torch.from_numpy(val).to(d), torch.from_numpy(x).to(d), torch.from_numpy(y).to(d))


def _cusparse(m, n, drp, dcol, dval, dx, y, alpha, beta, alg):
    import torch
    dy = torch.from_numpy(np.array(y, np.float64)).cuda()
    CS.spmv(m, n, drp, dcol, dval, dx, dy, alpha, beta, alg)
    return dy.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("alg", ["alg1", "alg2"])
@pytest.mark.parametrize("mat", list(MATS))
def test_plain_kernels_match_cusparse(cuda, mat, alg):
    import torch
    from sbb.device import Plan
    rp, col, val, x, y = MATS[mat]()
    m, n = len(rp) - 1, len(x)
    drp, dcol, dval, dx, dy = _dev(rp, col, val, x, y)
    for alpha, beta in ((1.0, 0.0), (-0.7, 0.3)):
        ref, sc = O.spmv_dd(rp, col, val, x, alpha, beta, y)
        ycs = _cusparse(m, n, drp, dcol, dval, dx, y, alpha, beta, alg)
        assert max_scaled_err(ycs, ref, sc) <= TOL_FP64, "cuSPARSE vs the oracle"
        for cfg in PLANS:
            P = Plan(drp, dcol, dval, n, **cfg)
            yy = dy.clone()
            P.spmv(dx, yy, alpha, beta)
            torch.cuda.synchronize()
            P.check()
            P.close()
            assert max_scaled_err(yy.cpu().numpy(), ycs, sc) <= TOL_FP64, (cfg, alpha, beta)


@pytest.mark.gpu
@pytest.mark.parametrize("version,kernel", [("baseline", 1), ("v1", 1), ("v1", 2), ("v1", 3),
                                            ("v2", 1), ("v2", 2), ("v2", 3)])
def test_dropin_reference_test_check(cuda, version, kernel):
    """dspmv_test.cu:268-279 and :390-401: x = 1, y = 0, alpha = 1, beta = 0,
    each version's y against cuSPARSE at absolute 1e-3; here also at the
    per-row bar."""
    from sbb import api
    rp, col, val, _, _ = rand_csr(11, 20000, 15000, 0, 40, p_empty=0.1,
                                  long_rows=[(7, 12000), (19000, 5000)])
    m, n, nnz = len(rp) - 1, 15000, int(rp[-1])
    x, y0 = np.ones(n), np.zeros(m)
    drp, dcol, dval, dx, _ = _dev(rp, col, val, x, y0)
    ycs = _cusparse(m, n, drp, dcol, dval, dx, y0, 1.0, 0.0, "alg1")
    y = y0.copy()
    args = (m, n, nnz, 1.0, val, rp, col, x, 0.0, y)
    if version == "baseline":
        rc = api.spMV_mgpu_baseline(*args, ngpu=1)
    elif version == "v1":
        rc = api.spMV_mgpu_v1(*args, ngpu=1, kernel=kernel)
    else:
        rc = api.spMV_mgpu_v2(*args, ngpu=1, kernel=kernel, nb=nnz // 7 + 1, q=2)
    assert rc == 0
    assert np.max(np.abs(y - ycs)) < 1e-3
    _, sc = O.spmv_dd(rp, col, val, x, 1.0, 0.0, y0)
    assert max_scaled_err(y, ycs, sc) <= TOL_FP64


@pytest.mark.gpu
@pytest.mark.parametrize("alg", ["alg1", "alg2"])
def test_full_size_c2_matches_cusparse(cuda, alg):
    """The 5.5M-row, 60M-nnz C2 matrix (one 1M-nnz row): the bench's plan
    (tiled, sigma 4) and the merge path against cuSPARSE; the per-row scale
    comes from cuSPARSE on |A| and |x|."""
    import torch
    from sbb import gen
    from sbb.device import Plan
    A = gen.c2()
    x = gen.uniform_vec(21, A.n)
    y = gen.uniform_vec(22, A.m)
    alpha, beta = 1.0, 0.5
    drp, dcol, dval, dx, dy = _dev(A.rowptr32(), A.col, A.val, x, y)
    ycs = _cusparse(A.m, A.n, drp, dcol, dval, dx, y, alpha, beta, alg)
    sa = _cusparse(A.m, A.n, drp, dcol, dval.abs(), dx.abs(), np.zeros(A.m), 1.0, 0.0, "alg1")
    sc = abs(alpha) * sa + np.abs(beta * y)
    for cfg in (dict(kernel="tiled", tile_sigma=4), dict(kernel="merge", items_per_thread=8)):
        P = Plan(drp, dcol, dval, A.n, **cfg)
        yy = dy.clone()
        P.spmv(dx, yy, alpha, beta)
        torch.cuda.synchronize()
        P.check()
        P.close()
        assert max_scaled_err(yy.cpu().numpy(), ycs, sc) <= TOL_FP64, cfg
