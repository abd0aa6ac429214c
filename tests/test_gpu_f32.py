"""GPU: the FP32-storage form (values and x stored as float; each product
formed exactly in FP64; row segments, carries, alpha and beta in FP64).

Two bars, per row with the scaled error of helpers.max_scaled_err:
  * against the FP64 double-double oracle on the ORIGINAL FP64 inputs:
    <= TOL_FP32 (1e-6) - the form's contract, input rounding included;
  * against the oracle on the FP32-ROUNDED inputs: <= 1e-12 - the arithmetic
    itself is as accurate as the FP64 kernels', so all of the error above is
    the rounding of val and x to float.
"""
import numpy as np
import pytest

import oracle as O
from helpers import TOL_FP32, max_scaled_err, rand_csr

pytestmark = pytest.mark.gpu

CONFIGS = [dict(kernel="vector", vector_width=v) for v in (4, 16, 32)] + \
          [dict(kernel="merge", items_per_thread=i) for i in (4, 8)] + \
          [dict(kernel="tiled", tile_sigma=s) for s in (4, 8, 16, 32)] + [dict(kernel="rows")] + \
          [dict(kernel="auto")]

MATS = {
    "uniform": lambda: rand_csr(11, 5000, 4000, 0, 30),
    "empty_rows": lambda: rand_csr(12, 4000, 3000, 0, 12, p_empty=0.6),
    "long_rows": lambda: rand_csr(13, 2000, 200000, 0, 8,
                                  long_rows=[(0, 150000), (999, 70000), (1999, 9000)]),
    "wide": lambda: rand_csr(15, 300, 100000, 100, 2000),
}


def run_f32(rp, col, val, x, y, n, alpha, beta, cfg, lanes=False):
    import torch
    from sbb.device import Plan
    d = torch.device("cuda:0")
    P = Plan(torch.from_numpy(rp.astype(np.int32)).to(d), torch.from_numpy(col).to(d),
             torch.from_numpy(val.astype(np.float32)).to(d), n, f32=True, f32_lanes=lanes,
             **cfg)
    yy = torch.from_numpy(y).to(d)
    P.spmv(torch.from_numpy(x.astype(np.float32)).to(d), yy, alpha, beta)
    torch.cuda.synchronize()
    P.check()
    P.close()
    return yy.cpu().numpy()


def check(rp, col, val, x, y, n, alpha, beta, cfg, lanes=False):
    got = run_f32(rp, col, val, x, y, n, alpha, beta, cfg, lanes)
    ref, sc = O.spmv_dd(rp, col, val, x, alpha, beta, y)
    e64 = max_scaled_err(got, ref, sc)
    v32, x32 = val.astype(np.float32).astype(np.float64), x.astype(np.float32).astype(np.float64)
    ref32, sc32 = O.spmv_dd(rp, col, v32, x32, alpha, beta, y)
    e32 = max_scaled_err(got, ref32, sc32)
    return e64, e32


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{v}" for v in c.values()))
@pytest.mark.parametrize("mat", sorted(MATS))
def test_f32_form_within_tolerance(cuda, cfg, mat):
    rp, col, val, x, y = MATS[mat]()
    n = int(col.max()) + 1 if len(col) else 1
    n = max(n, len(x))
    e64, e32 = check(rp, col, val, x, y, n, 1.25, -0.5, cfg)
    assert e64 <= TOL_FP32, e64
    assert e32 <= 1e-12, e32


@pytest.mark.parametrize("kernel", ["tiled", "rows"])
@pytest.mark.parametrize("which", ["c1", "c2"])
def test_f32_form_on_benchmark_matrices(cuda, which, kernel):
    """The C4 configuration (the 10k power-law matrix in FP32 storage) and the
    5.5M-row irregular matrix, tiled and row-block kernels: max and median
    per-row error."""
    from sbb import gen
    A = gen.c1() if which == "c1" else gen.c2()
    x = gen.uniform_vec(11 if which == "c1" else 21, A.n)
    y = gen.uniform_vec(22, A.m) if which == "c2" else np.zeros(A.m)
    beta = 0.5 if which == "c2" else 0.0
    e64, e32 = check(A.rowptr, A.col, A.val, x, y, A.n, 1.0, beta, dict(kernel=kernel))
    assert e64 <= TOL_FP32 and e32 <= 1e-12, (e64, e32)


# FP32 lane sums (sbb_plan_create_f32_lanes): a lane's run of k <= sigma
# products is summed in FP32, within k * 2^-24 of its exact value relative to
# sum |v*x|; everything after that is FP64.  So against the oracle on the
# rounded inputs the scaled error is at most sigma * 2^-24 (plus FP64
# rounding), and against the FP64 inputs it stays within TOL_FP32.
LANE_BOUND = {4: 4 * 2.0 ** -24 + 1e-12, 8: 8 * 2.0 ** -24 + 1e-12}


@pytest.mark.parametrize("sigma", [0, 4, 8])
@pytest.mark.parametrize("mat", sorted(MATS))
def test_f32_lane_sums_within_bound(cuda, sigma, mat):
    rp, col, val, x, y = MATS[mat]()
    n = max(int(col.max()) + 1 if len(col) else 1, len(x))
    cfg = dict(kernel="auto" if sigma == 0 else "tiled", tile_sigma=sigma)
    e64, e32 = check(rp, col, val, x, y, n, 1.25, -0.5, cfg, lanes=True)
    assert e64 <= TOL_FP32, e64
    assert e32 <= LANE_BOUND[sigma or 8], e32


@pytest.mark.parametrize("which", ["c1", "c2"])
def test_f32_lane_sums_on_benchmark_matrices(cuda, which):
    from sbb import gen
    A = gen.c1() if which == "c1" else gen.c2()
    x = gen.uniform_vec(11 if which == "c1" else 21, A.n)
    y = gen.uniform_vec(22, A.m) if which == "c2" else np.zeros(A.m)
    beta = 0.5 if which == "c2" else 0.0
    e64, e32 = check(A.rowptr, A.col, A.val, x, y, A.n, 1.0, beta, dict(kernel="auto"),
                     lanes=True)
    assert e64 <= TOL_FP32 and e32 <= LANE_BOUND[8], (e64, e32)


@pytest.mark.parametrize("cfg", [dict(kernel="merge"), dict(kernel="vector", vector_width=8),
                                 dict(kernel="rows"), dict(kernel="tiled", tile_sigma=16),
                                 dict(kernel="tiled", tile_sigma=32)],
                         ids=["merge", "vector", "rows", "tiled16", "tiled32"])
def test_f32_lane_sums_refuse_other_kernels(cuda, cfg):
    import torch
    from sbb.device import Plan, SbbError
    rp, col, val, x, y = MATS["uniform"]()
    d = torch.device("cuda:0")
    with pytest.raises(SbbError, match="lane sums"):
        Plan(torch.from_numpy(rp.astype(np.int32)).to(d), torch.from_numpy(col).to(d),
             torch.from_numpy(val.astype(np.float32)).to(d), len(x), f32=True, f32_lanes=True,
             **cfg)
