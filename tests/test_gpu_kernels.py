"""GPU: the device API's kernels against the accurate (double-double) oracle.

Error metric per row: |y - y_ref| / (|alpha|*sum_j |a_ij x_j| + |beta*y_i|)
<= TOL_FP64 (1e-12) for the FP64 kernels.  Integer work (the merge-path
partition) is compared bit for bit.
"""
import numpy as np
import pytest

import oracle as O
from helpers import TOL_FP64, max_scaled_err, rand_csr

pytestmark = pytest.mark.gpu

CONFIGS = [dict(kernel="vector", vector_width=v) for v in (2, 4, 8, 16, 32)] + \
          [dict(kernel="merge", items_per_thread=i) for i in (4, 6, 8, 12)] + \
          [dict(kernel="merge", items_per_thread=8, persistent=p) for p in (1, 2, 4)] + \
          [dict(kernel="tiled"), dict(kernel="tiled", tile_sigma=4), dict(kernel="tiled", tile_sigma=16),
           dict(kernel="rows"), dict(kernel="auto")]


def to_dev(rp, col, val, x, y, f32=False):
    import torch
    d = torch.device("cuda:0")
    vt = torch.float32 if f32 else torch.float64
    return (torch.from_numpy(rp.astype(np.int32)).to(d), torch.from_numpy(col).to(d),
            torch.from_numpy(val).to(d, vt), torch.from_numpy(x).to(d, vt),
            torch.from_numpy(y).to(d))


def run_plan(rp, col, val, x, y, n, alpha, beta, cfg, reps=1):
    import torch
    from sbb.device import Plan
    drp, dcol, dval, dx, dy = to_dev(rp, col, val, x, y)
    P = Plan(drp, dcol, dval, n, **cfg)
    outs = []
    for _ in range(reps):
        yy = dy.clone()
        P.spmv(dx, yy, alpha, beta)
        torch.cuda.synchronize()
        outs.append(yy.cpu().numpy())
    P.check()
    info = P.info()
    P.close()
    return outs, info


MATS = {
    "uniform": lambda: rand_csr(1, 5000, 4000, 0, 30),
    "empty_rows": lambda: rand_csr(2, 4000, 3000, 0, 12, p_empty=0.6),
    "long_rows": lambda: rand_csr(3, 2000, 200000, 0, 8,
                                  long_rows=[(0, 150000), (999, 70000), (1999, 9000)]),
    "one_row": lambda: rand_csr(4, 1, 50000, 40000, 40000),
    "wide": lambda: rand_csr(5, 300, 100000, 100, 2000),
    "tall": lambda: rand_csr(6, 100000, 500, 0, 3),
    "all_empty": lambda: rand_csr(7, 777, 100, 0, 0),
}


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{v}" for v in c.values()))
@pytest.mark.parametrize("mat", list(MATS))
def test_kernel_matches_oracle(cuda, cfg, mat):
    rp, col, val, x, y = MATS[mat]()
    n = len(x)
    for alpha, beta in ((1.0, 0.0), (-0.7, 0.3), (0.0, 2.0)):
        y_ref, sc = O.spmv_dd(rp, col, val, x, alpha, beta, y)
        (out,), _ = run_plan(rp, col, val, x, y, n, alpha, beta, cfg)
        assert max_scaled_err(out, y_ref, sc) <= TOL_FP64, (alpha, beta)


@pytest.mark.parametrize("ipt", [4, 8, 12])
@pytest.mark.parametrize("mat", ["uniform", "empty_rows", "long_rows", "tall"])
def test_merge_partition_bit_exact(cuda, ipt, mat):
    import torch
    from sbb.device import Plan
    rp, col, val, x, y = MATS[mat]()
    drp, dcol, dval, dx, dy = to_dev(rp, col, val, x, y)
    P = Plan(drp, dcol, dval, len(x), kernel="merge", items_per_thread=ipt)
    rows, nzs = P.partition()
    P.close()
    ref_rows, ref_nzs = O.merge_path_split(rp.astype(np.int32), 32 * ipt, len(rows) - 1)
    assert np.array_equal(rows, ref_rows) and np.array_equal(nzs, ref_nzs)


@pytest.mark.parametrize("cfg", [dict(kernel="merge", items_per_thread=8),
                                 dict(kernel="merge", items_per_thread=8, persistent=2),
                                 dict(kernel="vector", vector_width=8), dict(kernel="tiled"),
                                 dict(kernel="rows")])
def test_repeat_runs_bit_identical(cuda, cfg):
    rp, col, val, x, y = MATS["long_rows"]()
    outs, _ = run_plan(rp, col, val, x, y, len(x), 1.3, 0.4, cfg, reps=3)
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])


def test_bad_column_is_flagged_not_faulted(cuda):
    import torch
    from sbb.device import Plan, SbbError
    rp, col, val, x, y = MATS["uniform"]()
    col = col.copy()
    col[123] = len(x) + 5
    drp, dcol, dval, dx, dy = to_dev(rp, col, val, x, y)
    P = Plan(drp, dcol, dval, len(x), kernel="merge")
    P.spmv(dx, dy)
    with pytest.raises(SbbError):
        P.check()
    P.close()


@pytest.mark.parametrize("kernel", ["tiled", "rows"])
def test_bad_column_rejected_by_plan(cuda, kernel):
    """The tiled and row-block kernels range-check columns once, when their
    plan is built."""
    from sbb.device import Plan, SbbError
    rp, col, val, x, y = MATS["uniform"]()
    col = col.copy()
    col[-1] = -3
    drp, dcol, dval, dx, dy = to_dev(rp, col, val, x, y)
    with pytest.raises(SbbError):
        Plan(drp, dcol, dval, len(x), kernel=kernel)



def test_overlapping_x_and_y_rejected(cuda):
    """x must not overlap y (the kernels read x while they write y): refused
    with an error; adjacent, non-overlapping views of one buffer are fine."""
    import torch
    from sbb.device import Plan, SbbError
    rp, col, val, x, y = MATS["uniform"]()  # 5000 x 4000
    drp, dcol, dval, _, _ = to_dev(rp, col, val, x, y)
    buf = torch.zeros(9000, dtype=torch.float64, device="cuda")
    for cfg in (dict(kernel="vector", vector_width=8), dict(kernel="merge"), dict(kernel="tiled"),
                dict(kernel="rows")):
        P = Plan(drp, dcol, dval, 4000, **cfg)
        with pytest.raises(SbbError):
            P.spmv(buf[:4000], buf[3999:8999], 1.0, 0.0)
        P.spmv(buf[:4000], buf[4000:9000], 1.0, 0.0)
        torch.cuda.synchronize()
        P.check()
        P.close()
    assert torch.count_nonzero(buf) == 0

def test_bad_rowptr_rejected_at_plan(cuda):
    from sbb.device import Plan, SbbError
    rp, col, val, x, y = MATS["uniform"]()
    rp = rp.copy()
    rp[100] = rp[101] + 1
    drp, dcol, dval, dx, dy = to_dev(rp, col, val, x, y)
    with pytest.raises(SbbError):
        Plan(drp, dcol, dval, len(x), kernel="merge")


def test_config1_full_parity(cuda):
    """C1: n = 10,000 power-law matrix, alpha = 1, beta = 0, every kernel."""
    from sbb import gen
    A = gen.c1()
    x = gen.uniform_vec(11, A.n)
    y = np.zeros(A.m)
    y_ref, sc = O.spmv_dd(A.rowptr, A.col, A.val, x, 1.0, 0.0, y)
    for cfg in (dict(kernel="vector", vector_width=8), dict(kernel="merge"), dict(kernel="tiled"),
                dict(kernel="rows"), dict(kernel="auto")):
        (out,), _ = run_plan(A.rowptr, A.col, A.val, x, y, A.n, 1.0, 0.0, cfg)
        assert max_scaled_err(out, y_ref, sc) <= TOL_FP64


@pytest.mark.parametrize("which", ["c2", "c3"])
def test_full_size_parity(cuda, which):
    """C2 (5.5M rows, 60M nnz, one 1M-nnz row) and C3 at full size vs the oracle."""
    from sbb import gen
    A = gen.c2() if which == "c2" else gen.c3()
    x = gen.uniform_vec(21, A.n)
    y = gen.uniform_vec(22, A.m)
    beta = 0.5 if which == "c2" else 0.0
    y_ref, sc = O.spmv_dd(A.rowptr, A.col, A.val, x, 1.0, beta, y)
    for cfg in (dict(kernel="merge", items_per_thread=8), dict(kernel="tiled"), dict(kernel="rows"),
                dict(kernel="auto")):
        (out,), _ = run_plan(A.rowptr, A.col, A.val, x, y, A.n, 1.0, beta, cfg)
        assert max_scaled_err(out, y_ref, sc) <= TOL_FP64, cfg



def _host_bytes_available():
    """Free host memory for this process: MemAvailable, capped by a cgroup
    (v2) memory limit when one is set."""
    avail = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail = int(line.split()[1]) * 1024
    except OSError:
        pass
    try:
        with open("/sys/fs/cgroup/memory.max") as f:
            lim = f.read().strip()
        if lim != "max":
            with open("/sys/fs/cgroup/memory.current") as f:
                cur = int(f.read().strip())
            room = int(lim) - cur
            avail = room if avail is None else min(avail, room)
    except (OSError, ValueError):
        pass
    return avail or 0


def _wide_matrix():
    """n = 2^31 - 1 columns, columns 0 and n - 1 in many rows, one row of
    5,000 nnz across many tiles; integer values and y; alpha = 2, beta = 0.5;
    with x[c] = c mod 1000 the result (returned as `want`) is exact."""
    n = 2 ** 31 - 1
    rng = np.random.default_rng(77)
    lens = np.full(3000, 9, np.int64)
    lens[17], lens[2000] = 5000, 700
    rp = np.zeros(len(lens) + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    nnz = int(rp[-1])
    col = rng.integers(0, n, nnz).astype(np.int64)
    col[rp[:-1][::2]] = 0            # first nnz of every other row: column 0
    col[rp[1:][::3] - 1] = n - 1     # last nnz of every third row: column n - 1
    val = rng.integers(-5, 6, nnz).astype(np.float64)
    y0 = 2.0 * rng.integers(-1000, 1000, len(lens)).astype(np.float64)
    alpha, beta = 2.0, 0.5
    prod = val * (col % 1000).astype(np.float64)
    want = alpha * np.add.reduceat(prod, rp[:-1]) + beta * y0  # exact integers
    return dict(n=n, m=len(lens), nnz=nnz, rp=rp, col=col.astype(np.int32), val=val, y0=y0,
                alpha=alpha, beta=beta, want=want)


def test_column_indices_up_to_int32_max(cuda):
    """The widest matrix an int32 column index addresses (x is 17 GB on the
    device): every product and sum is an exact integer in FP64 (and in the
    FP32-storage form), so each kernel must give the exact result bit for
    bit whatever its summation order."""
    import torch
    from sbb.device import Plan
    free, _ = torch.cuda.mem_get_info()
    if free < 40 * 2 ** 30:
        pytest.skip("needs 40 GiB of free device memory")
    W = _wide_matrix()
    n, alpha, beta, want = W["n"], W["alpha"], W["beta"], W["want"]
    d = torch.device("cuda:0")
    x = torch.arange(n, dtype=torch.float64, device=d)
    x.remainder_(1000.0)
    drp = torch.from_numpy(W["rp"].astype(np.int32)).to(d)
    dcol = torch.from_numpy(W["col"]).to(d)
    dval = torch.from_numpy(W["val"]).to(d)
    dy0 = torch.from_numpy(W["y0"]).to(d)
    for cfg in (dict(kernel="vector", vector_width=8), dict(kernel="vector", vector_width=32),
                dict(kernel="merge", items_per_thread=8), dict(kernel="tiled", tile_sigma=4),
                dict(kernel="tiled", tile_sigma=16), dict(kernel="rows"), dict(kernel="auto")):
        P = Plan(drp, dcol, dval, n, **cfg)
        yy = dy0.clone()
        P.spmv(x, yy, alpha, beta)
        torch.cuda.synchronize()
        P.check()
        P.close()
        assert np.array_equal(yy.cpu().numpy(), want), cfg
    x32 = x.float()
    for kernel in ("tiled", "rows"):
        P = Plan(drp, dcol, dval.float(), n, kernel=kernel, f32=True)
        yy = dy0.clone()
        P.spmv(x32, yy, alpha, beta)
        torch.cuda.synchronize()
        P.check()
        P.close()
        assert np.array_equal(yy.cpu().numpy(), want), ("f32", kernel)
    del x32, x
    torch.cuda.empty_cache()


def test_dropin_column_indices_up_to_int32_max(cuda):
    """The same matrix through the drop-in, x (17 GB) in host memory."""
    import torch
    from sbb import api
    if _host_bytes_available() < 64 * 2 ** 30:
        pytest.skip("needs 64 GiB of free host memory")
    torch.cuda.empty_cache()
    if torch.cuda.mem_get_info()[0] < 40 * 2 ** 30:
        pytest.skip("needs 40 GiB of free device memory")
    W = _wide_matrix()
    xh = np.arange(W["n"], dtype=np.float64)
    np.remainder(xh, 1000.0, out=xh)
    yh = W["y0"].copy()
    assert api.spMV_mgpu_v1(W["m"], W["n"], W["nnz"], W["alpha"], W["val"], W["rp"], W["col"],
                            xh, W["beta"], yh, ngpu=1, kernel=3) == 0
    assert np.array_equal(yh, W["want"])


def _max_nnz_matrix(d):
    """nnz = 2^31 - 1 (the largest an int32 row pointer holds, and the
    reference's per-device cast): 2^24 rows of 128 nnz, the last of 127, so
    the last rows end at index 2^31 - 1.  Integer values (+-1..3), x[c] =
    c mod 1000, integer y, alpha = 2, beta = 0.5: every product and sum is an
    exact integer, and `want` is the exact result (a row-wise torch
    reduction in chunks of whole rows)."""
    import torch
    nnz, m, L, n = 2 ** 31 - 1, 2 ** 24, 128, 2 ** 20
    rp = torch.arange(m + 1, dtype=torch.int64, device=d) * L
    rp[-1] = nnz
    rp = rp.to(torch.int32)
    col = torch.empty(nnz, dtype=torch.int32, device=d)
    val = torch.empty(nnz, dtype=torch.float64, device=d)
    x = torch.arange(n, dtype=torch.float64, device=d).remainder_(1000.0)
    rows = torch.empty(m, dtype=torch.float64, device=d)
    CH = 1 << 27  # whole rows per chunk
    for s in range(0, nnz, CH):
        e = min(nnz, s + CH)
        idx = torch.arange(s, e, dtype=torch.int64, device=d)
        r, j = idx // L, idx % L
        c = (r * 37 + j * 5) % n
        col[s:e] = c.to(torch.int32)
        v = (1 + j % 3).to(torch.float64) * (1 - 2 * (r % 2)).to(torch.float64)
        val[s:e] = v
        p = v * x[c]
        full = (e - s) // L
        rows[s // L:s // L + full] = p[:full * L].view(full, L).sum(dim=1)
        if full * L < e - s:  # the last row (127 nnz)
            rows[s // L + full] = p[full * L:].sum()
        del idx, r, j, c, v, p
    y0 = 2.0 * (torch.arange(m, dtype=torch.float64, device=d).remainder_(2000.0) - 1000.0)
    alpha, beta = 2.0, 0.5
    want = (alpha * rows + beta * y0).cpu().numpy()
    return dict(nnz=nnz, m=m, n=n, rp=rp, col=col, val=val, x=x, y0=y0, alpha=alpha, beta=beta,
                want=want)


def test_nnz_at_int32_max(cuda):
    """Every kernel on a matrix of 2^31 - 1 nnz, bit for bit (the vector
    kernel's lanes step past index 2^31 - 1 on the last rows)."""
    import torch
    from sbb.device import Plan
    torch.cuda.empty_cache()
    if torch.cuda.mem_get_info()[0] < 100 * 2 ** 30:
        pytest.skip("needs 100 GiB of free device memory")
    W = _max_nnz_matrix(cuda)
    for cfg in (dict(kernel="vector", vector_width=32), dict(kernel="vector", vector_width=4),
                dict(kernel="merge", items_per_thread=8), dict(kernel="tiled", tile_sigma=4),
                dict(kernel="rows"), dict(kernel="auto")):
        P = Plan(W["rp"], W["col"], W["val"], W["n"], **cfg)
        yy = W["y0"].clone()
        P.spmv(W["x"], yy, W["alpha"], W["beta"])
        torch.cuda.synchronize()
        P.check()
        P.close()
        assert np.array_equal(yy.cpu().numpy(), W["want"]), cfg
    del W
    torch.cuda.empty_cache()


def test_dropin_nnz_at_int32_max(cuda):
    """The same matrix through spMV_mgpu_v1 (kernels 1 and 3) from host
    memory (26 GB of columns and values)."""
    import torch
    from sbb import api
    if _host_bytes_available() < 96 * 2 ** 30:
        pytest.skip("needs 96 GiB of free host memory")
    torch.cuda.empty_cache()
    if torch.cuda.mem_get_info()[0] < 100 * 2 ** 30:
        pytest.skip("needs 100 GiB of free device memory")
    W = _max_nnz_matrix(cuda)
    rp = W["rp"].cpu().numpy().astype(np.int64)
    rp[-1] = W["nnz"]
    col, val, x, y0 = (W[k].cpu().numpy() for k in ("col", "val", "x", "y0"))
    want, alpha, beta, m, n, nnz = (W[k] for k in ("want", "alpha", "beta", "m", "n", "nnz"))
    del W
    torch.cuda.empty_cache()
    for kernel in (1, 3):
        yh = y0.copy()
        assert api.spMV_mgpu_v1(m, n, nnz, alpha, val, rp, col, x, beta, yh, ngpu=1,
                                kernel=kernel) == 0
        assert np.array_equal(yh, want), kernel


def test_rows_at_int32_max(cuda):
    """m = 2^31 - 1 rows (row pointer 8.6 GB, y 17 GB): one nnz in every
    128th row and 10,000 in row 5.  The vector and merge kernels and the
    automatic choice (the merge path here: a long row, and more rows than a
    tile plan takes) give the exact result bit for bit; an explicit tile
    plan is refused with an error, not run."""
    import torch
    from sbb.device import Plan, SbbError
    torch.cuda.empty_cache()
    if torch.cuda.mem_get_info()[0] < 100 * 2 ** 30:
        pytest.skip("needs 100 GiB of free device memory")
    d = cuda
    m, n, long_row, long_len = 2 ** 31 - 1, 2 ** 20, 5, 10000
    # rowptr[r] = ceil(r / 128) + long_len * (r > long_row), in chunks
    rp = torch.empty(m + 1, dtype=torch.int32, device=d)
    CH = 1 << 28
    for s in range(0, m + 1, CH):
        r = torch.arange(s, min(m + 1, s + CH), dtype=torch.int64, device=d)
        rp[s:s + len(r)] = ((r + 127) // 128 + long_len * (r > long_row)).to(torch.int32)
        del r
    nnz = int(rp[-1].item())
    k = torch.arange(nnz, dtype=torch.int64, device=d)
    col = ((k * 37) % n).to(torch.int32)
    val = ((1 + k % 3) * (1 - 2 * (k % 2))).to(torch.float64)
    x = torch.arange(n, dtype=torch.float64, device=d).remainder_(1000.0)
    # row of nnz k: 0 for k = 0, the long row for k <= long_len, then every
    # 128th row in turn
    row_of = torch.where(k == 0, 0, torch.where(k <= long_len, long_row, (k - long_len) * 128))
    want = torch.zeros(m, dtype=torch.float64, device=d)
    want.index_add_(0, row_of, val * x[col.long()])  # exact integers
    del k, row_of
    y0 = torch.arange(m, dtype=torch.float64, device=d).remainder_(2000.0).sub_(1000.0).mul_(2.0)
    alpha, beta = 2.0, 0.5
    want.mul_(alpha).add_(y0, alpha=beta)
    yy = torch.empty_like(y0)
    for cfg in (dict(kernel="vector", vector_width=4), dict(kernel="merge", items_per_thread=8),
                dict(kernel="rows"), dict(kernel="auto")):
        P = Plan(rp, col, val, n, **cfg)
        if cfg["kernel"] == "auto":
            assert P.info()["kernel"] == 2  # the merge path
        yy.copy_(y0)
        P.spmv(x, yy, alpha, beta)
        torch.cuda.synchronize()
        P.check()
        P.close()
        assert torch.equal(yy, want), cfg
    with pytest.raises(SbbError):
        Plan(rp, col, val, n, kernel="tiled")


@pytest.mark.parametrize("f32", [False, True])
def test_unaligned_views(cuda, f32):
    """Row pointer, columns and values that are views at every element offset
    of a 16-byte block of larger buffers: the row-block kernel copies only the
    16-byte-aligned middle of each range by TMA and loads the ragged ends
    itself, so each offset must give the oracle's result (and every kernel
    must work on such views)."""
    import torch
    from sbb.device import Plan
    rp, col, val, x, y = rand_csr(8, 3000, 2500, 0, 40, p_empty=0.1,
                                  long_rows=[(7, 1000), (1500, 2400)])
    d = torch.device("cuda:0")
    vt = torch.float32 if f32 else torch.float64
    nnz, m = len(col), len(rp) - 1
    dx = torch.from_numpy(x).to(d, vt)
    xs = dx.double().cpu().numpy() if f32 else x
    vs = val.astype(np.float32).astype(np.float64) if f32 else val
    y_ref, sc = O.spmv_dd(rp, col, vs, xs, 1.1, -0.6, y)
    per16 = 4 if f32 else 2
    for off_i in range(4):
        for off_v in range(per16):
            brp = torch.zeros(m + 1 + 8, dtype=torch.int32, device=d)
            bcol = torch.zeros(nnz + 8, dtype=torch.int32, device=d)
            bval = torch.zeros(nnz + 8, dtype=vt, device=d)
            brp[off_i:off_i + m + 1] = torch.from_numpy(rp.astype(np.int32)).to(d)
            bcol[(3 - off_i):(3 - off_i) + nnz] = torch.from_numpy(col).to(d)
            bval[off_v:off_v + nnz] = torch.from_numpy(val).to(d, vt)
            drp = brp[off_i:off_i + m + 1]
            dcol = bcol[(3 - off_i):(3 - off_i) + nnz]
            dval = bval[off_v:off_v + nnz]
            for kernel in ("rows", "merge", "tiled", "vector"):
                P = Plan(drp, dcol, dval, len(x), kernel=kernel, f32=f32)
                yy = torch.from_numpy(y).to(d)
                P.spmv(dx, yy, 1.1, -0.6)
                torch.cuda.synchronize()
                P.check()
                P.close()
                tol = 1e-12 if not f32 else 1e-12
                assert max_scaled_err(yy.cpu().numpy(), y_ref, sc) <= tol, (kernel, off_i, off_v)


@pytest.mark.parametrize("cfg", [dict(kernel="tiled", tile_sigma=4), dict(kernel="tiled", tile_sigma=16),
                                 dict(kernel="merge", items_per_thread=8), dict(kernel="rows"),
                                 dict(kernel="vector", vector_width=8)])
def test_plan_spmv_captured_in_cuda_graph(cuda, cfg):
    """A plan's SpMVs captured in a CUDA graph and replayed give the same bits
    as the same calls launched directly (after one direct call on the device,
    which sets the launch configuration up)."""
    import torch
    from sbb.device import Plan
    rp, col, val, x, y = MATS["long_rows"]()
    drp, dcol, dval, dx, dy = to_dev(rp, col, val, x, y)
    P = Plan(drp, dcol, dval, len(x), **cfg)
    y_direct = dy.clone()
    for _ in range(3):
        P.spmv(dx, y_direct, 1.1, 0.7)
    torch.cuda.synchronize()
    y_graph = dy.clone()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=torch.cuda.Stream()):
        for _ in range(3):
            P.spmv(dx, y_graph, 1.1, 0.7)
    y_graph.copy_(dy)
    g.replay()
    torch.cuda.synchronize()
    P.check()
    assert torch.equal(y_graph, y_direct)
    del g
    P.close()


@pytest.mark.parametrize("persistent", [1, 2, 4])
def test_merge_work_queue_same_bits(cuda, persistent):
    """The persistent merge form, whose warps claim segments from a device
    work queue, gives the same bits as one warp per segment, call after call
    (the fix-up re-arms the queue), directly and from a CUDA graph."""
    import torch
    from sbb.device import Plan
    rp, col, val, x, y = rand_csr(11, 200000, 150000, 0, 20, long_rows=[(7, 90000)])
    drp, dcol, dval, dx, dy = to_dev(rp, col, val, x, y)
    ref, _ = run_plan(rp, col, val, x, y, len(x), 0.9, 0.4, dict(kernel="merge", items_per_thread=8))
    P = Plan(drp, dcol, dval, len(x), kernel="merge", items_per_thread=8, persistent=persistent)
    info = P.info()
    assert 0 < info["persistent"] and info["persistent"] * 8 < info["tiles"]  # the queue is used
    for _ in range(3):
        yy = dy.clone()
        P.spmv(dx, yy, 0.9, 0.4)
        torch.cuda.synchronize()
        assert np.array_equal(yy.cpu().numpy(), ref[0])
    yg = dy.clone()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=torch.cuda.Stream()):
        P.spmv(dx, yg, 0.9, 0.4)
    for _ in range(2):
        yg.copy_(dy)
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(yg.cpu().numpy(), ref[0])
    del g
    P.check()
    P.close()
    y_ref, sc = O.spmv_dd(rp, col, val, x, 0.9, 0.4, y)
    assert max_scaled_err(ref[0], y_ref, sc) <= TOL_FP64
