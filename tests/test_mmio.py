"""CPU: the Matrix Market reader (csrc/host/mmio.cpp) against scipy's.

The reader returns canonical CSR (rows and columns sorted, duplicates summed,
symmetric storage expanded) whatever the file's entry order.  The reference's
test driver used the file's COO order as CSR (SparseBLAS/test/dspmv_test.cu:
228-251, 305-306); the last test shows what that gives for a file in column
order.
"""
import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from sbb import gen, mmio


def _scipy_csr(path, pattern_value=1.0):
    M = scipy.io.mmread(str(path), spmatrix=True)
    M = sp.csr_matrix(M) if not sp.issparse(M) else M.tocsr()
    if M.dtype == bool or "pattern" in open(path).readline():
        M = M.astype(np.float64)
        M.data[:] = pattern_value
    M.sum_duplicates()
    M.sort_indices()
    return M


def _write(path, banner, m, n, entries, comments=("a comment",), crlf=False, fmt="{} {} {}"):
    nl = "\r\n" if crlf else "\n"
    lines = [banner] + ["% " + c for c in comments] + ["", f"{m} {n} {len(entries)}"]
    for e in entries:
        lines.append(fmt.format(*e))
    path.write_text(nl.join(lines) + nl)


def _check(path, pattern_value=1.0, exact=True):
    A = mmio.read(path, pattern_value)
    S = _scipy_csr(path, pattern_value)
    assert (A.m, A.n) == S.shape
    assert np.array_equal(A.rowptr, S.indptr) and np.array_equal(A.col, S.indices)
    if exact:
        assert np.array_equal(A.val, S.data)
    else:
        assert np.allclose(A.val, S.data, rtol=1e-15, atol=0)
    return A


def _random_entries(rng, m, n, k, integer=False):
    i = rng.integers(1, m + 1, k)
    j = rng.integers(1, n + 1, k)
    v = rng.integers(-9, 10, k) if integer else rng.uniform(-1, 1, k)
    return list(zip(i.tolist(), j.tolist(), v.tolist()))


def test_general_real_any_order_with_duplicates(tmp_path):
    rng = np.random.default_rng(1)
    e = _random_entries(rng, 300, 200, 4000)  # random order, duplicate (i, j) pairs
    p = tmp_path / "g.mtx"
    _write(p, "%%MatrixMarket matrix coordinate real general", 300, 200, e)
    _check(p, exact=False)


def test_symmetric_and_skew_symmetric_are_expanded(tmp_path):
    rng = np.random.default_rng(2)
    m = 250
    lower = [(i, j, v) for i, j, v in _random_entries(rng, m, m, 3000) if j < i]
    lower = list({(i, j): (i, j, v) for i, j, v in lower}.values())
    diag = [(i, i, float(i)) for i in range(1, m + 1, 7)]
    for sym, entries in (("symmetric", lower + diag), ("skew-symmetric", lower)):
        p = tmp_path / f"{sym}.mtx"
        _write(p, f"%%MatrixMarket matrix coordinate real {sym}", m, m, entries)
        A = _check(p)
        D = sp.csr_matrix((A.val, A.col, A.rowptr), shape=(m, m)).toarray()
        assert np.array_equal(D, D.T if sym == "symmetric" else -D.T)


def test_pattern_and_integer_fields(tmp_path):
    rng = np.random.default_rng(3)
    e = _random_entries(rng, 120, 90, 700, integer=True)
    p = tmp_path / "i.mtx"
    _write(p, "%%MatrixMarket matrix coordinate integer general", 120, 90, e)
    _check(p, exact=False)
    q = tmp_path / "p.mtx"
    _write(q, "%%MatrixMarket matrix coordinate pattern general", 120, 90,
           list({(i, j): (i, j) for i, j, _ in e}.values()), fmt="{} {}")
    A = _check(q, pattern_value=0.5)
    assert np.all(A.val == 0.5)


def test_crlf_comments_blank_lines_and_empty_rows(tmp_path):
    e = [(5, 3, 1.5), (1, 1, -2.0), (5, 1, 0.25), (9, 9, 3.0)]
    p = tmp_path / "c.mtx"
    _write(p, "%%MatrixMarket matrix coordinate real general", 10, 9, e,
           comments=("first", "second"), crlf=True)
    A = _check(p)
    assert A.rowptr.tolist() == [0, 1, 1, 1, 1, 3, 3, 3, 3, 4, 4]


def test_round_trip_of_a_generated_matrix(tmp_path):
    A = gen.uniform(4, 20000, 15000, 0, 12, p_empty=0.05)
    p = tmp_path / "r.mtx"
    mmio.write(p, A)
    B = mmio.read(p)
    assert np.array_equal(A.rowptr, B.rowptr) and np.array_equal(A.col, B.col)
    assert np.array_equal(A.val, B.val)


@pytest.mark.parametrize("text,msg", [
    ("hello\n1 1 1\n1 1 1\n", "banner"),
    ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n", "field"),
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", "format"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n", "line 3"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1.0\n2 2 2.0\n", "ends after 2"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 x 1.0\n", "line 3"),
])
def test_malformed_files_are_rejected_with_the_line(tmp_path, text, msg):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(mmio.MatrixMarketError, match=msg):
        mmio.read(p)


def test_reference_driver_order_bug_and_the_fix(tmp_path):
    """A file in column order (the usual Matrix Market order).  The
    reference's driver builds the row pointer from per-row counts but keeps
    the columns and values in file order; its y is wrong.  The reader's CSR
    gives the right y."""
    rng = np.random.default_rng(5)
    m = n = 60
    D = np.where(rng.random((m, n)) < 0.1, rng.uniform(-1, 1, (m, n)), 0.0)
    jj, ii = np.nonzero(D.T)  # column-major order
    e = list(zip((ii + 1).tolist(), (jj + 1).tolist(), D[ii, jj].tolist()))
    p = tmp_path / "colmajor.mtx"
    _write(p, "%%MatrixMarket matrix coordinate real general", m, n, e)
    x = rng.uniform(-1, 1, n)
    A = mmio.read(p)
    y_fixed = sp.csr_matrix((A.val, A.col, A.rowptr), shape=(m, n)) @ x
    assert np.allclose(y_fixed, D @ x, rtol=1e-13, atol=1e-13)
    # the reference's construction (dspmv_test.cu:228-251 with COO arrays as CSR)
    counts = np.bincount(ii, minlength=m)
    rp_ref = np.concatenate([[0], np.cumsum(counts)])
    y_ref_driver = sp.csr_matrix((D[ii, jj], jj, rp_ref), shape=(m, n)) @ x
    assert not np.allclose(y_ref_driver, D @ x, rtol=1e-6, atol=1e-6)


def test_bench_reads_a_matrix_market_file(tmp_path):
    """bench.py --mtx: the reference arm (CPU) runs on a file read by the
    library's reader."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    A = gen.uniform(9, 3000, 2000, 1, 20)
    p = tmp_path / "u.mtx"
    mmio.write(p, A)
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--mtx", str(p),
                        "--cpu-budget", "0.2"], cwd=root, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    assert d["impl"] == "reference" and d["value"] > 0
    assert "u.mtx" in d["config"]["workload"] and d["config"]["nnz"] == A.nnz
