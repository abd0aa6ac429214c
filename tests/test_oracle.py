"""CPU: the oracle pinned against the reference's golden fixtures and code."""
import math
from fractions import Fraction

import numpy as np
import pytest

import oracle as O
from helpers import golden_cases, golden_grfi, rand_csr

CASES = golden_cases()


def test_golden_fixture_count():
    assert len(CASES) > 300
    kinds = {(c["version"], c["kernel"], c["ngpu"]) for c in CASES}
    assert ("v2", 2, 1) in kinds and ("v1", 3, 1) in kinds and ("baseline", 1, 2) in kinds


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_fixture(c):
    """Bit-exact: the restatement reproduces the reference drivers' output."""
    rc, y = O.dropin(c["version"], c["m"], c["n"], c["nnz"], c["alpha"], c["val"], c["rowptr"],
                     c["col"], c["x"], c["beta"], c["y"], ngpu=c["ngpu"], kernel=c["kernel"],
                     nb=c["nb"] or None, q=c["q"])
    assert rc == c["rc"]
    assert np.array_equal(y, c["y_ref"])


def test_get_row_from_index_golden():
    n = 0
    for m, rp, idx, row in golden_grfi():
        assert O.get_row_from_index(rp, idx) == row
        n += 1
    assert n > 500


def test_bisection_lands_on_empty_row():
    """The reference's bisection returns a row of an empty run on an exact hit."""
    rp = np.array([0, 3, 4, 4, 5], np.int64)   # rows 2 is empty; idx 4 belongs to row 3
    assert O.get_row_from_index(rp, 4) == 2
    assert O.get_row_from_index(rp, 3) == 1


@pytest.mark.skipif(not O.ref_available(), reason="reference drivers not built here")
def test_oracle_vs_reference_random():
    rng = np.random.default_rng(7)
    for t in range(120):
        m = int(rng.integers(1, 40))
        n = int(rng.integers(1, 30))
        rp, col, val, x, y = rand_csr(int(rng.integers(1 << 30)), m, n, 0, 6,
                                      p_empty=float(rng.choice([0, .3, .7])))
        nnz = int(rp[-1])
        if nnz == 0:
            continue
        for m_idx in range(nnz):
            assert O.get_row_from_index(rp, m_idx) == O.ref().ref_get_row_from_index(m, rp, m_idx)
        alpha, beta = float(rng.uniform(-2, 2)), float(rng.choice([0.0, rng.uniform(-2, 2)]))
        for ver, kw in (("v1", dict(ngpu=int(rng.integers(1, 5)), kernel=1)),
                        ("v2", dict(kernel=2, nb=int(rng.integers(1, nnz + 1)), q=3)),
                        ("baseline", dict(ngpu=1))):
            if ver == "v1" and kw["ngpu"] > nnz:
                continue
            r1 = O.dropin(ver, m, n, nnz, alpha, val, rp, col, x, beta, y, **kw)
            r2 = O.ref_dropin(ver, m, n, nnz, alpha, val, rp, col, x, beta, y, **kw)
            assert r1[0] == r2[0] and np.array_equal(r1[1], r2[1])


def test_partitions_restated():
    rp = np.array([0, 2, 2, 2, 7, 8, 8, 12], np.int64)
    nnz = 12
    parts = O.v1_partition(rp, nnz, 3)
    assert [p[:2] for p in parts] == [(0, 3), (4, 7), (8, 11)]
    assert all(p[2] <= p[3] for p in parts)
    tasks = O.v2_tasks(rp, nnz, np.zeros(7), 5)
    assert len(tasks) == 3 and tasks[0][0] == 0 and tasks[-1][1] == nnz - 1


def test_dd_oracle_is_correctly_rounded():
    rng = np.random.default_rng(3)
    rp, col, val, x, y = rand_csr(11, 50, 40, 0, 30)
    yd, sc = O.spmv_dd(rp, col, val, x, 1.0, 0.0, y)
    for i in range(50):
        exact = sum((Fraction(float(val[k])) * Fraction(float(x[col[k]]))
                     for k in range(rp[i], rp[i + 1])), Fraction(0))
        ex = float(exact)  # correctly rounded
        assert abs(yd[i] - ex) <= np.spacing(abs(ex) + 1e-300)
    assert np.all(sc >= 0)


def test_dd_oracle_beats_naive_on_cancellation():
    # one row: 1e16, 1, -1e16 -> exact 1; a plain left-to-right sum gives 0
    rp = np.array([0, 3], np.int64)
    col = np.array([0, 1, 2], np.int32)
    val = np.array([1e16, 1.0, -1e16])
    x = np.ones(3)
    yd, _ = O.spmv_dd(rp, col, val, x, 1.0, 0.0, np.zeros(1))
    assert yd[0] == 1.0
    yh = O.spmv_host(rp, col, val, x, 1.0, 0.0, np.zeros(1))
    assert yh[0] == 0.0


def test_host_loop_threads_agree():
    rp, col, val, x, y = rand_csr(5, 2000, 500, 0, 40)
    a = O.spmv_host(rp, col, val, x, 0.5, 0.25, y, 1)
    b = O.spmv_host(rp, col, val, x, 0.5, 0.25, y, 4)
    assert np.array_equal(a, b)


def test_scaled_error_catches_planted_mistake():
    """A planted one-ulp-scale change passes; a 1e-9 change does not."""
    rp, col, val, x, y = rand_csr(9, 300, 200, 1, 20)
    yd, sc = O.spmv_dd(rp, col, val, x, 1.0, 0.5, y)
    ok = yd + 1e-14 * sc
    bad = yd.copy()
    bad[17] += 1e-9 * sc[17]
    assert O.rel_err(ok, yd, sc).max() <= 1e-12
    assert O.rel_err(bad, yd, sc).max() > 1e-12


def _brute_merge(rp32, d):
    """Walk the merge of row ends and nnz indices for d steps."""
    m = len(rp32) - 1
    i = j = 0
    base = rp32[0]
    for _ in range(d):
        if i < m and rp32[i + 1] <= base + j:
            i += 1
        else:
            j += 1
    return i, base + j


@pytest.mark.parametrize("seed", range(6))
def test_merge_path_split_matches_walk(seed):
    rng = np.random.default_rng(seed)
    rp, *_ = rand_csr(seed, int(rng.integers(1, 60)), 30, 0, 9, p_empty=0.3,
                      long_rows=[(0, 25)])
    rp32 = rp.astype(np.int32)
    items = int(rng.integers(1, 12))
    total = len(rp) - 1 + int(rp[-1])
    P = (total + items - 1) // items
    rows, nzs = O.merge_path_split(rp32, items, P)
    for p in range(P + 1):
        assert (rows[p], nzs[p]) == _brute_merge(rp32, min(p * items, total))
    assert rows[-1] == len(rp) - 1 and nzs[-1] == rp[-1]


def test_csr5_sigma_rule():
    assert O.csr5_sigma(100, 300) == 4
    assert O.csr5_sigma(100, 1000) == 10
    assert O.csr5_sigma(100, 10000) == 32
    assert O.csr5_sigma(10, 10000) == 6
