"""GPU: the batched form and the autotuner probe.

Batched results must be bit-identical (FP64) to running each matrix alone
with the same class, whether the batch runs as one persistent launch or as a
replayed CUDA graph; and each matrix must match the accurate oracle within
TOL_FP64.
"""
import numpy as np
import pytest

import oracle as O
from helpers import TOL_FP64, max_scaled_err

pytestmark = pytest.mark.gpu


def _mats(n_mats, seed_base, scale=0.05):
    """Small members of the batch families (sizes scaled down for test time)."""
    import torch
    from sbb import gen
    out = []
    for i in range(n_mats):
        p = gen.c5_params(i, seed_base)
        p.m = p.n = max(64, int(p.m * scale))
        if p.family == gen.PLFAMILY:
            p.lmax = float(min(p.n, p.lmax))
        A = gen.generate(p)
        x = gen.uniform_vec(1000 + i, A.n)
        y = gen.uniform_vec(2000 + i, A.m)
        out.append(dict(m=A.m, n=A.n, rp=A.rowptr, col_h=A.col, val_h=A.val, x_h=x, y_h=y,
                        alpha=1.0, beta=0.5, rowptr=torch.from_numpy(A.rowptr32()).cuda(),
                        col=torch.from_numpy(A.col).cuda(), val=torch.from_numpy(A.val).cuda(),
                        x=torch.from_numpy(x).cuda(), y=torch.from_numpy(y).cuda()))
    return out


def _oracle_err(d, got):
    y_ref, sc = O.spmv_dd(d["rp"], d["col_h"], d["val_h"], d["x_h"], d["alpha"], d["beta"],
                          d["y_h"])
    return max_scaled_err(got, y_ref, sc)


def _compare(mats, classes, outs, ref_mode="each"):
    """Bit-identity of every mode with ref_mode, with a report that names the
    matrix, its class, the differing rows and which side the oracle backs."""
    for mode, ys in outs.items():
        if mode == ref_mode:
            continue
        for i, d in enumerate(mats):
            a, b = ys[i], outs[ref_mode][i]
            if np.array_equal(a, b):
                continue
            bad = np.flatnonzero(a != b)
            raise AssertionError(
                f"{mode} vs {ref_mode}: matrix {i} class {classes[i]} m={d['m']} "
                f"nnz={len(d['col_h'])}: {len(bad)} rows differ (first {bad[:8].tolist()}); "
                f"oracle err {mode}={_oracle_err(d, a):.3g} {ref_mode}={_oracle_err(d, b):.3g}")


def _run_modes(B, mats, modes=("each", "run", "graph", "graph2")):
    import torch
    y0 = [d["y"].clone() for d in mats]
    outs = {}
    for mode in modes:
        for d, y in zip(mats, y0):
            d["y"].copy_(y)
        {"each": B.run_each, "run": B.run, "graph": B.run_graph, "graph2": B.run_graph}[mode]()
        torch.cuda.synchronize()
        B.check()
        outs[mode] = [d["y"].cpu().numpy().copy() for d in mats]
    return outs


def test_batch_bit_identical_to_each_and_matches_oracle(cuda):
    from sbb.batch import Batch, NUM_CLASSES
    mats = _mats(36, 5)
    rng = np.random.default_rng(3)
    classes = [int(c) for c in rng.integers(0, NUM_CLASSES, len(mats))]
    classes[:NUM_CLASSES] = list(range(NUM_CLASSES))  # every class at least once
    B = Batch(mats, classes)
    outs = _run_modes(B, mats)
    _compare(mats, classes, outs)
    for i, d in enumerate(mats):
        assert _oracle_err(d, outs["run"][i]) <= TOL_FP64, (i, classes[i])
    # one persistent kernel per kernel family present (4) + the fix-up
    assert B.launches() <= 5 and B.launches(per_matrix=True) >= len(mats)
    B.close()


@pytest.mark.parametrize("cls", [4, 5], ids=["merge", "tiled"])
def test_batch_carry_classes_long_and_empty_rows(cuda, cls):
    """Merge/tiled-class matrices whose long rows span many segments or tiles
    (multi-slot carry runs), with empty rows (the tiled class finishes them in
    the fix-up launch), mixed with a vector-class matrix."""
    import torch
    from helpers import rand_csr
    from sbb.batch import Batch
    mats = []
    for k in range(8):
        rp, col, val, x, y = rand_csr(50 + k, 800, 60000, 0, 6, p_empty=0.2 * (k % 3),
                                      long_rows=[(3, 40000), (400, 20000 + 1000 * k)])
        mats.append(dict(m=800, n=60000, rp=rp, col_h=col, val_h=val, x_h=x, y_h=y, alpha=0.7,
                         beta=-1.0 if k % 2 else 0.0,
                         rowptr=torch.from_numpy(rp.astype(np.int32)).cuda(),
                         col=torch.from_numpy(col).cuda(), val=torch.from_numpy(val).cuda(),
                         x=torch.from_numpy(x).cuda(), y=torch.from_numpy(y).cuda()))
    classes = [cls] * len(mats)
    classes[2] = 0  # a vector unit between carry-class units of one claim
    B = Batch(mats, classes)
    outs = _run_modes(B, mats, ("each", "run", "graph"))
    _compare(mats, classes, outs)
    for i, d in enumerate(mats):
        assert _oracle_err(d, outs["graph"][i]) <= TOL_FP64, (i, classes[i])
    B.close()


def test_tuner_times_every_class(cuda):
    from sbb.batch import NUM_CLASSES, tune
    d = _mats(1, 7)[0]
    ms = tune(d, reps=3)
    assert len(ms) == NUM_CLASSES and all(t > 0 for t in ms)


def test_batch_edge_cases(cuda):
    """An empty batch; matrices without nnz in every class (y = beta*y, and
    y = 0 when beta = 0, as a plain launch does); a matrix with no rows."""
    import torch
    from sbb.batch import Batch, NUM_CLASSES
    B = Batch([], [])
    B.run()
    B.run_graph()
    torch.cuda.synchronize()
    B.check()
    assert B.launches() == 0
    B.close()
    mats, classes = [], []
    for cls in range(NUM_CLASSES):
        for beta in (0.0, 0.5):
            m = 1000 + 37 * cls
            y = np.random.default_rng(cls).uniform(-1, 1, m)
            mats.append(dict(m=m, n=50, beta=beta, alpha=2.0, y_h=y,
                             rowptr=torch.zeros(m + 1, dtype=torch.int32, device="cuda"),
                             col=torch.zeros(0, dtype=torch.int32, device="cuda"),
                             val=torch.zeros(0, dtype=torch.float64, device="cuda"),
                             x=torch.ones(50, dtype=torch.float64, device="cuda"),
                             y=torch.from_numpy(y).cuda()))
            classes.append(cls)
    mats.append(dict(m=0, n=10, rowptr=torch.zeros(1, dtype=torch.int32, device="cuda"),
                     col=torch.zeros(0, dtype=torch.int32, device="cuda"),
                     val=torch.zeros(0, dtype=torch.float64, device="cuda"),
                     x=torch.ones(10, dtype=torch.float64, device="cuda"),
                     y=torch.zeros(0, dtype=torch.float64, device="cuda"), y_h=np.zeros(0),
                     beta=0.5))
    classes.append(5)
    B = Batch(mats, classes)
    for run in (B.run, B.run_graph):
        for d in mats:
            d["y"].copy_(torch.from_numpy(d["y_h"]))
        run()
        torch.cuda.synchronize()
        B.check()
        for d, c in zip(mats, classes):
            want = d["beta"] * d["y_h"] if d["beta"] != 0.0 else np.zeros_like(d["y_h"])
            assert np.array_equal(d["y"].cpu().numpy(), want), c
    B.close()
