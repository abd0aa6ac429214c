"""Generate the golden fixtures in this directory from the reference's own code.

Run in the development container, where oracle/_ref/libref.so can be built
from the reference sources (``make -C oracle ref REF=<its SparseBLAS
directory>``, or with SBB_REFERENCE_SRC set).  That library is the
reference's host drivers (SparseBLAS/src/dspmv_mgpu_{baseline,v1,v2}.cu and
spmv_helper.cu), compiled unchanged against CPU stand-ins for the CUDA runtime
and the removed legacy cuSPARSE csrmv (oracle/ref_shim.cpp).  Each fixture
holds a small CSR matrix, x, y, alpha, beta, the call's arguments and the
reference's output y, so the tests can check the oracle and the GPU path
against it without the reference present.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402


def rand_csr(rng, m, n, maxlen, p_empty, tie_tail=False):
    lens = rng.integers(1, maxlen + 1, m)
    lens[rng.random(m) < p_empty] = 0
    if tie_tail and m >= 4:
        # last non-empty row has one nnz and is preceded by empty rows: the
        # bisection can land on an empty row (misattribution) — reference quirk
        lens[-4:] = [0, 0, 1, 0]
    lens = np.minimum(lens, n)
    rp = np.zeros(m + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    col = np.concatenate([np.sort(rng.choice(n, l, replace=False)) if l else np.zeros(0, int)
                          for l in lens]).astype(np.int32)
    val = rng.uniform(-1, 1, int(rp[-1]))
    x = rng.uniform(-1, 1, n)
    y = rng.uniform(-1, 1, m)
    return rp, col, val, x, y


def cases():
    rng = np.random.default_rng(20260101)
    out = []
    shapes = [(1, 1, 1, 0.0), (2, 3, 3, 0.0), (7, 5, 4, 0.3), (33, 17, 8, 0.2), (64, 64, 12, 0.5),
              (120, 90, 20, 0.1), (257, 300, 9, 0.4), (300, 50, 30, 0.0)]
    k = 0
    mats = []
    for (m, n, maxlen, pe) in shapes:
        for tie in (False, True):
            rp, col, val, x, y = rand_csr(rng, m, n, maxlen, pe, tie_tail=tie)
            nnz = int(rp[-1])
            if nnz == 0:
                continue
            mid = len(mats)
            mats.append(dict(rowptr=rp, col=col, val=val, x=x, y=y))
            for alpha, beta in ((1.0, 0.0), (0.75, 0.5), (-1.25, 1.0)):
                calls = [("baseline", dict(ngpu=1)), ("v1", dict(ngpu=1, kernel=1)),
                         ("v1", dict(ngpu=1, kernel=2)), ("v1", dict(ngpu=1, kernel=3)),
                         ("v2", dict(ngpu=1, kernel=1, nb=nnz, q=1)),
                         ("v2", dict(ngpu=1, kernel=2, nb=max(1, nnz // 3), q=2)),
                         ("v2", dict(ngpu=1, kernel=1, nb=max(1, nnz // 7), q=4)),
                         ("v1", dict(ngpu=3, kernel=1)), ("baseline", dict(ngpu=2))]
                for ver, kw in calls:
                    if ver == "v1" and kw["ngpu"] > nnz:
                        continue
                    if ver == "baseline" and kw["ngpu"] > m:
                        continue
                    rc, yref = O.ref_dropin(ver, m, n, nnz, alpha, val, rp, col, x, beta, y,
                                            **kw)
                    out.append(dict(name=f"case{k:03d}", version=ver, m=m, n=n, nnz=nnz,
                                    alpha=alpha, beta=beta, mat=mid, y_ref=yref, rc=rc,
                                    ngpu=kw.get("ngpu", 1),
                                    kernel=kw.get("kernel", 1), nb=kw.get("nb", 0),
                                    q=kw.get("q", 1)))
                    k += 1
    # get_row_from_index answers on row pointers with runs of empty rows
    grfi = []
    for t in range(40):
        m = int(rng.integers(1, 50))
        lens = rng.integers(0, 4, m)
        lens[rng.random(m) < 0.5] = 0
        rp = np.zeros(m + 1, np.int64)
        rp[1:] = np.cumsum(lens)
        for idx in range(int(rp[-1])):
            grfi.append((m, rp.copy(), idx, O.ref().ref_get_row_from_index(m, rp, idx)))
    return mats, out, grfi


def main():
    if not O.ref_available():
        O.build(ref=True)
    mats, out, grfi = cases()
    arrays = {}
    meta = []
    for i, mt in enumerate(mats):
        for key, v in mt.items():
            arrays[f"mat{i:02d}/{key}"] = v
    for c in out:
        arrays[f"{c['name']}/y_ref"] = c["y_ref"]
        meta.append([c["name"], c["version"], c["mat"], c["m"], c["n"], c["nnz"], c["alpha"],
                     c["beta"], c["rc"], c["ngpu"], c["kernel"], c["nb"], c["q"]])
    np.savez_compressed(os.path.join(HERE, "dropin_cases.npz"), **arrays)
    with open(os.path.join(HERE, "dropin_cases.tsv"), "w") as f:
        f.write("name\tversion\tmat\tm\tn\tnnz\talpha\tbeta\trc\tngpu\tkernel\tnb\tq\n")
        for row in meta:
            f.write("\t".join(repr(v) if isinstance(v, float) else str(v) for v in row) + "\n")
    g = {"m": np.array([a[0] for a in grfi], np.int32),
         "idx": np.array([a[2] for a in grfi], np.int64),
         "row": np.array([a[3] for a in grfi], np.int32)}
    offs = np.zeros(len(grfi) + 1, np.int64)
    offs[1:] = np.cumsum([len(a[1]) for a in grfi])
    g["rowptr_flat"] = np.concatenate([a[1] for a in grfi])
    g["rowptr_off"] = offs
    np.savez_compressed(os.path.join(HERE, "get_row_from_index.npz"), **g)
    print(f"{len(meta)} drop-in cases, {len(grfi)} get_row_from_index answers")


if __name__ == "__main__":
    main()
