"""Shared test helpers: golden-fixture access and random CSR builders."""
from __future__ import annotations

import csv
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Per-row tolerance of the FP64 path against the accurate oracle:
# |y - y_ref| <= TOL_FP64 * (|alpha| * sum_j |a_ij x_j| + |beta y_i|).
TOL_FP64 = 1e-12
# FP32-storage form against the FP64 oracle, same scaling.
TOL_FP32 = 1e-6


def golden_cases():
    """List of dicts, one per drop-in fixture, with arrays attached."""
    data = np.load(os.path.join(GOLDEN, "dropin_cases.npz"))
    out = []
    with open(os.path.join(GOLDEN, "dropin_cases.tsv")) as f:
        for row in csv.DictReader(f, delimiter="\t"):
            c = dict(name=row["name"], version=row["version"], m=int(row["m"]), n=int(row["n"]),
                     nnz=int(row["nnz"]), alpha=float(row["alpha"]), beta=float(row["beta"]),
                     rc=int(row["rc"]), ngpu=int(row["ngpu"]), kernel=int(row["kernel"]),
                     nb=int(row["nb"]), q=int(row["q"]))
            mat = f"mat{int(row['mat']):02d}"
            for key in ("rowptr", "col", "val", "x", "y"):
                c[key] = data[f"{mat}/{key}"]
            c["y_ref"] = data[f"{c['name']}/y_ref"]
            out.append(c)
    return out


def golden_grfi():
    g = np.load(os.path.join(GOLDEN, "get_row_from_index.npz"))
    off = g["rowptr_off"]
    flat = g["rowptr_flat"]
    for i in range(len(g["m"])):
        yield int(g["m"][i]), flat[off[i]:off[i + 1]].copy(), int(g["idx"][i]), int(g["row"][i])


def rand_csr(seed, m, n, lmin=0, lmax=8, p_empty=0.0, long_rows=()):
    """Random CSR (int64 rowptr) with optional empty rows and long rows.

    long_rows: iterable of (row, length) forced lengths (length <= n).
    """
    rng = np.random.default_rng(seed)
    lens = rng.integers(lmin, lmax + 1, m) if m else np.zeros(0, np.int64)
    if m:
        lens[rng.random(m) < p_empty] = 0
    for r, L in long_rows:
        lens[r] = L
    lens = np.minimum(lens, n)
    rp = np.zeros(m + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    cols = []
    for L in lens:
        if L == 0:
            continue
        if L * 4 > n:
            c = np.sort(rng.choice(n, L, replace=False))
        else:
            c = np.unique(rng.integers(0, n, L + L // 4 + 4))[:L]
            while len(c) < L:
                c = np.unique(np.concatenate([c, rng.integers(0, n, L)]))[:L]
        cols.append(c)
    col = (np.concatenate(cols) if cols else np.zeros(0)).astype(np.int32)
    val = rng.uniform(-1, 1, int(rp[-1]))
    x = rng.uniform(-1, 1, n)
    y = rng.uniform(-1, 1, m)
    return rp, col, val, x, y


def max_scaled_err(y, y_ref, scale):
    d = np.abs(np.asarray(y) - y_ref)
    s = np.where(scale > 0, scale, 1.0)
    e = np.where(scale > 0, d / s, np.where(d == 0, 0.0, np.inf))
    return float(e.max()) if e.size else 0.0
