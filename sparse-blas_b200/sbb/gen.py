"""Seeded synthetic CSR matrices for the benchmark and test configurations.

The reference quotes its results on SuiteSparse matrices (circuit5M,
rail4284, ASIC_680k) that are not available here; these seeded families stand
in for them with the shapes, sizes and value distributions of the benchmark
configurations:

* ``c1``  n = 10,000 square; row lengths from a truncated power law
          (density ~ L^-2 on [1, 1000], floored), sorted distinct uniform
          columns; val, x ~ U(-1,1); alpha = 1, beta = 0.
* ``c2``  n = 5.5M square, circuit-like: diagonal + band of half-width 8
          (each off-diagonal slot kept with p = 0.43) + ceil(Pareto(alpha=2) on
          [1, 1000]) uniform long-range columns; 550 dense rows (0.01 %) with
          lengths Pareto(alpha=2) on [1e3, 1e6], one forced to 1,000,000;
          nnz ~ 60M; val, x, y ~ U(-1,1); beta = 0.5.
* ``c3``  4,284 x 1,092,610; log-normal row lengths (mean 2,640, sigma 1.0),
          columns as contiguous runs inside random 64-aligned blocks; all
          values 1.0; x ~ U(-1,1).
* ``c5``  512 matrices, n log-uniform in [1k, 200k], banded / power-law /
          block-diagonal families in equal thirds, nnz/row log-uniform in
          [4, 200]; matrix i uses seed 5+i (training set: 10000+i).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from ._lib import GenParams, gen

POWERLAW, CIRCUIT, SHORTWIDE, BANDED, PLFAMILY, BLOCKDIAG, UNIFORM = 1, 2, 3, 4, 5, 6, 7


@dataclass
class Csr:
    m: int
    n: int
    rowptr: np.ndarray   # int64, m+1
    col: np.ndarray      # int32
    val: np.ndarray      # float64
    name: str = ""

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def rowptr32(self) -> np.ndarray:
        return self.rowptr.astype(np.int32)

    def row_lengths(self) -> np.ndarray:
        return np.diff(self.rowptr)


def _vp(a):
    return a.ctypes.data_as(C.c_void_p)


def generate(p: GenParams, name: str = "") -> Csr:
    G = gen()
    rowptr = np.empty(p.m + 1, np.int64)
    nnz = G.sbbgen_rowptr(C.byref(p), _vp(rowptr))
    col = np.empty(nnz, np.int32)
    val = np.empty(nnz, np.float64)
    G.sbbgen_fill(C.byref(p), _vp(rowptr), _vp(col), _vp(val))
    return Csr(p.m, p.n, rowptr, col, val, name)


def uniform_vec(seed: int, n: int, lo=-1.0, hi=1.0) -> np.ndarray:
    out = np.empty(n, np.float64)
    gen().sbbgen_uniform(seed, n, lo, hi, _vp(out))
    return out


def params(**kw) -> GenParams:
    p = GenParams()
    defaults = dict(seed=1, family=UNIFORM, m=0, n=0, expo=2.0, lmin=1.0, lmax=1000.0, p=0.0,
                    hw=0, block=0, r=0.0, mu=0.0, sigma=0.0, ndense=0, dense_lo=0.0,
                    dense_hi=0.0, dense_expo=3.0, p_empty=0.0, unit_values=0)
    defaults.update(kw)
    for k, v in defaults.items():
        setattr(p, k, v)
    return p


def c1(seed=1, n=10_000) -> Csr:
    return generate(params(seed=seed, family=POWERLAW, m=n, n=n, expo=2.0, lmin=1.0,
                           lmax=1000.0), "c1_powerlaw_10k")


def c2(seed=2, n=5_500_000, p_band=0.43, ndense=550) -> Csr:
    return generate(params(seed=seed, family=CIRCUIT, m=n, n=n, hw=8, p=p_band, expo=3.0,
                           lmin=1.0, lmax=1000.0, ndense=ndense, dense_lo=1e3,
                           dense_hi=1e6, dense_expo=3.0), "c2_circuit_5.5M")


def c3(seed=3, m=4284, n=1_092_610) -> Csr:
    return generate(params(seed=seed, family=SHORTWIDE, m=m, n=n, mu=math.log(2640.0) - 0.5,
                           sigma=1.0, unit_values=1), "c3_shortwide_4284x1.09M")


def uniform(seed, m, n, lmin=0, lmax=8, p_empty=0.0) -> Csr:
    return generate(params(seed=seed, family=UNIFORM, m=m, n=n, lmin=lmin, lmax=lmax,
                           p_empty=p_empty), f"uniform_{m}x{n}")


def _pl_xmin(expo: float, r: float, lmax: float) -> float:
    """xmin so that the power law ~x^-expo on [xmin, lmax] has mean r."""
    def mean(a):
        b = lmax
        if abs(expo - 1) < 1e-9:
            return (b - a) / math.log(b / a)
        if abs(expo - 2) < 1e-9:
            return math.log(b / a) / (1 / a - 1 / b)
        k1, k2 = 1 - expo, 2 - expo
        return (k1 / k2) * (b ** k2 - a ** k2) / (b ** k1 - a ** k1)
    lo, hi = 1e-3, min(r, lmax) * 0.999999
    for _ in range(100):
        mid = math.sqrt(lo * hi)
        if mean(mid) < r:
            lo = mid
        else:
            hi = mid
    return max(1.0, math.sqrt(lo * hi))


def c5_params(i: int, seed_base: int = 5):
    """Parameters of matrix i of the batch (seed_base 5) or training set (10000)."""
    rng = np.random.default_rng(seed_base + i)
    n = int(round(math.exp(rng.uniform(math.log(1e3), math.log(2e5)))))
    r = float(math.exp(rng.uniform(math.log(4.0), math.log(200.0))))
    fam = i % 3
    seed = seed_base + i
    if fam == 0:
        hw = int(rng.integers(1, 65))
        return params(seed=seed, family=BANDED, m=n, n=n, hw=hw, r=r)
    if fam == 1:
        e = float(rng.uniform(1.5, 3.0))
        lmax = float(min(n, 50.0 * r))
        xmin = _pl_xmin(e, r, lmax)
        return params(seed=seed, family=PLFAMILY, m=n, n=n, expo=e, lmin=xmin, lmax=lmax)
    b = int(rng.integers(16, 257))
    return params(seed=seed, family=BLOCKDIAG, m=n, n=n, block=b, r=r)


def c5(i: int, seed_base: int = 5) -> Csr:
    fams = {0: "banded", 1: "powerlaw", 2: "blockdiag"}
    return generate(c5_params(i, seed_base), f"c5_{fams[i % 3]}_{i}")
