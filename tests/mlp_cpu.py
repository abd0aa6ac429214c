"""CPU (numpy, float64) restatement of the selector's MLP and features.

Test infrastructure only: the gradient check of the GPU forward / backward
kernels (csrc/kernels/k_mlp.cu) and of the feature kernel compares against
these functions.
"""
import numpy as np

from sbb.selector import N_PARAMS, OFF, unpack


def forward(P, X):
    v = unpack(np.asarray(P, np.float64), np.float64)
    sd = np.where(v["sd"] > 0, v["sd"], 1.0)
    Xn = (np.asarray(X, np.float64) - v["mu"]) / sd
    Z1 = Xn @ v["W1"].T + v["b1"]
    H1 = np.maximum(Z1, 0.0)
    Z2 = H1 @ v["W2"].T + v["b2"]
    H2 = np.maximum(Z2, 0.0)
    Y = H2 @ v["W3"].T + v["b3"]
    return Y, (v, Xn, Z1, H1, Z2, H2)


def loss_grad(P, X, T, W=None):
    """L = sum_n w_n sum_c (Y - T)^2 / (C sum_n w_n) and dL/dP (zero for the
    normalisation entries)."""
    Y, (v, Xn, Z1, H1, Z2, H2) = forward(P, X)
    N, C = Y.shape
    w = np.ones(N) if W is None else np.asarray(W, np.float64)
    inv = 1.0 / (C * w.sum())
    E = Y - np.asarray(T, np.float64)
    L = float((w[:, None] * E * E).sum() * inv)
    dY = 2.0 * inv * w[:, None] * E
    dZ2 = (dY @ v["W3"]) * (Z2 > 0)
    dZ1 = (dZ2 @ v["W2"]) * (Z1 > 0)
    G = np.zeros(N_PARAMS)
    out = {"W1": dZ1.T @ Xn, "b1": dZ1.sum(0), "W2": dZ2.T @ H1, "b2": dZ2.sum(0),
           "W3": dY.T @ H2, "b3": dY.sum(0)}
    for k, a in out.items():
        G[OFF[k]:OFF[k] + a.size] = a.ravel()
    return L, G


def features(rowptr, col, m, n):
    rp = np.asarray(rowptr, np.int64)
    L = np.diff(rp).astype(np.float64)
    nnz = float(rp[-1] - rp[0])
    M = max(m, 1)
    mean = nnz / M
    var = max(float((L * L).sum()) / M - mean * mean, 0.0)
    mx = float(L.max()) if m else 0.0
    ne = L > 0
    c = np.asarray(col, np.int64)
    first = c[rp[:-1][ne]]
    last = c[rp[1:][ne] - 1]
    span = float((np.abs(last - first) + 1).sum())
    n_ne = max(int(ne.sum()), 1)
    return np.array([
        np.log2(1 + m), np.log2(1 + n), np.log2(1 + nnz), np.log2(1 + mean),
        np.sqrt(var) / mean if mean > 0 else 0.0, np.log2(1 + mx),
        np.log2(1 + (mx / mean if mean > 0 else 0.0)), float((L == 0).sum()) / M,
        float((L <= 4).sum()) / M, float((L > 32).sum()) / M,
        float(L[L > 128].sum()) / nnz if nnz > 0 else 0.0, span / n_ne / max(n, 1)])
