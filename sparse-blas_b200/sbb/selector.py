"""Learned kernel-class selector: GPU features, an FP32 MLP trained on GPU.

The MLP (12 features -> 64 -> 64 -> 6, ReLU; parameter layout in
``include/sbb_spmv.h``) predicts, for each kernel class of the batched form
(``sbb.batch.CLASS_NAMES``), log2(t_class / t_best) of the class's plain
launch on the matrix, and the selector takes the class with the smallest
prediction.  Every step runs in the library's own CUDA kernels: the feature
kernel, the forward pass, the backward pass (per-sample error terms, then
per-parameter sums in a fixed sample order) and Adam.

Training data: timings of every class on 4,000 seeded matrices of the batch
families (``sbb.gen.c5_params(i, 10000)``), collected by ``collect`` with the
exhaustive class timer (``sbb.batch.tune``).  Regret of a choice over a set of
matrices = sum of the chosen classes' times / sum of the best times - 1.

    python -m sbb.selector collect --count 4000 --seed-base 10000 --out train.npz
    python -m sbb.selector train --data train.npz --out mlp_params.npy
"""
from __future__ import annotations

import argparse
import ctypes as C
import math
import os
import time

import numpy as np

from ._lib import last_error, lib

HERE = os.path.dirname(os.path.abspath(__file__))
DATA_DIR = os.path.join(HERE, "selector_data")
PARAMS_PATH = os.path.join(DATA_DIR, "mlp_params.npy")

N_FEATURES, N_HIDDEN, N_CLASSES = 12, 64, 6
_F, _H, _C = N_FEATURES, N_HIDDEN, N_CLASSES
OFF = {"mu": 0, "sd": _F, "W1": 2 * _F}
OFF["b1"] = OFF["W1"] + _H * _F
OFF["W2"] = OFF["b1"] + _H
OFF["b2"] = OFF["W2"] + _H * _H
OFF["W3"] = OFF["b2"] + _H
OFF["b3"] = OFF["W3"] + _C * _H
N_PARAMS = OFF["b3"] + _C
assert N_PARAMS == 5406


class SelectorError(RuntimeError):
    pass


def _ok(rc, what):
    if rc != 0:
        raise SelectorError(f"{what} failed ({rc}): {last_error()}")


def _stream(stream=None):
    import torch
    return C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def unpack(params, dtype=np.float32):
    """Views of the parameter blob: dict of mu, sd, W1, b1, W2, b2, W3, b3."""
    P = np.asarray(params, dtype)
    shapes = {"mu": (_F,), "sd": (_F,), "W1": (_H, _F), "b1": (_H,), "W2": (_H, _H),
              "b2": (_H,), "W3": (_C, _H), "b3": (_C,)}
    return {k: P[OFF[k]:OFF[k] + int(np.prod(s))].reshape(s) for k, s in shapes.items()}


def heuristic_class(rowptr):
    """The plain path's default choice (default_kernel_choice in
    csrc/host/plan.cpp) restricted to the batch classes: vector CSR with V =
    the next power of two >= the mean row length (4..32) when rows are short
    and even, the sigma = 4 tiles otherwise.  The "no MLP" baseline."""
    L = np.diff(np.asarray(rowptr, np.int64))
    mean = float(L.mean()) if len(L) else 0.0
    v, cls = 4, 0
    while v < 32 and v < mean:
        v <<= 1
        cls += 1
    mx = int(L.max()) if len(L) else 0
    return cls if (mx <= 4 * v and mx <= 128) else 5


def features(d, stream=None):
    """The 12 features of matrix d (dict with torch CUDA tensors rowptr, col
    and ints m, n), computed by the GPU feature kernel."""
    import torch
    out = torch.empty(_F, dtype=torch.float32, device=d["rowptr"].device)
    _ok(lib().sbb_features(d["m"], d["n"], d["col"].numel(), _p(d["rowptr"]), _p(d["col"]),
                           _p(out), _stream(stream)), "sbb_features")
    return out.cpu().numpy()


def targets(times):
    """log2(t_class / t_best) per matrix (the regression targets)."""
    t = np.asarray(times, np.float64)
    return np.log2(t / t.min(axis=1, keepdims=True)).astype(np.float32)


def sample_weights(times):
    """Weight of each matrix in the loss: its best time over the mean best
    time, so the fit follows the total time of a set (what regret measures)."""
    b = np.asarray(times, np.float64).min(axis=1)
    return (b / b.mean()).astype(np.float32)


def regret(times, classes):
    t = np.asarray(times, np.float64)
    return float(t[np.arange(len(t)), np.asarray(classes)].sum() / t.min(axis=1).sum() - 1.0)


def init_params(X, seed=0):
    """Input normalisation from the training features; He-uniform weights
    from a seeded generator; zero biases."""
    X = np.asarray(X, np.float64)
    rng = np.random.default_rng(seed)
    P = np.zeros(N_PARAMS, np.float32)
    v = unpack(P)
    v["mu"][:] = X.mean(axis=0)
    sd = X.std(axis=0)
    v["sd"][:] = np.where(sd > 1e-6, sd, 1.0)
    for k, fan_in in (("W1", _F), ("W2", _H), ("W3", _H)):
        lim = math.sqrt(6.0 / fan_in)
        v[k][:] = rng.uniform(-lim, lim, v[k].shape)
    return P


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def predict(params, X, stream=None):
    """Scores [N, 6] of the MLP on features X [N, 12] (GPU forward pass)."""
    import torch
    X = np.asarray(X, np.float32).reshape(-1, _F)
    P, Xd = _dev(params), _dev(X)
    Y = torch.empty((len(X), _C), dtype=torch.float32, device="cuda")
    _ok(lib().sbb_mlp_forward(_p(P), _p(Xd), len(X), _p(Y), _stream(stream)), "sbb_mlp_forward")
    return Y.cpu().numpy()


def choose(params, X):
    return np.argmin(predict(params, X), axis=1)


def grad(params, X, T, W=None, stream=None):
    """(loss, gradient) of the weighted MSE on the GPU."""
    import torch
    P, Xd, Td = _dev(params), _dev(X), _dev(T)
    Wd = _dev(W) if W is not None else None
    G = torch.empty(N_PARAMS, dtype=torch.float32, device="cuda")
    L = torch.empty(1, dtype=torch.float32, device="cuda")
    _ok(lib().sbb_mlp_grad(_p(P), _p(Xd), _p(Td), _p(Wd), len(X), _p(G), _p(L), _stream(stream)),
        "sbb_mlp_grad")
    return float(L.item()), G.cpu().numpy()


def train(X, times, steps=4000, lr=3e-3, wd=1e-4, seed=0, weighted=True, stream=None):
    """Full-batch Adam on the GPU from init_params(X, seed); returns the
    parameters and the loss of every step."""
    import torch
    X = np.asarray(X, np.float32)
    P = _dev(init_params(X, seed))
    Xd, Td = _dev(X), _dev(targets(times))
    Wd = _dev(sample_weights(times)) if weighted else None
    hist = torch.empty(steps, dtype=torch.float32, device="cuda")
    _ok(lib().sbb_mlp_train(_p(P), _p(Xd), _p(Td), _p(Wd), len(X), steps, lr, wd, _p(hist),
                            _stream(stream)), "sbb_mlp_train")
    return P.cpu().numpy(), hist.cpu().numpy()


def load_params(path=None):
    P = np.load(path or PARAMS_PATH).astype(np.float32)
    if P.shape != (N_PARAMS,):
        raise SelectorError(f"parameter file has shape {P.shape}, expected ({N_PARAMS},)")
    return P


class Selector:
    """Picks a batch class per matrix with the trained MLP, on the GPU."""

    def __init__(self, params=None):
        self.params = load_params() if params is None else np.asarray(params, np.float32)
        self._P = _dev(self.params)

    def select(self, d, stream=None):
        out = C.c_int(-1)
        _ok(lib().sbb_mlp_select(_p(self._P), d["m"], d["n"], d["col"].numel(), _p(d["rowptr"]),
                                 _p(d["col"]), C.byref(out), _stream(stream)), "sbb_mlp_select")
        return int(out.value)


def collect(count, seed_base, reps=5, log_every=250):
    """Features (GPU kernel), class timings (sbb.batch.tune, `reps` runs after
    a warm-up) and the heuristic's class of matrices c5_params(i, seed_base),
    i < count, with x, y ~ U(-1, 1), alpha = 1, beta = 0.5."""
    import torch
    from . import gen
    from .batch import tune
    feats, times, heur, nnz = [], [], [], []
    t0 = time.time()
    for i in range(count):
        A = gen.c5(i, seed_base)
        d = dict(m=A.m, n=A.n, alpha=1.0, beta=0.5,
                 rowptr=torch.from_numpy(A.rowptr32()).cuda(), col=torch.from_numpy(A.col).cuda(),
                 val=torch.from_numpy(A.val).cuda(),
                 x=torch.from_numpy(gen.uniform_vec(seed_base + 7 * i + 1, A.n)).cuda(),
                 y=torch.from_numpy(gen.uniform_vec(seed_base + 7 * i + 2, A.m)).cuda())
        feats.append(features(d))
        times.append(tune(d, reps=reps))
        heur.append(heuristic_class(A.rowptr))
        nnz.append(A.nnz)
        if log_every and (i + 1) % log_every == 0:
            print(f"collect: {i + 1}/{count} matrices, {time.time() - t0:.0f} s", flush=True)
    return {"features": np.array(feats, np.float32), "times_ms": np.array(times, np.float32),
            "heuristic": np.array(heur, np.int32), "nnz": np.array(nnz, np.int64),
            "seed_base": np.int64(seed_base), "reps": np.int64(reps),
            "gpu": np.array(torch.cuda.get_device_name())}


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m sbb.selector")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--count", type=int, default=4000)
    c.add_argument("--seed-base", type=int, default=10000)
    c.add_argument("--reps", type=int, default=5)
    c.add_argument("--out", required=True)
    t = sub.add_parser("train")
    t.add_argument("--data", required=True)
    t.add_argument("--eval", default=None, help="held-out timings (npz from collect)")
    t.add_argument("--steps", type=int, default=4000)
    t.add_argument("--lr", type=float, default=3e-3)
    t.add_argument("--wd", type=float, default=1e-4)
    t.add_argument("--seed", type=int, default=0)
    t.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    if a.cmd == "collect":
        np.savez_compressed(a.out, **collect(a.count, a.seed_base, a.reps))
        return
    D = np.load(a.data)
    P, hist = train(D["features"], D["times_ms"], a.steps, a.lr, a.wd, a.seed)
    np.save(a.out, P)
    print(f"loss {hist[0]:.4f} -> {hist[-1]:.4f}; train regret "
          f"mlp {regret(D['times_ms'], choose(P, D['features'])):.4f} "
          f"heuristic {regret(D['times_ms'], D['heuristic']):.4f}")
    if a.eval:
        E = np.load(a.eval)
        print(f"eval regret mlp {regret(E['times_ms'], choose(P, E['features'])):.4f} "
              f"heuristic {regret(E['times_ms'], E['heuristic']):.4f}")


if __name__ == "__main__":
    main()
