"""GPU: the selector's kernels against the float64 CPU restatement
(tests/mlp_cpu.py): feature kernel, forward pass, gradient check of the
backward pass, deterministic training, on-GPU selection."""
import numpy as np
import pytest

import mlp_cpu
from helpers import rand_csr
from sbb import selector as S

pytestmark = pytest.mark.gpu


def _dev_csr(rp, col, m, n):
    import torch
    return dict(m=m, n=n, rowptr=torch.from_numpy(np.asarray(rp, np.int32)).cuda(),
                col=torch.from_numpy(np.asarray(col, np.int32)).cuda())


def _problem(seed, N=300):
    rng = np.random.default_rng(seed)
    X = (rng.normal(size=(N, S.N_FEATURES)) * 3 + 1).astype(np.float32)
    times = np.exp(rng.normal(size=(N, S.N_CLASSES)))
    return S.init_params(X, seed), X, S.targets(times), S.sample_weights(times), times


@pytest.mark.parametrize("case", range(4))
def test_feature_kernel_matches_cpu(cuda, case):
    from sbb import gen
    if case < 3:
        m, n = (1000, 700, 3000)[case], (800, 5000, 3000)[case]
        rp, col, _, _, _ = rand_csr(10 + case, m, n, 0, (6, 40, 300)[case], p_empty=0.1 * case,
                                    long_rows=[(5, min(n, 2000))] if case == 2 else [])
    else:
        A = gen.c5(3)
        rp, col, m, n = A.rowptr, A.col, A.m, A.n
    got = S.features(_dev_csr(rp, col, m, n))
    want = mlp_cpu.features(rp, col, m, n)
    assert np.allclose(got, want, rtol=2e-6, atol=1e-6), (got, want)


def test_forward_matches_cpu(cuda):
    P, X, _, _, _ = _problem(1)
    want, _ = mlp_cpu.forward(P, X)
    got = S.predict(P, X)
    assert np.allclose(got, want, rtol=1e-4, atol=1e-4)


def test_gradient_check_against_cpu(cuda):
    """GPU loss and gradient (FP32 kernels) vs the float64 restatement, whose
    own gradient is checked by finite differences in test_selector.py."""
    P, X, T, W, _ = _problem(2)
    for w in (W, None):
        L, G = S.grad(P, X, T, w)
        Lc, Gc = mlp_cpu.loss_grad(P, X, T, w)
        assert abs(L - Lc) <= 1e-4 * abs(Lc)
        assert np.linalg.norm(G - Gc) <= 1e-4 * np.linalg.norm(Gc)
        assert np.allclose(G, Gc, rtol=1e-3, atol=1e-5 * np.abs(Gc).max())
        assert np.all(G[:S.OFF["W1"]] == 0)


def test_training_reduces_loss_and_is_deterministic(cuda):
    _, X, _, _, times = _problem(3)
    P1, h1 = S.train(X, times, steps=300, lr=3e-3)
    P2, h2 = S.train(X, times, steps=300, lr=3e-3)
    assert np.array_equal(P1, P2) and np.array_equal(h1, h2)
    assert h1[-1] < 0.5 * h1[0]
    # the GPU loss history agrees with the CPU loss of the final parameters'
    # predecessor only up to FP32; check the final parameters' CPU loss instead
    Lc, _ = mlp_cpu.loss_grad(P1, X, S.targets(times), S.sample_weights(times))
    assert Lc <= h1[-1] * 1.05 + 1e-6


def test_select_on_gpu_matches_cpu_argmin(cuda):
    from sbb import gen
    P = S.init_params(np.random.default_rng(4).normal(size=(50, S.N_FEATURES)), 4)
    sel = S.Selector(P)
    checked = 0
    for i in range(8):
        A = gen.c5(i, 77)
        d = _dev_csr(A.rowptr32(), A.col, A.m, A.n)
        y, _ = mlp_cpu.forward(P, mlp_cpu.features(A.rowptr, A.col, A.m, A.n)[None, :])
        s = np.sort(y[0])
        if s[1] - s[0] <= 1e-3 * max(1.0, abs(s[0])):
            continue  # a near-tie: FP32 and FP64 may order it either way
        assert sel.select(d) == int(np.argmin(y[0]))
        checked += 1
    assert checked >= 4


def test_gpu_forward_reproduces_committed_choices(cuda):
    """The GPU forward pass picks the same classes as the float64 CPU
    restatement on the committed held-out features (ties aside)."""
    import os
    E = np.load(os.path.join(S.DATA_DIR, "eval_c5_seed5_512.npz"))
    P = S.load_params()
    y_cpu, _ = mlp_cpu.forward(P, E["features"])
    y_gpu = S.predict(P, E["features"])
    assert np.allclose(y_gpu, y_cpu, rtol=1e-4, atol=1e-4)
    srt = np.sort(y_cpu, axis=1)
    clear = srt[:, 1] - srt[:, 0] > 1e-3
    assert np.array_equal(np.argmin(y_gpu, 1)[clear], np.argmin(y_cpu, 1)[clear])


def test_learned_plan_uses_the_selector_and_matches_oracle(cuda):
    """A SBB_KERNEL_LEARNED plan runs the built-in trained parameters on the
    GPU: it resolves to the class the selector picks (same configuration as
    that batch class) and its result matches the oracle."""
    import torch
    import oracle as O
    from helpers import TOL_FP64, max_scaled_err
    from sbb import gen
    from sbb.device import Plan
    sel = S.Selector()  # the committed parameters, the ones built into the library
    want_cfg = {0: (1, 4), 1: (1, 8), 2: (1, 16), 3: (1, 32), 4: (2, 6), 5: (3, 4)}
    seen = set()
    for i in range(9):
        A = gen.c5(i, 31)
        d = _dev_csr(A.rowptr32(), A.col, A.m, A.n)
        cls = sel.select(d)
        seen.add(cls)
        x = gen.uniform_vec(7 + i, A.n)
        y = gen.uniform_vec(8 + i, A.m)
        P = Plan(d["rowptr"], d["col"], torch.from_numpy(A.val).cuda(), A.n, kernel="learned")
        info = P.info()
        k, knob = want_cfg[cls]
        assert info["kernel"] == k
        assert knob == {1: info["vector_width"], 2: info["items_per_thread"],
                        3: info["tile_sigma"]}[k]
        yy = torch.from_numpy(y).cuda()
        P.spmv(torch.from_numpy(x).cuda(), yy, 1.0, 0.5)
        torch.cuda.synchronize()
        P.check()
        P.close()
        ref, sc = O.spmv_dd(A.rowptr, A.col, A.val, x, 1.0, 0.5, y)
        assert max_scaled_err(yy.cpu().numpy(), ref, sc) <= TOL_FP64
    assert len(seen) >= 2  # the matrices reach more than one class
