"""CPU: the selector's host logic and the CPU restatement used to check the
GPU kernels (gradient check by finite differences)."""
import numpy as np

import mlp_cpu
from sbb import selector as S


def _random_problem(seed, N=40):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(N, S.N_FEATURES)).astype(np.float32) * 3 + 1
    times = np.exp(rng.normal(size=(N, S.N_CLASSES)))
    P = S.init_params(X, seed).astype(np.float64)
    return P, X, S.targets(times), S.sample_weights(times)


def test_cpu_gradient_matches_finite_differences():
    P, X, T, W = _random_problem(1)
    L, G = mlp_cpu.loss_grad(P, X, T, W)
    rng = np.random.default_rng(2)
    idx = rng.choice(np.arange(S.OFF["W1"], S.N_PARAMS), 60, replace=False)
    h = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (mlp_cpu.loss_grad(Pp, X, T, W)[0] - mlp_cpu.loss_grad(Pm, X, T, W)[0]) / (2 * h)
        assert abs(fd - G[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, G[i])
    assert np.all(G[:S.OFF["W1"]] == 0)


def test_targets_weights_and_regret():
    t = np.array([[2.0, 1.0, 4.0], [1.0, 3.0, 1.5]])
    assert np.allclose(S.targets(t), [[1, 0, 2], [0, np.log2(3), np.log2(1.5)]])
    assert np.allclose(S.sample_weights(t), [1.0, 1.0])
    assert S.regret(t, [1, 0]) == 0.0
    assert np.isclose(S.regret(t, [0, 2]), (2.0 + 1.5) / 2.0 - 1)


def test_heuristic_class_matches_plain_rule():
    assert S.heuristic_class(np.arange(0, 401, 4)) == 0          # 4 per row -> vector 4
    assert S.heuristic_class(np.arange(0, 2001, 20)) == 3        # 20 per row -> vector 32
    rp = np.concatenate([[0], np.cumsum([3] * 99 + [500])])       # one long row -> tiled
    assert S.heuristic_class(rp) == 5


def test_init_params_normalises_inputs():
    P, X, _, _ = _random_problem(3)
    v = S.unpack(P.astype(np.float32))
    Xn = (X - v["mu"]) / v["sd"]
    assert np.allclose(Xn.mean(0), 0, atol=1e-5) and np.allclose(Xn.std(0), 1, atol=1e-4)


def _committed():
    import os
    E = np.load(os.path.join(S.DATA_DIR, "eval_c5_seed5_512.npz"))
    return S.load_params(), E


def test_committed_selector_beats_the_default_heuristic():
    """The trained MLP (committed parameters) on the 512 held-out batch
    matrices, timed on a B200 when the data was collected: its classes' total
    time is within 2% of the exhaustive best, and its regret is under half of
    the default heuristic's ("no MLP")."""
    P, E = _committed()
    y, _ = mlp_cpu.forward(P, E["features"])
    mlp = np.argmin(y, axis=1)
    r_mlp, r_heur = S.regret(E["times_ms"], mlp), S.regret(E["times_ms"], E["heuristic"])
    assert r_mlp < 0.02 and r_mlp < 0.5 * r_heur, (r_mlp, r_heur)
    # the held-out set was not trained on
    T = np.load(f"{S.DATA_DIR}/train_c5_seed10000_4000.npz")
    assert int(T["seed_base"]) == 10000 and int(E["seed_base"]) == 5 and len(T["times_ms"]) == 4000


def test_committed_data_shapes():
    P, E = _committed()
    assert P.shape == (S.N_PARAMS,) and np.all(np.isfinite(P))
    assert E["features"].shape == (512, S.N_FEATURES) and E["times_ms"].shape == (512, 6)
    assert np.all(E["times_ms"] > 0)


def test_embedded_parameters_match_the_committed_file(tmp_path):
    """The build step that puts the trained parameters into libsbb (for
    SBB_KERNEL_LEARNED plans) writes every float exactly."""
    import os
    import re
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    script = os.path.join(here, "..", "sparse-blas_b200", "csrc", "gen", "embed_params.py")
    out = tmp_path / "p.inc"
    subprocess.run([sys.executable, script, S.PARAMS_PATH, str(out)], check=True)
    body = out.read_text().split("{", 1)[1]
    vals = np.array([float(v) for v in re.findall(r"([-+0-9.e]+)f", body)], np.float32)
    assert np.array_equal(vals, S.load_params())
