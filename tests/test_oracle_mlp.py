"""The oracle of the step-size perceptron (oracle/mlp.c) pinned on the CPU: its
hand-written backward pass against central differences of its own loss in
binary64, and its binary16 mode close to binary64."""
import numpy as np


def _problem(seed=0, n=48):
    rng = np.random.default_rng(seed)
    import oracle
    npar = oracle.lib().orc_mlp_nparam()
    P = (rng.standard_normal(npar) * 0.2).astype(np.float32)
    norm = np.concatenate([rng.standard_normal(11), np.abs(rng.standard_normal(11)) + 0.5, [0.3, 1.7]])
    X = rng.standard_normal((n, 11)).astype(np.float32)
    Y = rng.standard_normal(n).astype(np.float32)
    return P, norm.astype(np.float32), X, Y


def test_mlp_backward_matches_finite_differences(oracle_lib):
    P, norm, X, Y = _problem()
    loss, g = oracle_lib.mlp_loss_grad(P, norm, X, Y, fp16=False)
    assert loss > 0
    rng = np.random.default_rng(1)
    # every block of parameters: W1, b1, W2, b2, W3, b3, W4, b4
    picks = [3, 700, 705, 2000, 4870, 6000, 9030, 9100, 9152] + list(rng.integers(0, len(P), 12))
    for p in picks:
        a, b = P.copy(), P.copy()
        a[p] += 1e-3
        b[p] -= 1e-3
        la, _ = oracle_lib.mlp_loss_grad(a, norm, X, Y, fp16=False, grad=False)
        lb, _ = oracle_lib.mlp_loss_grad(b, norm, X, Y, fp16=False, grad=False)
        fd = (la - lb) / (np.float64(a[p]) - np.float64(b[p]))
        assert abs(fd - g[p]) <= 1e-5 * max(1.0, abs(g[p])) + 1e-7, (p, fd, g[p])


def test_mlp_fp16_mode_close_to_binary64(oracle_lib):
    P, norm, X, Y = _problem(2)
    l16, g16 = oracle_lib.mlp_loss_grad(P, norm, X, Y, fp16=True)
    l64, g64 = oracle_lib.mlp_loss_grad(P, norm, X, Y, fp16=False)
    assert abs(l16 - l64) < 1e-2 * l64
    assert np.linalg.norm(g16 - g64) < 2e-2 * np.linalg.norm(g64)
    y16 = oracle_lib.mlp_predict(P, norm, X, fp16=True)
    y64 = oracle_lib.mlp_predict(P, norm, X, fp16=False)
    assert np.max(np.abs(y16 - y64)) < 2e-2 * np.max(np.abs(y64))
