"""The FP64 MLP oracle pinned by central finite differences (CPU)."""
import numpy as np

from oracle import mlp as M


def _small_problem(seed=0, m=24):
    rng = np.random.default_rng(seed)
    p = np.zeros(M.NPARAMS)
    for off, (a, b) in zip(M.OFF_W, M.SHAPE_W):
        p[off:off + a * b] = rng.uniform(-1, 1, a * b) * np.sqrt(6.0 / (a + b))
    for off, n in zip(M.OFF_B, M.SHAPE_B):
        p[off:off + n] = 0.1 * rng.normal(size=n)
    X = rng.normal(size=(m, M.N_IN))
    T = rng.normal(size=(m, M.N_OUT))
    return rng, p, X, T


def test_layout_sizes():
    assert M.NPARAMS == 200706
    assert M.NW == 199680
    assert M.OFF_B[0] == M.NW


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, -2.5, 3.0e-3])
    r = M.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0)
    assert r[0] == 1.0 and r[1] == 1.0
    assert r[2] == 1.0 + 2.0 ** -7
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 3.0e-3 * 2.0 ** -8


def test_gradient_matches_finite_differences():
    rng, p, X, T = _small_problem()
    loss, g = M.loss_and_grad(p, X, T)
    # a few entries of every weight matrix and bias vector
    idx = []
    for off, (a, b) in zip(M.OFF_W, M.SHAPE_W):
        idx += list(off + rng.choice(a * b, 6, replace=False))
    for off, n in zip(M.OFF_B, M.SHAPE_B):
        idx += list(off + rng.choice(n, 2, replace=False))
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (M.loss_and_grad(p + e, X, T)[0] - M.loss_and_grad(p - e, X, T)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-6 * abs(g[i]), (i, fd, g[i])


def test_emulated_gradient_close_to_exact():
    _, p, X, T = _small_problem(1, 64)
    _, g = M.loss_and_grad(p, X, T)
    _, gb = M.loss_and_grad(p, X, T, emulate_bf16=True)
    assert np.linalg.norm(gb - g) <= 0.05 * np.linalg.norm(g)
