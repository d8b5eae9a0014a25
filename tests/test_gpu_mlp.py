"""Warm-start MLP kernels against the FP64 oracle (GPU)."""
import numpy as np
import pytest

from oracle import mlp as M

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def net():
    from fmm3dbie_b200.warmstart import WarmStartMLP, init_params
    p = init_params(3)
    rng = np.random.default_rng(4)
    p[M.NW:] = (0.05 * rng.normal(size=M.NPARAMS - M.NW)).astype(np.float32)
    n = WarmStartMLP(params=p, max_rows=4096)
    yield n, p.astype(np.float64)
    n.close()


def _batch(m, seed):
    rng = np.random.default_rng(seed)
    X = rng.uniform(-1, 1, (m, M.N_IN)).astype(np.float32)
    T = np.stack([np.sin(2 * X[:, 0] + X[:, 4]), np.cos(X[:, 1] * X[:, 5])], 1).astype(np.float32)
    return X, T


@pytest.mark.parametrize("m", [1, 200, 4096])
def test_forward_matches_oracle(net, m):
    import torch
    n, p = net
    X, _ = _batch(m, 10 + m)
    Y = n.forward(torch.from_numpy(X).cuda()).cpu().numpy()
    Ye, _ = M.forward(p, X.astype(np.float64), emulate_bf16=True)
    Yx, _ = M.forward(p, X.astype(np.float64))
    assert _rel(Y, Ye) < 2e-3
    assert _rel(Y, Yx) < 3e-2


@pytest.mark.parametrize("m", [130, 3000])
def test_gradient_matches_oracle(net, m):
    """Gradient check of the forward/backward kernels per parameter block:
    against the oracle with the same bf16 storage (kernel arithmetic) and
    against exact FP64 (size of the bf16 storage effect)."""
    import torch
    n, p = net
    X, T = _batch(m, 20 + m)
    G, loss = n.grad(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
    G = G.cpu().numpy().astype(np.float64)
    le, ge = M.loss_and_grad(p, X.astype(np.float64), T.astype(np.float64), emulate_bf16=True)
    lx, gx = M.loss_and_grad(p, X.astype(np.float64), T.astype(np.float64))
    assert abs(float(loss.item()) - le) <= 2e-3 * le
    blocks = [(o, a * b) for o, (a, b) in zip(M.OFF_W, M.SHAPE_W)] + \
             [(o, k) for o, k in zip(M.OFF_B, M.SHAPE_B)]
    for off, size in blocks:
        s = slice(off, off + size)
        assert _rel(G[s], ge[s]) < 1e-2, (off, _rel(G[s], ge[s]))
        assert _rel(G[s], gx[s]) < 6e-2, (off, _rel(G[s], gx[s]))


def test_adam_first_step(net):
    """First Adam step: p1 = p0 - lr * g / (|g| + eps) (bias-corrected moments)."""
    import torch
    from fmm3dbie_b200.warmstart import WarmStartMLP
    _, p = net
    n = WarmStartMLP(params=p.astype(np.float32), max_rows=512)
    X, T = _batch(512, 7)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    G, _ = n.grad(Xd, Td)
    p0 = n.params().cpu().numpy().astype(np.float64)
    g = G.cpu().numpy().astype(np.float64)
    n.train_step(Xd, Td, 1e-3)
    p1 = n.params().cpu().numpy().astype(np.float64)
    want = p0 - 1e-3 * g / (np.abs(g) + 1e-8)
    assert np.max(np.abs(p1 - want)) < 2e-6
    assert int(n.info()[6]) == 1
    n.close()


def test_training_reduces_loss():
    import torch
    from fmm3dbie_b200.warmstart import WarmStartMLP
    n = WarmStartMLP(seed=1, max_rows=2048)
    X, T = _batch(2048, 99)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    losses = torch.zeros(400, device="cuda")
    for it in range(400):
        n.train_step(Xd, Td, 2e-3, losses[it:it + 1])
    ls = losses.cpu().numpy()
    assert np.all(np.isfinite(ls))
    assert ls[-1] < 0.05 * ls[0], (ls[0], ls[-1])
    n.close()


def test_predict_density_matches_forward(net):
    """predict_density = forward on the gathered features, remodulated; the
    demodulation kernel inverts the modulation."""
    import torch
    from fmm3dbie_b200.warmstart import demodulate, torus_surface
    n, _ = net
    s = torus_surface(8, 4, 3)
    sv = torch.from_numpy(np.ascontiguousarray(s.srcvals)).cuda()
    rng = np.random.default_rng(5)
    d = rng.normal(size=(3, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    dirk = np.concatenate([d, np.array([[1.5], [4.0], [7.5]])], 1)
    x0 = n.predict_density(sv, dirk)
    xs, kc, ks = n.norm
    x = s.srcvals[:, 0:3]
    nrm = s.srcvals[:, 9:12]
    for q in range(3):
        F = np.concatenate([np.repeat(dirk[q:q + 1, :3], s.npts, 0),
                            np.full((s.npts, 1), (dirk[q, 3] - kc) / ks), x / xs, nrm], 1)
        Y = n.forward(torch.from_numpy(F.astype(np.float32)).cuda()).cpu().numpy()
        tau = Y[:, 0] + 1j * Y[:, 1]
        want = tau * np.exp(1j * dirk[q, 3] * (x @ dirk[q, :3]))
        got = x0[:, q].cpu().numpy()
        assert _rel(got, want) < 1e-6
    tau_back = torch.empty((3, s.npts), dtype=torch.complex64, device="cuda")
    demodulate(sv, dirk, x0.contiguous(), tau_back)
    for q in range(3):
        back = tau_back[q].cpu().numpy() * np.exp(1j * dirk[q, 3] * (x @ dirk[q, :3]))
        assert _rel(back, x0[:, q].cpu().numpy()) < 1e-6


@pytest.mark.parametrize("m", [128, 1000, 4096])
def test_tcgen05_forward_matches(net, m):
    """Hidden-layer forward on tcgen05 (tensor memory accumulator) against
    the mma.sync tiles and the oracle."""
    import torch
    n, p = net
    X, _ = _batch(m, 40 + m)
    Xd = torch.from_numpy(X).cuda()
    n.set_engine(0)
    Y0 = n.forward(Xd).cpu().numpy()
    n.set_engine(1)
    try:
        Y1 = n.forward(Xd).cpu().numpy()
        info = n.info()
    finally:
        n.set_engine(0)
    assert info[9] == 0, "tcgen05 completion wait timed out"
    Ye, _ = M.forward(p, X.astype(np.float64), emulate_bf16=True)
    assert _rel(Y1, Y0) < 1e-3
    assert _rel(Y1, Ye) < 2e-3
