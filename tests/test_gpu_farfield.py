"""bie_farfield_dev: the far-field sum (the lfmm3d/hfmm3d role) on device
buffers, against an FP64 numpy direct sum."""
import ctypes as C

import numpy as np
import pytest

from fmm3dbie_b200 import _lib as L

pytestmark = pytest.mark.gpu


def direct(kind, zk, src, nrm, ch, dp, targ, thresh):
    d = targ[:, None, :] - src[None, :, :]
    r2 = np.sum(d * d, 2)
    ok = r2 >= thresh * thresh
    r = np.sqrt(np.where(ok, r2, 1.0))
    dn = np.sum(d * nrm[None], 2)
    e = np.exp(1j * zk * r) if kind == 1 else 1.0
    k = (ch[None] / r + dp[None] * dn * (1 - 1j * zk * r) / r ** 3) * e / (4 * np.pi)
    return np.sum(np.where(ok, k, 0), 1)


def run(torch, kind, zk, src, nrm, ch, dp, targ, thresh, iprec, fn="bie_farfield_dev"):
    dev = "cuda"
    soa = lambda a: torch.tensor(np.ascontiguousarray(a.T), device=dev)  # noqa: E731
    s, n, t = soa(src), soa(nrm), soa(targ)
    if kind == 1:
        c = torch.tensor(ch.astype(complex), device=dev)
        d = torch.tensor(dp.astype(complex), device=dev)
        pot = torch.zeros(targ.shape[0], dtype=torch.complex128, device=dev)
    else:
        c = torch.tensor(ch.real, device=dev)
        d = torch.tensor(dp.real, device=dev)
        pot = torch.zeros(targ.shape[0], dtype=torch.float64, device=dev)
    z = np.array([zk.real, zk.imag])
    f = getattr(L.lib(), fn)
    st = f(kind, L.ptr(z), src.shape[0], C.c_void_p(s.data_ptr()), C.c_void_p(n.data_ptr()),
           C.c_void_p(c.data_ptr()), C.c_void_p(d.data_ptr()), targ.shape[0],
           C.c_void_p(t.data_ptr()), thresh, iprec, C.c_void_p(pot.data_ptr()),
           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    L.check(st, fn)
    torch.cuda.synchronize()
    return pot.cpu().numpy()


def problem(seed, ns=3000, nt=700):
    rng = np.random.default_rng(seed)
    src = rng.uniform(-1, 1, (ns, 3))
    nrm = rng.normal(size=(ns, 3))
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    ch = rng.normal(size=ns) + 1j * rng.normal(size=ns)
    dp = rng.normal(size=ns) + 1j * rng.normal(size=ns)
    targ = np.vstack([rng.uniform(-1.5, 1.5, (nt - 50, 3)), src[:50]])  # 50 coincident points
    return src, nrm, ch, dp, targ


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


@pytest.mark.parametrize("kind,zk", [(0, 0j), (1, 2.5 + 0j), (1, 1.5 + 0.3j), (1, 40.0 + 0j)])
def test_farfield_matches_direct_sum(torch, kind, zk):
    """zk = 40 puts k r up to ~200 (many quadrants of the FP64 sine/cosine
    reduction); the FP32 bound there reflects the phase error k r 2^-24."""
    src, nrm, ch, dp, targ = problem(1)
    thresh = 1e-14
    ref = direct(kind, zk, src, nrm, ch if kind else ch.real, dp if kind else dp.real, targ, thresh)
    got64 = run(torch, kind, zk, src, nrm, ch, dp, targ, thresh, 0)
    got32 = run(torch, kind, zk, src, nrm, ch, dp, targ, thresh, 1)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got64 - ref)) < 1e-12 * scale
    tol32 = 2e-5 if abs(zk) < 10 else 2e-4
    assert np.max(np.abs(got32 - ref)) < tol32 * scale


@pytest.mark.parametrize("kind,zk", [(0, 0j), (1, 2.5 + 0j), (1, 1.5 + 0.3j)])
def test_farfield_hierarchical(torch, kind, zk, monkeypatch):
    """Above the size threshold (forced here with BIE_FAR_METHOD=tree) the
    sum is evaluated hierarchically: within 1e-8 (FP64) and 1e-5 (FP32) of
    the direct sum, coincident source/target points included."""
    src, nrm, ch, dp, targ = problem(2, ns=40000, nt=30000)
    thresh = 1e-14
    monkeypatch.setenv("BIE_FAR_METHOD", "direct")
    ref = run(torch, kind, zk, src, nrm, ch, dp, targ, thresh, 0)
    monkeypatch.setenv("BIE_FAR_METHOD", "tree")
    for iprec, tol in ((0, 1e-8), (1, 1e-5)):
        got = run(torch, kind, zk, src, nrm, ch, dp, targ, thresh, iprec)
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        print(f"\nkind {kind} zk {zk} iprec {iprec}: tree vs direct {err:.2e}")
        assert err < tol
