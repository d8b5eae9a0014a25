"""Uneven batches of surfaces (32-ellipsoid shape, reduced).  The streams
engine: each surface's solve on its own stream equals the same solve run
alone.  The graph engine (all surfaces in one persistent launch per matvec
stage, replayed from a CUDA graph): its matvec equals the surfaces' own plans,
graph and plain launches agree exactly, and its solves match the streams
engine."""
import numpy as np
import pytest

from fmm3dbie_b200.batch import SurfaceBatch, uneven_ellipsoids

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


@pytest.mark.parametrize("kind", [0, 1])
def test_uneven_batch_concurrent_equals_sequential(torch, kind):
    items, rhs, srcs = uneven_ellipsoids(kind, nsurf=32, nrhs=2, seed=4)
    # keep the small surfaces (80 patches) so the test stays quick
    keep = [q for q, it in enumerate(items) if it.surf.npatches == 80][:4]
    items = [items[q] for q in keep]
    rhs = [rhs[q] for q in keep]
    srcs = [srcs[q] for q in keep]
    B = SurfaceBatch(items, 1e-7, engine="streams")
    R = [torch.tensor(np.ascontiguousarray(r), device="cuda") for r in rhs]
    for mode in (0, 1):
        xs, infos, ms = B.solve(R, mode=mode, eps_gmres=1e-10, concurrent=True)
        ys, _, _ = B.solve(R, mode=mode, eps_gmres=1e-10, concurrent=False)
        for q in range(len(items)):
            a, b = xs[q].cpu().numpy(), ys[q].cpu().numpy()
            assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
            assert np.all(infos[q]["rres"] <= 1e-10)
        assert ms > 0
    # exterior field of the first surface, first source (second oracle)
    it, x = items[0], xs[0].cpu().numpy()[:, 0]
    s = it.surf
    w = s.qwts()
    rng = np.random.default_rng(0)
    d = rng.normal(size=(50, 3))
    targ = 8.0 * d / np.linalg.norm(d, axis=1)[:, None]
    dx = targ[:, None, :] - s.xyz[None, :, :]
    r = np.linalg.norm(dx, axis=2)
    dn = np.sum(dx * s.normals[None], 2)
    k = 0.0 if kind == 0 else it.params[0]
    al, be = (it.params if kind == 0 else it.params[1:])
    ker = (al / r + be * dn * (1 - 1j * k * r) / r ** 3) * np.exp(1j * k * r) / (4 * np.pi)
    u = ker @ (w * x)
    r0 = np.linalg.norm(targ - srcs[0][0], axis=1)
    ue = np.exp(1j * k * r0) / (4 * np.pi * r0)
    # coarse surfaces (80 patches, order 4-8): a discretisation-level check
    assert np.max(np.abs(u - ue)) / np.max(np.abs(ue)) < 1e-3
    B.close()


def _small_batch(kind, nsurf=5, nrhs=2):
    items, rhs, _ = uneven_ellipsoids(kind, nsurf=32, nrhs=nrhs, seed=4)
    keep = [q for q, it in enumerate(items) if it.surf.npatches <= 320][:nsurf]
    return [items[q] for q in keep], [rhs[q] for q in keep]


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("nd", [1, 3])
def test_graph_batch_matvec_equals_plans(torch, kind, nd):
    from fmm3dbie_b200 import Plan
    items, _ = _small_batch(kind)
    B = SurfaceBatch(items, 1e-7, engine="graph")
    rng = np.random.default_rng(7)
    dt = torch.complex128 if kind == 1 else torch.float64
    xs = []
    for it in items:
        a = rng.normal(size=(it.surf.npts, nd))
        if kind == 1:
            a = a + 1j * rng.normal(size=a.shape)
        xs.append(torch.tensor(a, dtype=dt, device="cuda"))
    xb = B.concat(xs)
    for iprec, tol in ((0, 1e-12), (1, 1e-6)):
        yb = B.matvec(xb, iprec)
        B.set_graph(False)
        yb2 = B.matvec(xb, iprec)
        B.set_graph(True)
        assert torch.equal(yb, yb2)
        for q, (it, st) in enumerate(zip(items, B.setups)):
            P = Plan(it.kind, it.params, it.surf, st.near, st.over)
            ref = P.matvec(xs[q].contiguous(), iprec)
            P.close()
            got = B.split(yb)[q]
            err = float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))
            assert err < tol, (q, iprec, err)
    B.close()


@pytest.mark.parametrize("kind", [0, 1])
def test_graph_batch_solve_matches_streams(torch, kind):
    items, rhs = _small_batch(kind, nsurf=4)
    R = [torch.tensor(np.ascontiguousarray(r), device="cuda") for r in rhs]
    G = SurfaceBatch(items, 1e-7, engine="graph")
    S = SurfaceBatch(items, 1e-7, engine="streams")
    for mode in (0, 1):
        xg, ig, msg = G.solve(R, mode=mode, eps_gmres=1e-10)
        xs, is_, _ = S.solve(R, mode=mode, eps_gmres=1e-10)
        for q in range(len(items)):
            assert np.all(ig[q]["rres"] <= 1e-10), ig[q]["rres"]
            err = float(torch.linalg.norm(xg[q] - xs[q]) / torch.linalg.norm(xs[q]))
            assert err < 1e-8, (mode, q, err)
        assert msg > 0
    G.close()
    S.close()
