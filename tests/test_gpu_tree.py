"""Hierarchical far field (GPU): the dual-tree barycentric Lagrange method
against the direct sum over all pairs, through the same plan matvec (near
correction included), for Laplace and Helmholtz (real and complex k), FP64
and FP32, one and several densities, and a range of opening angles and grid
sizes that exercises every interaction form (PP, PC, CP, CC)."""
import numpy as np
import pytest

from fmm3dbie_b200 import surface as S

pytestmark = pytest.mark.gpu


def _rel(a, b, w):
    num = ((w[:, None] * (a - b).abs() ** 2).sum(0)) ** 0.5
    den = ((w[:, None] * b.abs() ** 2).sum(0)) ** 0.5
    return float((num / den).max())


@pytest.fixture(scope="module",
                params=[(0, 0.0), (1, 2.0), (1, 4.0 + 0.5j)], ids=["laplace", "helm", "helm_ck"])
def plan(request):
    import torch
    from fmm3dbie_b200 import Plan
    kind, zk = request.param
    s = S.icosa_ellipsoid(2, 4, (1.0, 2.0, 3.0))
    zp = (1.0, 1.0) if kind == 0 else (zk, -1j * zk, 1.0)
    st = S.setup(s, kind, 1e-7, zp)
    P = Plan(kind, zp, s, st.near, st.over)
    w = torch.tensor(s.qwts(), device="cuda")
    yield kind, P, s, w
    P.close()


def _density(s, nd, kind, seed):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.randn(s.npts, nd, generator=g, dtype=torch.float64)
    if kind == 1:
        x = x + 1j * torch.randn(s.npts, nd, generator=g, dtype=torch.float64)
    return x.cuda().contiguous()


# (theta, p, FP64 bound): the bounds are those of the weighted relative L2
# error of the whole matvec against the direct sum
CASES = [(0.8, 2, 0.5), (0.6, 3, 5e-2), (0.7, 4, 2e-2), (0.5, 6, 2e-4), (0.5, 8, 2e-5),
         (0.5, 10, 2e-6)]


@pytest.mark.parametrize("theta,p,tol", CASES)
@pytest.mark.parametrize("nd", [1, 3])
def test_tree_matches_direct_fp64(plan, theta, p, tol, nd):
    kind, P, s, w = plan
    x = _density(s, nd, kind, 7 + nd)
    P.set_far_method(0, 0)
    y = P.matvec(x, 0)
    P.set_far_method(0, 1, theta, p)
    info = P.get_far_method(0)
    yt = P.matvec(x, 0)
    P.set_far_method(0, 0)
    err = _rel(yt, y, w)
    print(f"\nkind {kind} theta {theta} p {p} nd {nd}: {err:.2e}  "
          f"(PP {info['pp'] + info['pp_check']:.0f} PC {info['pc']:.0f} CP {info['cp']:.0f} "
          f"CC {info['cc']:.0f}, evals {info['kernel_evals']:.3e} of "
          f"{float(s.npts) * P.nptso:.3e})")
    assert info["method"] == 1
    assert err < tol


@pytest.mark.parametrize("theta,p,leaf,tol",
                         [(0.6, 2, 16, 0.5), (0.6, 4, 32, 2e-2), (0.5, 8, 64, 1e-5)])
def test_tree_small_leaves(plan, theta, p, leaf, tol):
    """Small leaves: many CP and CC interactions and proxy-target items."""
    kind, P, s, w = plan
    x = _density(s, 2, kind, 5)
    P.set_far_method(0, 0)
    y = P.matvec(x, 0)
    P.set_far_method(0, 1, theta, p, leaf, leaf)
    info = P.get_far_method(0)
    yt = P.matvec(x, 0)
    P.set_far_method(0, 0)
    err = _rel(yt, y, w)
    print(f"\nkind {kind} theta {theta} p {p} leaf {leaf}: {err:.2e} (CP {info['cp']:.0f} "
          f"CC {info['cc']:.0f})")
    assert err < tol


def test_tree_forms_exercised(plan):
    """The accuracy cases above include lists with every interaction form."""
    kind, P, s, w = plan
    seen = {"pp": 0, "pc": 0, "cp": 0, "cc": 0}
    for theta, p, leaf in ((0.7, 4, 0), (0.6, 4, 32), (0.6, 2, 16)):
        P.set_far_method(0, 1, theta, p, leaf, leaf)
        info = P.get_far_method(0)
        for f in seen:
            seen[f] += info[f] + (info["pp_check"] if f == "pp" else 0)
    P.set_far_method(0, 0)
    print(f"\nkind {kind}: forms {seen}")
    assert all(v > 0 for v in seen.values())


@pytest.mark.parametrize("nd,p", [(1, 0), (2, 0), (1, 6), (1, 10)])
def test_tree_fp32(plan, nd, p):
    """FP32 tree matvec (FP32 W_eff refolded for the tree's centring)
    against the FP64 direct matvec, and switching back restores the direct
    FP32 result."""
    kind, P, s, w = plan
    x = _density(s, nd, kind, 3)
    P.set_far_method(0, 0)
    y64 = P.matvec(x, 0)
    P.set_far_method(1, 0)
    y32 = P.matvec(x, 1)
    e_direct = _rel(y32, y64, w)
    P.set_far_method(1, 1, 0.0, p)
    yt32 = P.matvec(x, 1)
    P.set_far_method(0, 1, 0.0, p)
    yt64 = P.matvec(x, 0)
    P.set_far_method(0, 0)
    e_tree64 = _rel(yt64, y64, w)
    e_tree = _rel(yt32, y64, w)
    P.set_far_method(1, 0)
    yb = P.matvec(x, 1)
    e_back = _rel(yb, y32, w)
    print(f"\nkind {kind} nd {nd} p {p}: FP32 direct {e_direct:.2e}, FP32 tree {e_tree:.2e} "
          f"(FP64 tree {e_tree64:.2e}), back {e_back:.2e}")
    # FP32 rounding of the proxy terms (about 1e-6) or the interpolation
    # error of a small grid, whichever is larger
    assert e_tree < max(20 * e_direct, 3e-5, 2 * e_tree64)
    assert e_back < 1e-6


def test_tree_solve(plan):
    """GMRES with the hierarchical far field converges to the direct
    solution."""
    kind, P, s, w = plan
    x = _density(s, 1, kind, 11)[:, 0].contiguous()
    rhs = P.matvec(x, 0)  # any right-hand side
    P.set_far_method(0, 0)
    sol_d = P.solve(rhs, 0.5, mode=0, numit=100, eps_gmres=1e-10)[0]
    P.set_far_method(0, 1, 0.5, 10)
    sol_t = P.solve(rhs, 0.5, mode=0, numit=100, eps_gmres=1e-10)[0]
    P.set_far_method(0, 0)
    err = _rel(sol_t[:, None], sol_d[:, None], w)
    print(f"\nkind {kind}: tree solve vs direct solve {err:.2e}")
    assert err < 1e-5


@pytest.mark.parametrize("nd", [2, 7, 9, 20])
def test_tree_multi_density(plan, nd):
    """Several densities per block (groups of 4, 8, 16; the last group
    partial) equal the one-density tree matvec column by column (FP64: same
    interactions, other summation order) and, in FP32, stay within FP32
    accuracy of it."""
    import torch
    kind, P, s, w = plan
    x = _density(s, nd, kind, 20 + nd)
    for iprec, tol in ((0, 1e-11), (1, 3e-6)):
        P.set_far_method(iprec, 1, 0.6, 4, 32, 32)  # small leaves: every form
        y = P.matvec(x, iprec)
        cols = [0, nd // 2, nd - 1]
        err = 0.0
        for m in cols:
            y1 = P.matvec(x[:, m].contiguous(), iprec)
            err = max(err, _rel(y[:, m:m + 1], y1[:, None], w))
        P.set_far_method(iprec, 0)
        print(f"\nkind {kind} nd {nd} prec {iprec}: multi-density vs one density {err:.2e}")
        assert err < tol


@pytest.mark.parametrize("kind", [0, 1])
def test_tree_vs_oracle(kind):
    """The hierarchical matvec (forced on a 4,800-node surface) against the
    oracle's exact FP64 matvec, with grids that approximate part of the far
    field: within the interpolation error of the grid."""
    import oracle
    import torch
    from fmm3dbie_b200 import Plan
    s = S.icosa_ellipsoid(2, 4, (1.0, 2.0, 3.0))
    params = (1.0, 1.0) if kind == 0 else (2.0, -2.0j, 1.0)
    st = S.setup(s, kind, 1e-7, params)
    rng = np.random.default_rng(4)
    sig = rng.normal(size=s.npts) + (1j * rng.normal(size=s.npts) if kind else 0)
    ref = oracle.lpcomp(kind, s, params, st.near, st.over, sig)
    w = s.qwts()
    P = Plan(kind, params, s, st.near, st.over)
    x = torch.tensor(sig, device="cuda")
    for prec, theta, p, tol in ((0, 0.5, 8, 1e-5), (1, 0.5, 8, 2e-5), (0, 0.7, 4, 2e-2)):
        P.set_far_method(prec, 1, theta, p)
        info = P.get_far_method(prec)
        got = P.matvec(x, prec).cpu().numpy()
        P.set_far_method(prec, 0)
        err = np.sqrt(np.sum(w * np.abs(got - ref) ** 2) / np.sum(w * np.abs(ref) ** 2))
        print(f"\nkind {kind} prec {prec} theta {theta} p {p}: tree vs oracle {err:.2e} "
              f"(PC {info['pc']:.0f} CP {info['cp']:.0f} CC {info['cc']:.0f})")
        assert info["pc"] + info["cp"] + info["cc"] > 0
        assert err < tol
    P.close()
