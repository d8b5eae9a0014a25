"""Device near-quadrature generator against the host generator (GPU).

Both run the same rules, tolerance and refinement, so the weights agree to
round-off except where a refinement decision sits at the threshold; there
the two differ by about the tolerance.  Checked per case: the near
potential of a smooth density (relative L2 difference <= 10 eps), the worst
pair (max-norm difference relative to the row's max-norm <= 1e3 eps) and
the fraction of pairs identical to 1e-10 relative.
"""
import numpy as np
import pytest

from fmm3dbie_b200 import surface as S

pytestmark = pytest.mark.gpu


def _near_setup(s, targs=None, ipatch_id=None, uvs=None):
    if targs is None:
        targs = s.srcvals
        ipatch_id, uvs = s.patch_id_uvs()
    rfac, rfac0 = S.get_rfacs(int(s.norders.mean()), int(s.iptype.mean()))
    cms, rads = S.get_centroid_rads(s)
    row_ptr, col_ind = S.findnear(cms, rads * rfac, targs)
    iquad = S.get_iquad_rsc(s, row_ptr, col_ind)
    return targs, ipatch_id, uvs, row_ptr, col_ind, iquad, rfac0


def _compare(s, kind, eps, params, near):
    targs, ipatch_id, uvs, row_ptr, col_ind, iquad, rfac0 = near
    wc = S.getnearquad(s, kind, eps, params, targs, ipatch_id, uvs, row_ptr, col_ind, iquad, rfac0,
                       engine="cpu")
    st = np.zeros(3, np.int64)
    wg = S.getnearquad(s, kind, eps, params, targs, ipatch_id, uvs, row_ptr, col_ind, iquad, rfac0,
                       engine="gpu", stats=st)
    assert wg.shape == wc.shape and np.all(np.isfinite(wg))
    nt = targs.shape[0]
    x = s.srcvals[:, 0:3]
    sig = np.cos(x[:, 0] + 0.5 * x[:, 1]) * np.exp(0.3 * x[:, 2])
    pots = []
    for w in (wc, wg):
        pot = np.zeros(nt, dtype=w.dtype)
        for t in range(nt):
            for k in range(row_ptr[t] - 1, row_ptr[t + 1] - 1):
                p = col_ind[k] - 1
                a, b = s.ixyzs[p] - 1, s.ixyzs[p + 1] - 1
                pot[t] += w[iquad[k] - 1:iquad[k + 1] - 1] @ sig[a:b]
        pots.append(pot)
    pot_err = np.linalg.norm(pots[1] - pots[0]) / np.linalg.norm(pots[0])
    worst, same = 0.0, 0
    nnz = col_ind.shape[0]
    for k in range(nnz):
        a, b = iquad[k] - 1, iquad[k + 1] - 1
        scale = np.max(np.abs(wc[a:b]))
        d = np.max(np.abs(wg[a:b] - wc[a:b])) / scale
        worst = max(worst, d)
        same += d <= 1e-10
    print(f"\nkind {kind} eps {eps:.0e}: pairs {nnz} (self {st[1]}, near {st[2]}), kernel evals "
          f"{st[0]}; near-potential diff {pot_err:.2e}, worst pair {worst:.2e}, "
          f"identical {same / nnz:.4f}")
    assert st[1] + st[2] == nnz
    assert pot_err <= 10 * eps
    assert worst <= 1e3 * eps
    assert same >= 0.9 * nnz
    return st


@pytest.mark.parametrize("kind,params", [(0, (1.0, 1.0)), (1, (1.3, -1.3j, 1.0)),
                                         (1, (2.0 + 0.4j, 0.5 - 1.0j, 1.0))])
def test_sphere_order4(kind, params):
    s = S.icosa_sphere(1, 4)
    _compare(s, kind, 1e-7, params, _near_setup(s))


def test_ellipsoid_order8_helmholtz():
    """45 basis functions: more than one basis index per lane."""
    s = S.icosa_ellipsoid(1, 8, (1.0, 2.0, 3.0))
    _compare(s, 1, 1e-6, (1.0, -1.0j, 1.0), _near_setup(s))


def test_torus_quads_helmholtz():
    from fmm3dbie_b200.warmstart import torus_surface
    s = torus_surface(16, 8, 5)
    _compare(s, 1, 1e-7, (2.0, -2.0j, 1.0), _near_setup(s))


def test_off_surface_targets_laplace():
    """Targets off the surface (no self pairs), some of them very close."""
    s = S.icosa_ellipsoid(1, 6, (1.0, 2.0, 3.0))
    rng = np.random.default_rng(3)
    pick = rng.choice(s.npts, 300, replace=False)
    h = rng.uniform(1e-3, 0.2, 300) * rng.choice([-1.0, 1.0], 300)
    targs = s.srcvals[pick, 0:3] + h[:, None] * s.srcvals[pick, 9:12]
    ipatch_id = -np.ones(300, np.int64)
    uvs = np.zeros((300, 2))
    st = _compare(s, 0, 1e-7, (1.0, 1.0), _near_setup(s, targs, ipatch_id, uvs))
    assert st[1] == 0


def test_setup_engine_switch():
    """The simple solver entry points take the engine set in the library."""
    from fmm3dbie_b200 import _lib as L
    lib = L.lib()
    old = lib.bie_get_nearquad_engine()
    try:
        assert lib.bie_set_nearquad_engine(1) == 0
        assert lib.bie_get_nearquad_engine() == 1
        assert lib.bie_set_nearquad_engine(5) != 0
    finally:
        lib.bie_set_nearquad_engine(old)


@pytest.mark.parametrize("levels,budget_mb", [("-1", None), ("0", None), ("5", None), ("2", "3")])
def test_refinement_cache_settings(monkeypatch, levels, budget_mb):
    """Without the cache of uniform refinement levels, with one level, with
    five, and with a budget small enough to split the patches into groups:
    the same weights as the host generator."""
    monkeypatch.setenv("BIE_NEARQUAD_CACHE_LEVELS", levels)
    if budget_mb:
        monkeypatch.setenv("BIE_NEARQUAD_CACHE_BUDGET_MB", budget_mb)
    s = S.icosa_ellipsoid(1, 6, (1.0, 2.0, 3.0))
    _compare(s, 1, 1e-7, (1.5, -1.5j, 1.0), _near_setup(s))


def test_chebyshev_quads_and_mixed_patches():
    """Tensor Chebyshev quads (iptype 12) and one surface mixing triangles of
    orders 4 and 6 with Chebyshev quads of order 5."""
    from _surfaces import concat, torus_cheb
    t = torus_cheb()
    _compare(t, 1, 1e-7, (2.0, -2.0j, 1.0), _near_setup(t))
    m = concat(S.icosa_sphere(1, 4), S.icosa_ellipsoid(1, 6, (1.0, 2.0, 3.0)), torus_cheb(8, 4, 5),
               shifts=[(0, 0, 0), (6, 0, 0), (0, 8, 0)])
    _compare(m, 0, 1e-7, (1.0, 1.0), _near_setup(m))
