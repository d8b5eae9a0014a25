"""Device setup steps against the host ones (GPU): near lists (findnear),
far-field orders (get_far_order) and oversampled geometry (oversample_geom).

Near lists are decided with the same rounding on both sides and must be
identical; far orders are decisions of a tolerance test on integrals that
agree to rounding and must be identical on these surfaces; the oversampled
geometry agrees to rounding.
"""
import numpy as np
import pytest

from fmm3dbie_b200 import surface as S

pytestmark = pytest.mark.gpu


def _surfaces():
    from _surfaces import concat, torus_cheb
    from fmm3dbie_b200.warmstart import torus_surface
    return {
        "sphere4": S.icosa_sphere(1, 4),
        "ellipsoid6": S.icosa_ellipsoid(2, 6, (1.0, 2.0, 3.0)),
        "ellipsoid8": S.icosa_ellipsoid(1, 8, (0.7, 1.5, 2.5)),
        "torus5": torus_surface(16, 8, 5),
        "torus5_chebyshev": torus_cheb(),
        "mixed": concat(S.icosa_sphere(1, 4), S.icosa_ellipsoid(1, 6, (1.0, 2.0, 3.0)),
                        torus_cheb(8, 4, 5), shifts=[(0, 0, 0), (6, 0, 0), (0, 8, 0)]),
    }


SURF = _surfaces()


def _near(s, targs=None):
    if targs is None:
        targs = s.srcvals
    rfac, _ = S.get_rfacs(int(s.norders.mean()), int(s.iptype.mean()))
    cms, rads = S.get_centroid_rads(s)
    return targs, cms, rads, rfac


@pytest.mark.parametrize("name", list(SURF))
def test_findnear_same_lists(name):
    s = SURF[name]
    targs, cms, rads, rfac = _near(s)
    rc, cc = S.findnear(cms, rads * rfac, targs, engine="cpu")
    rg, cg = S.findnear(cms, rads * rfac, targs, engine="gpu")
    assert np.array_equal(rc, rg) and np.array_equal(cc, cg)


def test_findnear_off_surface_targets():
    s = SURF["ellipsoid6"]
    rng = np.random.default_rng(7)
    targs = rng.uniform(-4, 4, (5000, 3))          # many outside the centroids' box
    targs[:2000] = s.srcvals[rng.choice(s.npts, 2000), :3] * 1.01
    _, cms, rads, rfac = _near(s)
    rc, cc = S.findnear(cms, rads * rfac, targs, engine="cpu")
    rg, cg = S.findnear(cms, rads * rfac, targs, engine="gpu")
    assert np.array_equal(rc, rg) and np.array_equal(cc, cg)
    assert rc[-1] - 1 > 2000


@pytest.mark.parametrize("name", list(SURF))
@pytest.mark.parametrize("kind,ikerorder,zk", [(0, 0, 0.0), (1, 0, 2.0), (1, -1, 1.5 + 0.3j)])
def test_far_order_same_orders(name, kind, ikerorder, zk):
    s = SURF[name]
    targs, cms, rads, rfac = _near(s)
    rp, ci = S.findnear(cms, rads * rfac, targs)
    for eps in (1e-4, 1e-7):
        nc, ic = S.get_far_order(eps, s, cms, rads, targs, ikerorder, zk, rp, ci, rfac,
                                 engine="cpu")
        ng, ig = S.get_far_order(eps, s, cms, rads, targs, ikerorder, zk, rp, ci, rfac,
                                 engine="gpu")
        assert np.array_equal(nc, ng), (eps, np.flatnonzero(nc != ng)[:10])
        assert np.array_equal(ic, ig)


@pytest.mark.parametrize("name", list(SURF))
def test_oversample_geom_matches(name):
    s = SURF[name]
    targs, cms, rads, rfac = _near(s)
    rp, ci = S.findnear(cms, rads * rfac, targs)
    nf, ixo = S.get_far_order(1e-7, s, cms, rads, targs, 0, 2.0, rp, ci, rfac)
    nf = nf.copy()
    nf[::3] = s.norders[::3]                        # some patches keep their own order
    ixo = np.concatenate([[1], 1 + np.cumsum([(n + 1) * (n + 2) // 2 if t == 1 else (n + 1) ** 2
                                               for n, t in zip(nf, s.iptype)])]).astype(np.int64)
    oc = S.oversample_geom(s, nf, ixo, engine="cpu")
    og = S.oversample_geom(s, nf, ixo, engine="gpu")
    assert np.max(np.abs(oc - og)) < 1e-13


def test_setup_engines_agree():
    s = SURF["ellipsoid6"]
    params = (2.0, -2.0j, 1.0)
    sc = S.setup(s, 1, 1e-7, params, engine="cpu")
    sg = S.setup(s, 1, 1e-7, params, engine="gpu")
    assert np.array_equal(sc.near.row_ptr, sg.near.row_ptr)
    assert np.array_equal(sc.near.col_ind, sg.near.col_ind)
    assert np.array_equal(sc.over.novers, sg.over.novers)
    assert np.max(np.abs(sc.over.srcover - sg.over.srcover)) < 1e-13
    assert np.max(np.abs(sc.near.wnear - sg.near.wnear)) < 1e-6 * np.max(np.abs(sc.near.wnear))
