"""The oracle's own setup (oracle/oracle_setup.c: surfaces, brute-force near
lists, far orders, oversampled geometry, weights and an adaptive near
quadrature with rules of its own) against the product's host setup, and the
oracle-only pipeline against the reference's known answers.

Bars: identical near lists and far-field orders; oversampled geometry and
weights to rounding (1e-13); near potentials (the wnear part of the matvec
applied to a random density) within 10 eps of the configuration.  Measured:
1e-9 (sphere, eps 1e-6), 4e-10 (ellipsoid, eps 1e-7) and 6e-7 on the coarse
torus at k = 8 (eps 1e-7; two wavelengths per patch; the product's rule
reaches 8e-10 there at eps 1e-10, and the oracle's weights move by 1e-11
when its tolerance is tightened 1e4 times)."""
import json
import os

import numpy as np
import pytest

import oracle
from fmm3dbie_b200 import surface as S
from conftest import wnorm

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "sphere_spectra.json")))


def _near_matrix(s, near):
    """wnear as a sparse target x node matrix."""
    import scipy.sparse as sp
    rp, ci, iq = near.row_ptr, near.col_ind, near.iquad
    nt = rp.shape[0] - 1
    rows = np.repeat(np.arange(nt), np.diff(rp))
    npols = np.diff(s.ixyzs)[ci - 1]
    ent_row = np.repeat(rows, npols)
    first = np.repeat(s.ixyzs[ci - 1] - 1, npols)
    offs = np.arange(ent_row.shape[0]) - np.repeat(iq[:-1] - 1, npols)
    return sp.csr_matrix((near.wnear, (ent_row, first + offs)), shape=(nt, s.npts))


def test_surfaces_match_product(built):
    """The reference's icosahedron refinement and ellipsoid chart, and the
    quad torus, generated independently by the oracle and the product."""
    for nref, n, ax in ((1, 4, (1.0, 1.0, 1.0)), (2, 6, (1.0, 2.0, 3.0)), (1, 8, (0.7, 1.3, 2.9))):
        a, b = S.icosa_ellipsoid(nref, n, ax), oracle.icosa_ellipsoid(nref, n, ax)
        assert np.array_equal(a.norders, b.norders) and np.array_equal(a.ixyzs, b.ixyzs)
        assert np.abs(a.srcvals - b.srcvals).max() < 1e-14
        assert np.abs(a.srccoefs - b.srccoefs).max() < 1e-13
    from fmm3dbie_b200.warmstart import torus_surface
    a, b = torus_surface(8, 4, 5), oracle.torus_quad(8, 4, 5)
    assert np.abs(a.srcvals - b.srcvals).max() < 1e-14
    assert np.abs(a.srccoefs - b.srccoefs).max() < 1e-13
    # outward normals, closed surface area
    s = oracle.icosa_ellipsoid(2, 6)
    assert np.all(np.sum(s.normals * s.xyz, 1) > 0)
    assert abs(s.qwts().sum() - 4 * np.pi) < 1e-6


def test_hkrand_matches_product(built):
    for seed in (0, 1, 7, 1001 + 11, 3042 + 25, 4095, 123456):
        assert oracle.hkrand(seed) == S.hkrand(seed)


CASES = {
    "sphere80_o4_laplace": (lambda: S.icosa_sphere(1, 4), 0, 1e-6, (1.0, 1.0)),
    "ellipsoid80_o6_helmholtz": (lambda: S.icosa_ellipsoid(1, 6, (1.0, 2.0, 3.0)), 1, 1e-7,
                                 (2.0, -2.0j, 1.0)),
    "torus32_quads_helmholtz_k8": (lambda: __import__("fmm3dbie_b200.warmstart", fromlist=["x"])
                                   .torus_surface(8, 4, 5), 1, 1e-7, (8.0, -8.0j, 1.0)),
}


@pytest.mark.parametrize("case", list(CASES))
def test_setup_matches_product(built, case):
    make, kind, eps, params = CASES[case]
    s = make()
    sp = S.setup(s, kind, eps, params, engine="cpu")
    so = oracle.setup(s, kind, eps, params)
    assert (sp.rfac, sp.rfac0) == (so.rfac, so.rfac0)
    assert np.abs(sp.cms - so.cms).max() < 1e-14 and np.abs(sp.rads - so.rads).max() < 1e-14
    # near lists: the same pairs (within-row order is not contractual)
    assert np.array_equal(sp.near.row_ptr, so.near.row_ptr)
    for i in range(s.npts):
        a, b = sp.near.row_ptr[i] - 1, sp.near.row_ptr[i + 1] - 1
        assert np.array_equal(np.sort(sp.near.col_ind[a:b]), np.sort(so.near.col_ind[a:b]))
    # far orders and oversampled geometry
    assert np.array_equal(sp.over.novers, so.over.novers)
    assert np.abs(sp.over.srcover - so.over.srcover).max() < 1e-13
    assert np.abs(sp.over.wover - so.over.wover).max() < 1e-13 * so.over.wover.max()
    assert np.abs(s.qwts() - oracle.qwts(s)).max() < 1e-15 * s.qwts().max() * 10
    # near quadrature: near potentials of a random density
    rng = np.random.default_rng(8)
    sig = rng.normal(size=s.npts) + (1j * rng.normal(size=s.npts) if kind else 0)
    pp = _near_matrix(s, sp.near) @ sig
    po = _near_matrix(s, so.near) @ sig
    err = np.max(np.abs(pp - po)) / np.max(np.abs(po))
    print(f"\n{case}: near potentials max rel diff {err:.2e} (eps {eps:g})")
    assert err < 10 * eps


def test_oracle_pipeline_known_answers(built):
    """Surface, setup, near quadrature and matvec all by the oracle: the sphere
    spectra S_0 Y = Y/3, D_0 Y = -Y/6 and S_k, D_k (values from scipy in
    tests/golden) on 320 order-6 patches."""
    s = oracle.icosa_ellipsoid(2, 6)
    w = oracle.qwts(s)
    z = s.xyz[:, 2]
    st = oracle.setup(s, 0, 1e-7, (1.0, 1.0))
    ev = GOLD["laplace"]["1"]["S"] + GOLD["laplace"]["1"]["D"]
    pot = oracle.lpcomp(0, s, (1.0, 1.0), st.near, st.over, z)
    e_lap = wnorm(w, pot - ev * z) / wnorm(w, ev * z)
    k = 2.0
    g = GOLD["helmholtz"][f"{k}:1"]
    zp = (k, -1j * k, 1.0)
    evh = -1j * k * complex(*g["S"]) + complex(*g["D"])
    st = oracle.setup(s, 1, 1e-7, zp)
    poth = oracle.lpcomp(1, s, zp, st.near, st.over, z.astype(complex))
    e_helm = wnorm(w, poth - evh * z) / wnorm(w, evh * z)
    print(f"\noracle-only sphere spectra: Laplace S+D {e_lap:.2e}, Helmholtz k=2 CFIE {e_helm:.2e}")
    # order-6 discretisation error of Y_1^0 (measured 1.8e-6 / 4.7e-7; the
    # Laplace eigenvalue 1/3 - 1/6 is the smaller one, so its relative error
    # is the larger)
    assert e_lap < 5e-6 and e_helm < 2e-6


def test_stepwise_gmres_matches_oracle_gmres(built):
    """The oracle's stepwise GMRES (timed by the benchmark's CPU legs) is
    the oracle's C GMRES: same iterations, residuals and solution."""
    s = oracle.icosa_ellipsoid(1, 4, (1.0, 2.0, 3.0))
    zp = (2.0, -2.0j, 1.0)
    st = oracle.setup(s, 1, 1e-6, zp)
    r = np.linalg.norm(s.xyz - np.array([0.1, -0.2, 0.3]), axis=1)
    rhs = np.exp(2j * r) / (4 * np.pi * r)
    ref, nit, errs, rres, status = oracle.gmres(1, s, zp, st.near, st.over, 0.5, rhs, numit=60,
                                                eps_gmres=1e-10)
    g = oracle.GmresSolver(1, s, zp, st.near, st.over, 0.5, rhs, numit=60, eps_gmres=1e-10)
    while not g.step():
        pass
    x, m, errs2, rres2 = g.finish()
    assert status == 0 and m == nit
    assert np.allclose(errs2, errs, rtol=1e-8, atol=0)
    assert abs(rres2 - rres) <= 1e-3 * rres + 1e-15
    w = oracle.qwts(s)
    assert wnorm(w, x - ref) / wnorm(w, ref) < 1e-12
