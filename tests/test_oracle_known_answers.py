"""Pins the FP64 oracle (and the host setup / near quadrature that feed it)
to the reference's known-answer tests: sphere spectra
(matlab/test/lap3d_dirichlet_routsTest.m:9-34,
matlab/test/helm3d_dirichlet_routsTest.m:10-35), Green's identity
(test/lap_wrappers/test_lap_wrappers_qg_lp.f:190-239,
test/helm_wrappers/test_helm_wrappers_qg_lp.f:218-260) and the interior
point-source solve checked at exterior targets
(examples/helmholtz/helm_dir_iter_example.f)."""
import json
import os

import numpy as np
import pytest

import oracle
from fmm3dbie_b200 import surface as S
from conftest import wnorm

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "sphere_spectra.json")))


def _rel(w, a, b):
    return wnorm(w, a - b) / wnorm(w, b)


@pytest.fixture(scope="module")
def sphere8(built):
    # order 8 on 320 patches keeps the discretisation error below the
    # quadrature target
    return S.icosa_sphere(2, 8)


@pytest.mark.parametrize("params,which", [((1.0, 0.0), "S"), ((0.0, 1.0), "D"), ((1.0, 1.0), "SD")])
def test_laplace_sphere_spectrum(sphere8, params, which):
    s = sphere8
    st = S.setup(s, 0, 1e-7, params)
    z = s.xyz[:, 2]
    ev = params[0] * GOLD["laplace"]["1"]["S"] + params[1] * GOLD["laplace"]["1"]["D"]
    pot = oracle.lpcomp(0, s, params, st.near, st.over, z)
    assert _rel(s.qwts(), pot, ev * z) < 2e-6


def test_laplace_sphere_single_layer(sphere4):
    # sphere, 320 order-4 patches: S_0 Y_1^0 = Y_1^0 / 3 to eps
    st = S.setup(sphere4, 0, 1e-6, (1.0, 0.0))
    z = sphere4.xyz[:, 2]
    pot = oracle.lpcomp(0, sphere4, (1.0, 0.0), st.near, st.over, z)
    assert _rel(sphere4.qwts(), pot, z / 3) < 5e-6


@pytest.mark.parametrize("k,parts", [(1.1, "S"), (1.1, "D"), (2.0, "SD")])
def test_helmholtz_sphere_spectrum(sphere8, k, parts):
    s = sphere8
    z = s.xyz[:, 2]
    g = GOLD["helmholtz"][f"{k}:1"]
    es, ed = complex(*g["S"]), complex(*g["D"])
    cases = {"S": ((k, 1.0, 0.0), es), "D": ((k, 0.0, 1.0), ed),
             "SD": ((k, -1j * k, 1.0), -1j * k * es + ed)}
    for zp, ev in [cases[parts]]:
        st = S.setup(s, 1, 1e-7, zp)
        pot = oracle.lpcomp(1, s, zp, st.near, st.over, z.astype(complex))
        assert _rel(s.qwts(), pot, ev * z) < 2e-6, (zp, _rel(s.qwts(), pot, ev * z))


def _point_source(kind, k, x0, x, n=None):
    d = x - x0
    r = np.linalg.norm(d, axis=1)
    if kind == 0:
        u = 1 / (4 * np.pi * r)
        dudn = None if n is None else -np.sum(d * n, 1) / (4 * np.pi * r ** 3)
    else:
        u = np.exp(1j * k * r) / (4 * np.pi * r)
        dudn = None if n is None else np.sum(d * n, 1) * (1j * k * r - 1) * np.exp(1j * k * r) / (4 * np.pi * r ** 3)
    return u, dudn


@pytest.mark.parametrize("kind", [0, 1])
def test_greens_identity(built, kind):
    s = S.icosa_ellipsoid(1, 8, (1.0, 2.0, 3.0))
    k = 1.1
    x0 = np.array([3.1, -2.7, 4.3])  # exterior source: u harmonic inside
    u, dudn = _point_source(kind, k, x0, s.xyz, s.normals)
    pS = (1.0, 0.0) if kind == 0 else (k, 1.0, 0.0)
    pD = (0.0, 1.0) if kind == 0 else (k, 0.0, 1.0)
    stS = S.setup(s, kind, 1e-7, pS)
    stD = S.setup(s, kind, 1e-7, pD)
    sl = oracle.lpcomp(kind, s, pS, stS.near, stS.over, dudn)
    dl = oracle.lpcomp(kind, s, pD, stD.near, stD.over, u)
    err = _rel(s.qwts(), 2 * (sl - dl), u)
    assert err < 5e-6, err


@pytest.mark.parametrize("kind", [0, 1])
def test_greens_identity_quad_torus(built, kind):
    """Quad patches (iptype 11, tensor Gauss-Legendre nodes): the warm-start
    torus family at 16 x 8 patches of 6 x 6 nodes; the source sits above the
    hole, outside the tube."""
    from fmm3dbie_b200.warmstart import torus_surface
    s = torus_surface(16, 8, 5)
    k = 3.0
    x0 = np.array([0.3, 0.2, 1.7])
    u, dudn = _point_source(kind, k, x0, s.xyz, s.normals)
    pS = (1.0, 0.0) if kind == 0 else (k, 1.0, 0.0)
    pD = (0.0, 1.0) if kind == 0 else (k, 0.0, 1.0)
    stS = S.setup(s, kind, 1e-7, pS)
    stD = S.setup(s, kind, 1e-7, pD)
    sl = oracle.lpcomp(kind, s, pS, stS.near, stS.over, dudn)
    dl = oracle.lpcomp(kind, s, pD, stD.near, stD.over, u)
    err = _rel(s.qwts(), 2 * (sl - dl), u)
    assert err < 3e-5, err   # 1.0e-5 measured (3.4e-7 at 32 x 16 patches)


def test_interior_point_source_solve(ellipsoid_small, ellipsoid_helm_setup):
    """Second oracle: exterior field of an interior source (ellipsoid (1,2,3) point-source shape)."""
    s = ellipsoid_small
    k = 2.0
    zp = (k, -1j * k, 1.0)
    x0 = np.array([0.1, -0.2, 0.3])
    rhs, _ = _point_source(1, k, x0, s.xyz)
    st = ellipsoid_helm_setup
    soln, niter, errs, rres, status = oracle.gmres(1, s, zp, st.near, st.over, 0.5, rhs, numit=100,
                                                    eps_gmres=1e-10)
    assert status == 0 and rres < 1e-9
    rng = np.random.default_rng(2)
    d = rng.normal(size=(100, 3))
    targ = 5 * d / np.linalg.norm(d, axis=1)[:, None]
    # smooth rule, accurate far from the surface (helm_dir_iter_example.f)
    w = s.qwts()
    dx = targ[:, None, :] - s.xyz[None, :, :]
    r = np.linalg.norm(dx, axis=2)
    dn = np.sum(dx * s.normals[None], 2)
    ker = (zp[1] / r + zp[2] * dn * (1 - 1j * k * r) / r ** 3) * np.exp(1j * k * r) / (4 * np.pi)
    u = ker @ (w * soln)
    ue, _ = _point_source(1, k, x0, targ)
    # 80 order-6 patches: the discretisation error is ~4e-6 here
    assert np.max(np.abs(u - ue)) / np.max(np.abs(ue)) < 1e-5
