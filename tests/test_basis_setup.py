"""Host setup: node tables, bases, surfaces, near lists, far order
(CPU; the reference's test_koornexps.f / test_find_near.f / test_surf_routs.f
checks restated)."""
import ctypes as C

import numpy as np
import pytest

from fmm3dbie_b200 import _lib as L
from fmm3dbie_b200 import surface as S


def _exps(iptype, norder):
    lib = L.lib()
    lib.bie_init(None)
    npols = L.I64()
    lib.bie_get_npols(iptype, norder, C.byref(npols))
    n = npols.value
    uvs = np.zeros((n, 2))
    um = np.zeros((n, n), order="F")
    vm = np.zeros((n, n), order="F")
    w = np.zeros(n)
    L.check(lib.bie_get_disc_exps(norder, n, iptype, L.ptr(uvs), um.ctypes.data_as(L.PDBL),
                                  vm.ctypes.data_as(L.PDBL), L.ptr(w)), "disc_exps")
    return uvs, um, vm, w


def _pols(iptype, norder, uv):
    lib = L.lib()
    n = (norder + 1) * (norder + 2) // 2 if iptype == 1 else (norder + 1) ** 2
    p = np.zeros(n)
    u = np.asarray(uv, float)
    lib.bie_get_basis_pols(L.ptr(u), norder, n, iptype, L.ptr(p))
    return p


def _simplex_rule(n):
    x, w = np.polynomial.legendre.leggauss(n)
    a, wa = 0.5 * (x + 1), 0.5 * w
    U, V, W = [], [], []
    for i in range(n):
        for j in range(n):
            U.append(a[i]); V.append(a[j] * (1 - a[i])); W.append(wa[i] * wa[j] * (1 - a[i]))
    return np.array(U), np.array(V), np.array(W)


@pytest.mark.parametrize("norder", [0, 1, 3, 4, 6, 8, 12, 20])
def test_vr_tables(built, norder):
    uvs, um, vm, w = _exps(1, norder)
    assert abs(w.sum() - 0.5) < 1e-13
    assert np.all(uvs > 0) and np.all(uvs.sum(1) < 1)
    assert np.allclose(um @ vm, np.eye(len(w)), atol=1e-9)


@pytest.mark.parametrize("norder", [2, 5, 8])
def test_koornwinder_orthonormal(built, norder):
    U, V, W = _simplex_rule(2 * norder + 4)
    P = np.array([_pols(1, norder, (u, v)) for u, v in zip(U, V)])
    G = P.T @ (P * W[:, None])
    assert np.allclose(G, np.eye(P.shape[1]), atol=1e-12)


@pytest.mark.parametrize("norder", [3, 5, 8])
def test_quad_gl_nodes(built, norder):
    uvs, um, vm, w = _exps(11, norder)
    x, wg = np.polynomial.legendre.leggauss(norder + 1)
    assert np.allclose(uvs[: norder + 1, 0], x, atol=1e-14)   # ascending, u fastest
    assert np.allclose(uvs[:: norder + 1, 1], x, atol=1e-14)
    assert abs(w.sum() - 4.0) < 1e-13
    assert np.allclose(um @ vm, np.eye(len(w)), atol=1e-10)


def test_sphere_area_and_normals(sphere4):
    w = sphere4.qwts()
    assert abs(w.sum() - 4 * np.pi) < 1e-8
    x = sphere4.xyz
    assert np.allclose(np.linalg.norm(x, axis=1), 1.0, atol=1e-14)
    assert np.allclose(sphere4.normals, x, atol=1e-13)  # outward


def test_ellipsoid_volume(ellipsoid_small):
    s = S.icosa_ellipsoid(2, 6, (1.0, 2.0, 3.0))
    w = s.qwts()
    vol = np.sum(w * np.sum(s.xyz * s.normals, 1)) / 3.0  # divergence theorem
    assert abs(vol - 4 * np.pi / 3 * 6) < 1e-6


def test_torus_volume(built):
    s = S.torus_quad(32, 16, 5)
    w = s.qwts()
    vol = np.sum(w * np.sum(s.xyz * s.normals, 1)) / 3.0
    # V = 2 pi^2 R * mean(r(p)^2) = 2 pi^2 R (r0^2 + r1^2/2)
    exact = 2 * np.pi ** 2 * 2.0 * (0.6 ** 2 + 0.15 ** 2 / 2)
    assert abs(vol - exact) < 1e-7 * exact


def test_findnear_matches_brute_force(sphere4):
    cms, rads = S.get_centroid_rads(sphere4)
    rfac, _ = S.get_rfacs(4, 1)
    rp, ci = S.findnear(cms, rads * rfac, sphere4.srcvals)
    d2 = ((sphere4.xyz[:, None, :] - cms[None, :, :]) ** 2).sum(-1)
    brute = d2 <= (rads * rfac)[None, :] ** 2
    for i in range(0, sphere4.npts, 37):
        row = sorted(ci[rp[i] - 1: rp[i + 1] - 1] - 1)
        assert row == list(np.nonzero(brute[i])[0])
    assert rp[-1] - 1 == brute.sum()


def test_iquad_is_cumulative(sphere_lap_setup, sphere4):
    near = sphere_lap_setup.near
    npols = np.diff(sphere4.ixyzs)
    assert near.iquad[0] == 1
    assert np.array_equal(np.diff(near.iquad), npols[near.col_ind - 1])


def _dlaran_ref(iseed):
    # LAPACK DLARAN, written independently from its published definition
    m = [494, 322, 2508, 2549]
    s = [0, 0, 0, (2 * iseed + 1) % 4096]
    it4 = s[3] * m[3]; it3 = it4 // 4096; it4 -= 4096 * it3
    it3 += s[2] * m[3] + s[3] * m[2]; it2 = it3 // 4096; it3 -= 4096 * it2
    it2 += s[1] * m[3] + s[2] * m[2] + s[3] * m[1]; it1 = it2 // 4096; it2 -= 4096 * it1
    it1 += s[0] * m[3] + s[1] * m[2] + s[2] * m[1] + s[3] * m[0]; it1 %= 4096
    r = 1.0 / 4096
    return r * (it1 + r * (it2 + r * (it3 + r * it4)))


@pytest.mark.parametrize("seed", [1, 7, 1002, 1011, 3043, 3067, 4095])
def test_hkrand(built, seed):
    assert S.hkrand(seed) == _dlaran_ref(seed)


def test_far_order_and_oversampling(sphere4, sphere_lap_setup):
    over = sphere_lap_setup.over
    assert set(np.unique(over.novers)) <= {1, 2, 3, 4, 6, 8, 10, 12, 14, 16}
    # oversampled geometry lies on the sphere up to the order-4 interpolation error
    r = np.linalg.norm(over.srcover[:, :3], axis=1)
    assert np.max(np.abs(r - 1)) < 1e-4
    assert abs(over.wover.sum() - 4 * np.pi) < 1e-5
    # oversampling of a smooth function: x*y on the sphere
    f = sphere4.xyz[:, 0] * sphere4.xyz[:, 1]
    fo = S.oversample_fun_surf(sphere4, f, over.novers, over.ixyzso)
    assert np.max(np.abs(fo - over.srcover[:, 0] * over.srcover[:, 1])) < 1e-4


def test_oversample_matches_oracle(sphere4, sphere_lap_setup):
    import oracle
    over = sphere_lap_setup.over
    f = np.cos(sphere4.xyz @ np.array([0.3, -1.2, 0.7]))
    a = S.oversample_fun_surf(sphere4, f, over.novers, over.ixyzso)
    b = oracle.oversample_fun_surf(sphere4, f, over.novers, over.ixyzso)
    assert np.max(np.abs(a - b)) < 1e-13


def test_fmm_thresh(sphere4):
    t = S.get_fmm_thresh(sphere4.srcvals, sphere4.srcvals)
    x = sphere4.xyz
    assert t == 2.0 ** -51 * float(np.max(x.max(0) - x.min(0)))


def test_go3_roundtrip(tmp_path, sphere4):
    p = tmp_path / "s.go3"
    S.write_go3(sphere4, p)
    t = S.read_go3(p)
    assert t.npatches == sphere4.npatches and t.npts == sphere4.npts
    assert np.allclose(t.srcvals, sphere4.srcvals, atol=1e-15)
    assert np.allclose(t.srccoefs, sphere4.srccoefs, atol=1e-13)


def test_reference_go3_mesh_if_present(built):
    """Reads a mesh shipped with the reference (geometries/sphere_192_o03.go3)
    when FMM3DBIE_REFERENCE names a reference checkout."""
    import os
    root = os.environ.get("FMM3DBIE_REFERENCE")
    if not root:
        pytest.skip("FMM3DBIE_REFERENCE is not set")
    path = os.path.join(root, "geometries", "sphere_192_o03.go3")
    if not os.path.exists(path):
        pytest.skip("reference geometry not present")
    s = S.read_go3(path)
    assert s.npatches == 192 and s.npts == 1920
    assert abs(s.qwts().sum() - 4 * np.pi) < 1e-3


def test_chebyshev_torus_matches_legendre_torus():
    """The Chebyshev-node torus of the device tests describes the same surface
    as the Gauss-Legendre one: same area and the same near list sizes."""
    from _surfaces import torus_cheb
    from fmm3dbie_b200.warmstart import torus_surface
    tc = torus_cheb(16, 8, 5)
    tl = torus_surface(16, 8, 5)
    assert abs(tc.qwts().sum() - tl.qwts().sum()) < 1e-8 * tl.qwts().sum()
    assert np.all(tc.iptype == 12)
