"""GPU GMRES solvers against the oracle GMRES (zgmres_guru / dgmres_guru,
gmres_routs.f90:13,375) and against analytic point-source fields."""
import numpy as np
import pytest

import oracle
from fmm3dbie_b200 import Plan, layer
from fmm3dbie_b200 import surface as S
from conftest import wnorm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def _ps(k, x0, x):
    r = np.linalg.norm(x - x0, axis=1)
    return np.exp(1j * k * r) / (4 * np.pi * r)


def _exterior_field(s, soln, zp, targ):
    k = zp[0]
    w = s.qwts()
    dx = targ[:, None, :] - s.xyz[None, :, :]
    r = np.linalg.norm(dx, axis=2)
    dn = np.sum(dx * s.normals[None], 2)
    ker = (zp[1] / r + zp[2] * dn * (1 - 1j * k * r) / r ** 3) * np.exp(1j * k * r) / (4 * np.pi)
    return ker @ (w * soln)


def test_helmholtz_gmres_matches_oracle(torch, ellipsoid_small, ellipsoid_helm_setup):
    s, st = ellipsoid_small, ellipsoid_helm_setup
    zp = (2.0, -2.0j, 1.0)
    rhs = _ps(2.0, np.array([0.1, -0.2, 0.3]), s.xyz)
    ref, nit_ref, errs_ref, rres_ref, _ = oracle.gmres(1, s, zp, st.near, st.over, 0.5, rhs,
                                                      numit=100, eps_gmres=1e-10)
    niter, errs, rres, soln, status = layer.helm_comb_dir_solver_guru(
        s, 1e-7, zp, 100, 1, rhs, st.near, st.over, 1e-10)
    assert status == 0
    assert abs(niter - nit_ref) <= 1
    assert rres < 1e-9
    w = s.qwts()
    assert wnorm(w, soln - ref) / wnorm(w, ref) < 1e-9
    # residual history tracks the oracle's
    m = min(niter, nit_ref) - 1
    assert np.allclose(np.log10(errs[:m]), np.log10(errs_ref[:m]), atol=0.05)


def test_laplace_gmres_matches_oracle(torch, sphere4, sphere_lap_setup):
    s, st = sphere4, sphere_lap_setup
    x0 = np.array([0.1, 0.2, -0.3])
    rhs = 1 / (4 * np.pi * np.linalg.norm(s.xyz - x0, axis=1))
    ref, nit_ref, _, _, _ = oracle.gmres(0, s, (1.0, 1.0), st.near, st.over, 0.5, rhs, numit=60,
                                         eps_gmres=1e-10)
    niter, errs, rres, soln, status = layer.lap_comb_dir_solver_guru(
        s, 1e-6, (1.0, 1.0), 60, 1, rhs, st.near, st.over, 1e-10)
    assert status == 0 and abs(niter - nit_ref) <= 1 and rres < 1e-9
    w = s.qwts()
    assert wnorm(w, soln - ref) / wnorm(w, ref) < 1e-9


def test_simple_solver_equals_guru(torch, ellipsoid_small, ellipsoid_helm_setup):
    """helm_comb_dir_solver (setup inside) == guru path (test_helm_wrappers_qg_lp.f:285)."""
    s, st = ellipsoid_small, ellipsoid_helm_setup
    zp = (2.0, -2.0j, 1.0)
    rhs = _ps(2.0, np.array([0.1, -0.2, 0.3]), s.xyz)
    a = layer.helm_comb_dir_solver(s, 1e-7, zp, 100, 1, rhs, 1e-10)
    b = layer.helm_comb_dir_solver_guru(s, 1e-7, zp, 100, 1, rhs, st.near, st.over, 1e-10)
    assert a[0] == b[0]
    assert np.max(np.abs(a[3] - b[3])) < 1e-12 * np.max(np.abs(b[3]))


def test_mixed_precision_solve(torch, ellipsoid_small, ellipsoid_helm_setup):
    s, st = ellipsoid_small, ellipsoid_helm_setup
    zp = (2.0, -2.0j, 1.0)
    x0 = np.array([0.1, -0.2, 0.3])
    rhs = _ps(2.0, x0, s.xyz)
    P = Plan(1, zp, s, st.near, st.over)
    r = torch.tensor(rhs, device="cuda")
    x64, i64 = P.solve(r, 0.5, mode=0, numit=100, eps_gmres=1e-12)
    xm, im = P.solve(r, 0.5, mode=1, numit=100, eps_gmres=1e-10)
    assert i64["status"] == 0 and im["status"] == 0
    assert im["rres"][0] <= 1e-10
    w = s.qwts()
    a, b = x64.cpu().numpy(), xm.cpu().numpy()
    assert wnorm(w, a - b) / wnorm(w, a) < 1e-9
    # exterior field against the analytic point source (second oracle)
    rng = np.random.default_rng(2)
    d = rng.normal(size=(100, 3))
    targ = 5 * d / np.linalg.norm(d, axis=1)[:, None]
    u = _exterior_field(s, b, zp, targ)
    ue = _ps(2.0, x0, targ)
    assert np.max(np.abs(u - ue)) / np.max(np.abs(ue)) < 1e-5


def test_batched_systems_match_individual(torch, ellipsoid_small, ellipsoid_helm_setup):
    s, st = ellipsoid_small, ellipsoid_helm_setup
    zp = (2.0, -2.0j, 1.0)
    rng = np.random.default_rng(3)
    dirs = rng.normal(size=(4, 3))
    dirs /= np.linalg.norm(dirs, axis=1)[:, None]
    rhs = -np.exp(1j * 2.0 * s.xyz @ dirs.T)  # minus incident plane waves
    P = Plan(1, zp, s, st.near, st.over)
    R = torch.tensor(rhs, device="cuda")
    for mode in (0, 1):
        X, info = P.solve(R, 0.5, mode=mode, numit=100, eps_gmres=1e-10)
        X = X.cpu().numpy()
        for m in range(4):
            x1, _ = P.solve(R[:, m].contiguous(), 0.5, mode=mode, numit=100, eps_gmres=1e-10)
            x1 = x1.cpu().numpy()
            assert np.max(np.abs(X[:, m] - x1)) < 1e-8 * np.max(np.abs(x1))
    # host ext entry point, batched mixed precision
    niter, rres, soln, stt = layer.helm_comb_dir_solver_guru_ext(s, 1e-7, zp, 100, 1, rhs, st.near,
                                                                  st.over, 1e-10, iprec=1)
    assert stt == 0 and np.all(rres <= 1e-10)
    assert np.max(np.abs(soln - X)) < 1e-8 * np.max(np.abs(X))


def test_host_buffer_solve_matches_device_plan(torch, ellipsoid_small, ellipsoid_helm_setup):
    """The host-buffer solver uploads the near quadrature in near-pair chunks
    whose folds run on their own stream beside the solve's first far field;
    from pinned buffers that overlap is real.  Its solution must be the
    device-resident plan's (same kernels, same W_eff)."""
    s, st = ellipsoid_small, ellipsoid_helm_setup
    zp = (2.0, -2.0j, 1.0)
    assert st.near.row_ptr[-1] - 1 >= 8 * 1024  # enough near pairs for the chunked upload
    rhs = _ps(2.0, np.array([0.1, -0.2, 0.3]), s.xyz)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    near_p = S.NearField(pin(st.near.row_ptr), pin(st.near.col_ind), pin(st.near.iquad),
                         pin(st.near.wnear))
    P = Plan(1, zp, s, st.near, st.over)
    xd, info = P.solve(torch.tensor(rhs, device="cuda"), 0.5, mode=1, numit=100,
                       eps_gmres=1e-10)
    xd = xd.cpu().numpy()
    w = s.qwts()
    for _ in range(2):  # the second call reuses the pinned staging of the first
        niter, rres, soln, status = layer.helm_comb_dir_solver_guru_ext(
            s, 1e-7, zp, 100, 1, pin(rhs[:, None]), near_p, st.over, 1e-10, iprec=1)
        assert status == 0 and rres[0] <= 1e-10
        assert niter[0] == info["niter"][0]
        assert wnorm(w, soln[:, 0] - xd) / wnorm(w, xd) < 1e-12


def test_concurrent_plan_builds(torch, ellipsoid_small, ellipsoid_helm_setup):
    """Plan builds in two threads at once: one stages its host arrays in the
    library's pinned buffer, the other in pageable memory; both operators
    equal a plan built alone."""
    import threading
    s, st = ellipsoid_small, ellipsoid_helm_setup
    zp = (2.0, -2.0j, 1.0)
    rng = np.random.default_rng(11)
    sig = rng.normal(size=s.npts) + 1j * rng.normal(size=s.npts)
    ref_plan = Plan(1, zp, s, st.near, st.over)
    x = torch.tensor(sig, device="cuda")
    ref = {p: ref_plan.matvec(x, p).cpu().numpy() for p in (0, 1)}
    out, errs = {}, []
    barrier = threading.Barrier(2)

    def work(i):
        try:
            barrier.wait()
            P = Plan(1, zp, s, st.near, st.over)
            out[i] = {p: P.matvec(x, p).cpu().numpy() for p in (0, 1)}
            P.close()
        except Exception as e:  # reported below, in the test's own thread
            errs.append(e)

    th = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for i in range(2):
        for p in (0, 1):
            d = np.linalg.norm(out[i][p] - ref[p]) / np.linalg.norm(ref[p])
            assert d < 1e-13, (i, p, d)
