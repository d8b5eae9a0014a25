"""Reference-shaped entry points for the combined-field Dirichlet path.

Each function takes host (numpy) arrays in the reference layout and calls
the matching C-ABI entry point of libfmm3dbie_b200.so (host buffers in, host
buffers out; the work runs on the current CUDA device):

  lap:  lpcomp_lap_comb_dir_addsub   lap_comb_dir.f90:633
        lap_comb_dir_eval_addsub     lap_comb_dir.f90:806
        lap_comb_dir_eval            lap_comb_dir.f90:408
        lap_comb_dir_solver          lap_comb_dir.f90:1189
        lap_comb_dir_solver_guru     lap_comb_dir.f90:1459
  helm: lpcomp_helm_comb_dir_addsub  helm_comb_dir.f:658
        helm_comb_dir_eval_addsub    helm_comb_dir.f:856
        helm_comb_dir_eval           helm_comb_dir.f:440
        lpcomp_helm_comb_dir         (the f2py name of helm_comb_dir_eval,
                                      python/setup.py:39)
        helm_comb_dir_solver         helm_comb_dir.f:1808
        helm_comb_dir_solver_guru    helm_comb_dir.f:2071

Errors raise fmm3dbie_b200.BieError; GMRES non-convergence is reported in
the returned status like the reference (which returns niter = numit).
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .surface import NearField, Oversampled, Surface


def _lib():
    lib = L.lib()
    L.check(lib.bie_init(None), "bie_init")
    return lib


def _near(near: NearField, cplx: bool):
    w = np.ascontiguousarray(near.wnear, complex if cplx else float)
    wv = w.view(float) if cplx else w
    return (near.nnz, L.ptr(near.row_ptr), L.ptr(near.col_ind), L.ptr(near.iquad), near.nquad), wv


def _over(over: Oversampled):
    return (L.ptr(over.novers), over.nptso, L.ptr(over.ixyzso), L.ptr(over.srcover),
            L.ptr(over.wover))


def _zp(zpars):
    return np.ascontiguousarray(np.asarray(zpars, complex)).view(float)


def _cv(x):
    x = np.ascontiguousarray(x, complex)
    return x, x.view(float)


# ---- Laplace ----------------------------------------------------------------
def lpcomp_lap_comb_dir_addsub(surf: Surface, eps, dpars, near: NearField, over: Oversampled,
                               sigma):
    lib = _lib()
    dp = np.asarray(dpars, float)
    sig = np.ascontiguousarray(sigma, float)
    pot = np.zeros(surf.npts)
    (nnz, rp, ci, iq, nq), wv = _near(near, False)
    L.check(lib.bie_lpcomp_lap_comb_dir_addsub(*surf.args(), eps, 2, L.ptr(dp), 0, None, 0, None,
                                               nnz, rp, ci, iq, nq, 1, L.ptr(wv), *_over(over), 0,
                                               None, 1, L.ptr(sig), L.ptr(pot)),
            "lpcomp_lap_comb_dir_addsub")
    return pot


def lap_comb_dir_eval_addsub(surf: Surface, targs, eps, dpars, near: NearField,
                             over: Oversampled, sigma):
    lib = _lib()
    targs = np.ascontiguousarray(targs, float)
    dp = np.asarray(dpars, float)
    sig = np.ascontiguousarray(sigma, float)
    pot = np.zeros(targs.shape[0])
    (nnz, rp, ci, iq, nq), wv = _near(near, False)
    L.check(lib.bie_lap_comb_dir_eval_addsub(*surf.args(), targs.shape[1], targs.shape[0],
                                             L.ptr(targs), eps, L.ptr(dp), nnz, rp, ci, iq, nq,
                                             L.ptr(wv), *_over(over), L.ptr(sig), L.ptr(pot)),
            "lap_comb_dir_eval_addsub")
    return pot


def lap_comb_dir_eval(surf: Surface, targs, ipatch_id, uvs_targ, eps, dpars, sigma):
    lib = _lib()
    targs = np.ascontiguousarray(targs, float)
    nt = targs.shape[0]
    ipatch_id = np.ascontiguousarray(ipatch_id if ipatch_id is not None else -np.ones(nt), np.int64)
    uvs_targ = np.ascontiguousarray(uvs_targ if uvs_targ is not None else np.zeros((nt, 2)), float)
    dp = np.asarray(dpars, float)
    sig = np.ascontiguousarray(sigma, float)
    pot = np.zeros(nt)
    L.check(lib.bie_lap_comb_dir_eval(*surf.args(), targs.shape[1], nt, L.ptr(targs),
                                      L.ptr(ipatch_id), L.ptr(uvs_targ), eps, L.ptr(dp), L.ptr(sig),
                                      L.ptr(pot)), "lap_comb_dir_eval")
    return pot


def lap_comb_dir_solver(surf: Surface, eps, dpars, numit, ifinout, rhs, eps_gmres):
    """Returns (niter, errs, rres, soln, status)."""
    lib = _lib()
    dp = np.asarray(dpars, float)
    r = np.ascontiguousarray(rhs, float)
    soln = np.zeros(surf.npts)
    errs = np.zeros(numit + 1)
    niter = np.zeros(1, np.int64)
    rres = np.zeros(1)
    st = lib.bie_lap_comb_dir_solver(*surf.args(), eps, L.ptr(dp), numit, ifinout, L.ptr(r),
                                     eps_gmres, L.ptr(niter), L.ptr(errs), L.ptr(rres), L.ptr(soln))
    if st not in (0, 3, 4):
        L.check(st, "lap_comb_dir_solver")
    return int(niter[0]), errs, float(rres[0]), soln, st


def lap_comb_dir_solver_guru(surf: Surface, eps, dpars, numit, ifinout, rhs, near: NearField,
                             over: Oversampled, eps_gmres):
    lib = _lib()
    dp = np.asarray(dpars, float)
    r = np.ascontiguousarray(rhs, float)
    soln = np.zeros(surf.npts)
    errs = np.zeros(numit + 1)
    niter = np.zeros(1, np.int64)
    rres = np.zeros(1)
    (nnz, rp, ci, iq, nq), wv = _near(near, False)
    st = lib.bie_lap_comb_dir_solver_guru(*surf.args(), eps, L.ptr(dp), numit, ifinout, L.ptr(r),
                                          nnz, rp, ci, iq, nq, 1, L.ptr(wv), *_over(over),
                                          eps_gmres, L.ptr(niter), L.ptr(errs), L.ptr(rres),
                                          L.ptr(soln))
    if st not in (0, 3, 4):
        L.check(st, "lap_comb_dir_solver_guru")
    return int(niter[0]), errs, float(rres[0]), soln, st


# ---- Helmholtz ----------------------------------------------------------------
def lpcomp_helm_comb_dir_addsub(surf: Surface, eps, zpars, near: NearField, over: Oversampled,
                                sigma):
    lib = _lib()
    zp = _zp(zpars)
    _, sv = _cv(sigma)
    pot = np.zeros(surf.npts, complex)
    (nnz, rp, ci, iq, nq), wv = _near(near, True)
    L.check(lib.bie_lpcomp_helm_comb_dir_addsub(*surf.args(), eps, 0, None, 3, L.ptr(zp), 0, None,
                                                nnz, rp, ci, iq, nq, 1, L.ptr(wv), *_over(over), 0,
                                                None, 1, L.ptr(sv), L.ptr(pot.view(float))),
            "lpcomp_helm_comb_dir_addsub")
    return pot


def helm_comb_dir_eval_addsub(surf: Surface, targs, eps, zpars, near: NearField,
                              over: Oversampled, sigma):
    lib = _lib()
    targs = np.ascontiguousarray(targs, float)
    zp = _zp(zpars)
    _, sv = _cv(sigma)
    pot = np.zeros(targs.shape[0], complex)
    (nnz, rp, ci, iq, nq), wv = _near(near, True)
    L.check(lib.bie_helm_comb_dir_eval_addsub(*surf.args(), targs.shape[1], targs.shape[0],
                                              L.ptr(targs), eps, L.ptr(zp), nnz, rp, ci, iq, nq,
                                              L.ptr(wv), *_over(over), L.ptr(sv),
                                              L.ptr(pot.view(float))), "helm_comb_dir_eval_addsub")
    return pot


def helm_comb_dir_eval(surf: Surface, targs, ipatch_id, uvs_targ, eps, zpars, sigma):
    lib = _lib()
    targs = np.ascontiguousarray(targs, float)
    nt = targs.shape[0]
    ipatch_id = np.ascontiguousarray(ipatch_id if ipatch_id is not None else -np.ones(nt), np.int64)
    uvs_targ = np.ascontiguousarray(uvs_targ if uvs_targ is not None else np.zeros((nt, 2)), float)
    zp = _zp(zpars)
    _, sv = _cv(sigma)
    pot = np.zeros(nt, complex)
    L.check(lib.bie_helm_comb_dir_eval(*surf.args(), targs.shape[1], nt, L.ptr(targs),
                                       L.ptr(ipatch_id), L.ptr(uvs_targ), eps, L.ptr(zp),
                                       L.ptr(sv), L.ptr(pot.view(float))), "helm_comb_dir_eval")
    return pot


def lpcomp_helm_comb_dir(norders, ixyzs, iptype, srccoefs, srcvals, targs, ipatch_id, uvs_targ,
                         eps, zpars, sigma):
    """The f2py binding's call shape (python/helm3d_dirsolver_csc_demo.py:62):
    Fortran-shaped srccoefs (9,npts), srcvals (12,npts), targs (ndt,ntarg)
    are accepted as well as their point-major transposes."""
    def pm(a, rows):
        a = np.asarray(a, float)
        return np.ascontiguousarray(a.T if a.shape[0] == rows and a.shape[1] != rows else a)
    sv = pm(srcvals, 12)
    sc = pm(srccoefs, 9)
    t = np.asarray(targs, float)
    if t.ndim == 2 and t.shape[0] in (3, 12) and t.shape[1] not in (3, 12):
        t = t.T
    uv = np.asarray(uvs_targ, float)
    if uv.ndim == 2 and uv.shape[0] == 2 and uv.shape[1] != 2:
        uv = uv.T
    surf = Surface(np.ascontiguousarray(norders, np.int64), np.ascontiguousarray(ixyzs, np.int64),
                   np.ascontiguousarray(iptype, np.int64), sv, sc)
    return helm_comb_dir_eval(surf, np.ascontiguousarray(t), ipatch_id, uv, eps, zpars, sigma)


def helm_comb_dir_solver(surf: Surface, eps, zpars, numit, ifinout, rhs, eps_gmres):
    lib = _lib()
    zp = _zp(zpars)
    _, rv = _cv(rhs)
    soln = np.zeros(surf.npts, complex)
    errs = np.zeros(numit + 1)
    niter = np.zeros(1, np.int64)
    rres = np.zeros(1)
    st = lib.bie_helm_comb_dir_solver(*surf.args(), eps, L.ptr(zp), numit, ifinout, L.ptr(rv),
                                      eps_gmres, L.ptr(niter), L.ptr(errs), L.ptr(rres),
                                      L.ptr(soln.view(float)))
    if st not in (0, 3, 4):
        L.check(st, "helm_comb_dir_solver")
    return int(niter[0]), errs, float(rres[0]), soln, st


def helm_comb_dir_solver_guru(surf: Surface, eps, zpars, numit, ifinout, rhs, near: NearField,
                              over: Oversampled, eps_gmres):
    lib = _lib()
    zp = _zp(zpars)
    _, rv = _cv(rhs)
    soln = np.zeros(surf.npts, complex)
    errs = np.zeros(numit + 1)
    niter = np.zeros(1, np.int64)
    rres = np.zeros(1)
    (nnz, rp, ci, iq, nq), wv = _near(near, True)
    st = lib.bie_helm_comb_dir_solver_guru(*surf.args(), eps, L.ptr(zp), numit, ifinout,
                                           L.ptr(rv), nnz, rp, ci, iq, nq, 1, L.ptr(wv),
                                           *_over(over), eps_gmres, L.ptr(niter), L.ptr(errs),
                                           L.ptr(rres), L.ptr(soln.view(float)))
    if st not in (0, 3, 4):
        L.check(st, "helm_comb_dir_solver_guru")
    return int(niter[0]), errs, float(rres[0]), soln, st


def helm_comb_dir_solver_guru_ext(surf: Surface, eps, zpars, numit, ifinout, rhs,
                                  near: NearField, over: Oversampled, eps_gmres, iprec=1):
    """nrhs independent right-hand sides rhs (npts, nrhs); iprec 1 = mixed
    precision refinement.  Returns (niter[nrhs], rres[nrhs], soln, status)."""
    lib = _lib()
    zp = _zp(zpars)
    r = np.asarray(rhs, complex)
    if r.ndim == 1:
        r = r[:, None]
    nrhs = r.shape[1]
    _, rv = _cv(r)
    soln = np.zeros((surf.npts, nrhs), complex)
    niter = np.zeros(nrhs, np.int64)
    rres = np.zeros(nrhs)
    (nnz, rp, ci, iq, nq), wv = _near(near, True)
    st = lib.bie_helm_comb_dir_solver_guru_ext(*surf.args(), eps, L.ptr(zp), numit, ifinout, nrhs,
                                               L.ptr(rv), nnz, rp, ci, iq, nq, L.ptr(wv),
                                               *_over(over), eps_gmres, iprec, L.ptr(niter),
                                               L.ptr(rres), L.ptr(soln.view(float)))
    if st not in (0, 3, 4):
        L.check(st, "helm_comb_dir_solver_guru_ext")
    return niter, rres, soln, st
