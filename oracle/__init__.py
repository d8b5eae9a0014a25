"""FP64 CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package; the product never does.  See oracle.c for the reference
routines restated and for the parity status.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "oracle.c")
LIB = os.path.join(HERE, "liboracle.so")

I64 = C.c_int64
PI64 = C.POINTER(C.c_int64)
PDBL = C.POINTER(C.c_double)


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.run(["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", SRC,
                        "-o", LIB + ".tmp", "-lm"], check=True)
        os.replace(LIB + ".tmp", LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.oracle_set_vr_nodes.argtypes = [I64, I64, PDBL]
        L.oracle_eval_addsub.argtypes = [I64, I64, PI64, PI64, PI64, I64, I64, I64, PDBL, PDBL,
                                         I64, PI64, PI64, PI64, PDBL, PI64, I64, PI64, PDBL, PDBL,
                                         PDBL, PDBL]
        L.oracle_gmres.argtypes = [I64, I64, PI64, PI64, PI64, I64, PDBL, PDBL, PDBL, I64, PI64,
                                   PI64, PI64, PDBL, PI64, I64, PI64, PDBL, PDBL, PDBL, PDBL,
                                   I64, C.c_double, PI64, PDBL, PDBL, PDBL]
        L.oracle_oversample_fun_surf.argtypes = [I64, I64, PI64, PI64, PI64, I64, PDBL, PI64,
                                                 PI64, I64, PDBL]
        L.oracle_fmm_thresh.argtypes = [I64, PDBL, I64, I64, PDBL, I64]
        L.oracle_fmm_thresh.restype = C.c_double
        _lib = L
        _load_nodes(L)
    return _lib


def _load_nodes(L):
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from fmm3dbie_b200 import tables
    t = tables.read_table()
    for n, (uvs, _w) in t.items():
        a = np.ascontiguousarray(uvs, float)
        L.oracle_set_vr_nodes(n, len(uvs) // 2, a.ctypes.data_as(PDBL))


def _p(a):
    if a is None:
        return None
    if a.dtype == np.int64:
        return a.ctypes.data_as(PI64)
    return a.ctypes.data_as(PDBL)


def _f(a, dt=float):
    return np.ascontiguousarray(a, dtype=dt)


def _params(kind, params):
    if kind == 0:
        return _f(params, float)
    return np.ascontiguousarray(np.asarray(params, complex)).view(float)


def eval_addsub(kind, surf, targs, params, near, over, sigma):
    """lpcomp / eval_addsub restated; returns pot (float64 or complex128)."""
    L = lib()
    targs = _f(targs)
    nt = targs.shape[0]
    sig = _f(sigma, float if kind == 0 else complex)
    sigv = sig if kind == 0 else sig.view(float)
    w = _f(near.wnear, float if kind == 0 else complex)
    wv = w if kind == 0 else w.view(float)
    pot = np.zeros(nt, float if kind == 0 else complex)
    potv = pot if kind == 0 else pot.view(float)
    pr = _params(kind, params)
    ier = L.oracle_eval_addsub(kind, surf.npatches, _p(surf.norders), _p(surf.ixyzs),
                               _p(surf.iptype), surf.npts, targs.shape[1], nt, _p(targs), _p(pr),
                               near.nnz, _p(near.row_ptr), _p(near.col_ind), _p(near.iquad), _p(wv),
                               _p(over.novers), over.nptso, _p(over.ixyzso), _p(over.srcover),
                               _p(over.wover), _p(sigv), _p(potv))
    if ier:
        raise RuntimeError(f"oracle_eval_addsub failed ({ier})")
    return pot


def lpcomp(kind, surf, params, near, over, sigma):
    return eval_addsub(kind, surf, surf.srcvals, params, near, over, sigma)


def oversample_fun_surf(surf, u, novers, ixyzso):
    L = lib()
    u = _f(u)
    nd = 1 if u.ndim == 1 else u.shape[1]
    nptso = int(ixyzso[-1] - 1)
    out = np.zeros((nptso, nd)) if u.ndim > 1 else np.zeros(nptso)
    ier = L.oracle_oversample_fun_surf(nd, surf.npatches, _p(surf.norders), _p(surf.ixyzs),
                                       _p(surf.iptype), surf.npts, _p(u), _p(_f(novers, np.int64)),
                                       _p(_f(ixyzso, np.int64)), nptso, _p(out))
    if ier:
        raise RuntimeError(f"oracle_oversample_fun_surf failed ({ier})")
    return out


def gmres(kind, surf, params, near, over, zid, rhs, numit=200, eps_gmres=1e-10):
    """zgmres_guru / dgmres_guru restated with the oracle matvec."""
    L = lib()
    wts = surf.qwts()
    r = _f(rhs, float if kind == 0 else complex)
    rv = r if kind == 0 else r.view(float)
    soln = np.zeros(surf.npts, float if kind == 0 else complex)
    sv = soln if kind == 0 else soln.view(float)
    w = _f(near.wnear, float if kind == 0 else complex)
    wv = w if kind == 0 else w.view(float)
    pr = _params(kind, params)
    z = np.array([complex(zid).real, complex(zid).imag])
    niter = np.zeros(1, np.int64)
    errs = np.zeros(numit + 1)
    rres = np.zeros(1)
    st = L.oracle_gmres(kind, surf.npatches, _p(surf.norders), _p(surf.ixyzs), _p(surf.iptype),
                        surf.npts, _p(surf.srcvals), _p(wts), _p(pr), near.nnz, _p(near.row_ptr),
                        _p(near.col_ind), _p(near.iquad), _p(wv), _p(over.novers), over.nptso,
                        _p(over.ixyzso), _p(over.srcover), _p(over.wover), _p(z), _p(rv), numit,
                        eps_gmres, _p(niter), _p(errs), _p(rres), _p(sv))
    return soln, int(niter[0]), errs[: int(niter[0])], float(rres[0]), st
