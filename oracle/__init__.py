"""FP64 CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this
package; the product never does, and this package imports nothing from the
product.  oracle.c restates the matvec (lpcomp_*_comb_dir_addsub) and GMRES;
oracle_setup.c the surfaces and the setup (near list, far orders,
oversampled geometry, weights, near quadrature); see those files for the
reference routines restated and for the parity status.
"""
from __future__ import annotations

import ctypes as C
import glob
import math
import os
import struct
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRCS = sorted(glob.glob(os.path.join(HERE, "*.c")))
HDRS = sorted(glob.glob(os.path.join(HERE, "*.h")))
LIB = os.path.join(HERE, "liboracle.so")
# Vioreanu-Rokhlin node/weight tables written at build time from the
# reference's koorn-*.txt (layout: b"BIEVR001", int32 nmax, then per order
# int32 npols, float64 uvs[2 npols], float64 wts[npols])
VR_TABLE = os.path.join(os.path.dirname(HERE), "fmm3dbie_b200", "_data", "vioreanu_rokhlin.bin")

I64 = C.c_int64
PI64 = C.POINTER(C.c_int64)
PDBL = C.POINTER(C.c_double)


# oracle_far.c (the timed far field) is built with -ffast-math so that its
# loops vectorise onto libmvec's sine and cosine; the parity code is not.
CFLAGS = ["-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC"]
FAST = {"oracle_far.c": ["-ffast-math"]}


def build(force: bool = False) -> str:
    deps = SRCS + HDRS
    if force or not os.path.exists(LIB) or any(os.path.getmtime(LIB) < os.path.getmtime(d)
                                               for d in deps):
        objs = []
        for src in SRCS:
            obj = os.path.join(HERE, "_" + os.path.basename(src) + ".o")
            subprocess.run(["gcc"] + CFLAGS + FAST.get(os.path.basename(src), []) +
                           ["-c", src, "-o", obj], check=True)
            objs.append(obj)
        subprocess.run(["gcc", "-shared", "-fopenmp"] + objs + ["-o", LIB + ".tmp", "-lmvec",
                                                                "-lm"], check=True)
        for o in objs:
            os.remove(o)
        os.replace(LIB + ".tmp", LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.oracle_set_vr_nodes.argtypes = [I64, I64, PDBL]
        L.oracle_set_vr_table.argtypes = [I64, I64, PDBL, PDBL]
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
        L.oracle_icosa_npatches.argtypes = [I64]
        L.oracle_icosa_npatches.restype = I64
        L.oracle_surf_icosa_ellipsoid.argtypes = [I64, I64, PDBL, PDBL, PI64, PI64, PI64, PDBL,
                                                  PDBL]
        L.oracle_surf_torus_quad.argtypes = [I64, I64, I64, C.c_double, C.c_double, C.c_double,
                                             I64, PI64, PI64, PI64, PDBL, PDBL]
        L.oracle_get_qwts.argtypes = [I64, PI64, PI64, PI64, I64, PDBL, PDBL]
        L.oracle_get_rfacs.argtypes = [I64, I64, PDBL, PDBL]
        L.oracle_get_rfacs.restype = None
        L.oracle_get_centroid_rads.argtypes = [I64, PI64, PI64, PI64, I64, PDBL, PDBL, PDBL]
        L.oracle_findnear.argtypes = [PDBL, I64, PDBL, I64, PDBL, I64, PI64, PI64]
        L.oracle_hkrand.argtypes = [I64]
        L.oracle_hkrand.restype = C.c_double
        L.oracle_get_far_order.argtypes = [C.c_double, I64, PI64, PI64, PI64, PDBL, PDBL, I64,
                                           PDBL, I64, I64, PDBL, I64, PDBL, I64, PI64, PI64,
                                           C.c_double, PI64, PI64]
        L.oracle_oversample_geom.argtypes = [I64, PI64, PI64, PI64, I64, PDBL, PDBL, PI64, PI64,
                                             I64, PDBL]
        L.oracle_set_far_method.argtypes = [I64, C.c_double, I64, I64]
        L.oracle_set_nq_tol.argtypes = [C.c_double]
        L.oracle_set_nq_tol.restype = None
        L.oracle_getnearquad.argtypes = [I64, I64, PI64, PI64, PI64, I64, PDBL, PDBL, I64, I64,
                                         PDBL, PI64, PDBL, C.c_double, PDBL, I64, PI64, PI64,
                                         PI64, I64, PDBL, PI64]
        _lib = L
        _load_nodes(L)
    return _lib


def read_vr_table(path: str = VR_TABLE):
    """{norder: (uvs[2*npols], wts[npols])} from the build's table file."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != b"BIEVR001":
        raise ValueError(f"{path}: not a Vioreanu-Rokhlin table file")
    (nmax,) = struct.unpack_from("<i", data, 8)
    off, out = 12, {}
    for n in range(nmax + 1):
        (npols,) = struct.unpack_from("<i", data, off)
        off += 4
        uvs = np.frombuffer(data, "<f8", 2 * npols, off).copy()
        off += 16 * npols
        wts = np.frombuffer(data, "<f8", npols, off).copy()
        off += 8 * npols
        out[n] = (uvs, wts)
    return out


def _load_nodes(L):
    for n, (uvs, wts) in read_vr_table().items():
        L.oracle_set_vr_table(n, len(wts), uvs.ctypes.data_as(PDBL), wts.ctypes.data_as(PDBL))


def set_far_method(method: int, theta: float = 0.0, ncheb: int = 0, leaf: int = 0) -> None:
    """Far field of the oracle's matvec: 0 exact scalar direct sum (the parity
    oracle, default); 1 vectorised direct sum; 2 barycentric Lagrange
    treecode (theta, Chebyshev points per side, sources per leaf; 0 keeps
    the current values, initially 0.5, 9, 256).  Methods 1 and 2 stand in
    for the FMM in timed CPU solves."""
    if lib().oracle_set_far_method(method, theta, ncheb, leaf):
        raise ValueError(f"bad far-field method {method}")


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
    wts = qwts(surf)
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


# ---- surfaces and setup (oracle_setup.c) -----------------------------------
@dataclass
class OSurface:
    """The reference's discretisation arrays (as the product's Surface)."""
    norders: np.ndarray
    ixyzs: np.ndarray
    iptype: np.ndarray
    srcvals: np.ndarray
    srccoefs: np.ndarray

    @property
    def npatches(self):
        return int(self.norders.shape[0])

    @property
    def npts(self):
        return int(self.srcvals.shape[0])

    @property
    def xyz(self):
        return self.srcvals[:, 0:3]

    @property
    def normals(self):
        return self.srcvals[:, 9:12]

    def qwts(self):
        return qwts(self)


@dataclass
class ONear:
    row_ptr: np.ndarray
    col_ind: np.ndarray
    iquad: np.ndarray
    wnear: np.ndarray

    @property
    def nnz(self):
        return int(self.col_ind.shape[0])

    @property
    def nquad(self):
        return int(self.iquad[-1] - 1)


@dataclass
class OOver:
    novers: np.ndarray
    ixyzso: np.ndarray
    srcover: np.ndarray
    wover: np.ndarray

    @property
    def nptso(self):
        return int(self.srcover.shape[0])


@dataclass
class OSetup:
    near: ONear
    over: OOver
    rfac: float
    rfac0: float
    cms: np.ndarray = field(repr=False)
    rads: np.ndarray = field(repr=False)
    kernel_evals: int = 0


def _surf_arrays(npat, npols):
    npts = npat * npols
    return (np.zeros(npat, np.int64), np.zeros(npat + 1, np.int64), np.zeros(npat, np.int64),
            np.zeros((npts, 12)), np.zeros((npts, 9)))


def icosa_ellipsoid(nref, norder, axes=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0)) -> OSurface:
    """xtri_platonic icosahedron refined nref times, radially projected onto
    center + axes * x/|x| (xtri_ellipsoid_eval), order-norder RV nodes."""
    L = lib()
    npat = int(L.oracle_icosa_npatches(nref))
    a = _surf_arrays(npat, (norder + 1) * (norder + 2) // 2)
    ax, ce = _f(axes), _f(center)
    ier = L.oracle_surf_icosa_ellipsoid(nref, norder, _p(ax), _p(ce), *(_p(x) for x in a))
    if ier:
        raise RuntimeError(f"oracle_surf_icosa_ellipsoid failed ({ier})")
    return OSurface(*a)


def torus_quad(nu, nv, norder, R=2.0, r0=0.6, r1=0.15, m=3) -> OSurface:
    L = lib()
    a = _surf_arrays(nu * nv, (norder + 1) ** 2)
    ier = L.oracle_surf_torus_quad(nu, nv, norder, R, r0, r1, m, *(_p(x) for x in a))
    if ier:
        raise RuntimeError(f"oracle_surf_torus_quad failed ({ier})")
    return OSurface(*a)


def _sargs(s):
    return (s.npatches, _p(_f(s.norders, np.int64)), _p(_f(s.ixyzs, np.int64)),
            _p(_f(s.iptype, np.int64)), s.npts)


def qwts(s) -> np.ndarray:
    L = lib()
    w = np.zeros(s.npts)
    sv = _f(s.srcvals)
    ier = L.oracle_get_qwts(*_sargs(s), _p(sv), _p(w))
    if ier:
        raise RuntimeError(f"oracle_get_qwts failed ({ier})")
    return w


def rfacs(norder, iptype):
    a, b = C.c_double(), C.c_double()
    lib().oracle_get_rfacs(norder, iptype, C.byref(a), C.byref(b))
    return a.value, b.value


def centroid_rads(s):
    cms = np.zeros((s.npatches, 3))
    rads = np.zeros(s.npatches)
    lib().oracle_get_centroid_rads(*_sargs(s), _p(_f(s.srccoefs)), _p(cms), _p(rads))
    return cms, rads


def findnear(cms, rad_near, targs):
    """Brute-force near list (findnearslow): 1-based row_ptr, col_ind."""
    L = lib()
    cms, rad_near, targs = _f(cms), _f(rad_near), _f(targs)
    nt = targs.shape[0]
    row_ptr = np.zeros(nt + 1, np.int64)
    L.oracle_findnear(_p(cms), cms.shape[0], _p(rad_near), targs.shape[1], _p(targs), nt,
                      _p(row_ptr), None)
    col_ind = np.zeros(max(int(row_ptr[-1] - 1), 1), np.int64)
    L.oracle_findnear(_p(cms), cms.shape[0], _p(rad_near), targs.shape[1], _p(targs), nt,
                      _p(row_ptr), _p(col_ind))
    return row_ptr, col_ind[: int(row_ptr[-1] - 1)]


def iquad_rsc(s, row_ptr, col_ind):
    """get_iquad_rsc: iquad = 1 + cumulative basis sizes of the listed patches."""
    npols = np.diff(_f(s.ixyzs, np.int64))
    return np.concatenate([[1], 1 + np.cumsum(npols[col_ind - 1])]).astype(np.int64)


def hkrand(iseed: int) -> float:
    return float(lib().oracle_hkrand(iseed))


def far_order(eps, s, cms, rads, targs, ikerorder, zk, row_ptr, col_ind, rfac):
    L = lib()
    targs = _f(targs)
    nf = np.zeros(s.npatches, np.int64)
    ixo = np.zeros(s.npatches + 1, np.int64)
    z = np.array([complex(zk).real, complex(zk).imag])
    ier = L.oracle_get_far_order(eps, *_sargs(s)[:4], _p(_f(cms)), _p(_f(rads)), s.npts,
                                 _p(_f(s.srccoefs)), targs.shape[1], targs.shape[0], _p(targs),
                                 ikerorder, _p(z), col_ind.shape[0], _p(_f(row_ptr, np.int64)),
                                 _p(_f(col_ind, np.int64)), rfac, _p(nf), _p(ixo))
    if ier:
        raise RuntimeError(f"oracle_get_far_order failed ({ier})")
    return nf, ixo


def oversample_geom(s, novers, ixyzso):
    L = lib()
    nptso = int(ixyzso[-1] - 1)
    so = np.zeros((nptso, 12))
    ier = L.oracle_oversample_geom(*_sargs(s), _p(_f(s.srccoefs)), _p(_f(s.srcvals)),
                                   _p(_f(novers, np.int64)), _p(_f(ixyzso, np.int64)), nptso,
                                   _p(so))
    if ier:
        raise RuntimeError(f"oracle_oversample_geom failed ({ier})")
    return so


def patch_id_uvs(s):
    """Patch (1-based) and parameter coordinates of every node."""
    ip = np.zeros(s.npts, np.int64)
    uv = np.zeros((s.npts, 2))
    tab = read_vr_table()
    for p in range(s.npatches):
        a, b = int(s.ixyzs[p] - 1), int(s.ixyzs[p + 1] - 1)
        ip[a:b] = p + 1
        n = int(s.norders[p])
        if int(s.iptype[p]) == 1:
            uv[a:b] = tab[n][0].reshape(-1, 2)
        else:
            x = np.polynomial.legendre.leggauss(n + 1)[0]
            uv[a:b, 0] = np.tile(x, n + 1)
            uv[a:b, 1] = np.repeat(x, n + 1)
    return ip, uv


def getnearquad(s, kind, eps, params, targs, ipatch_id, uvs_targ, row_ptr, col_ind, iquad):
    """getnearquad_{lap,helm}_comb_dir_eval with the oracle's own rules;
    returns (wnear, kernel evaluations)."""
    L = lib()
    targs = _f(targs)
    nt = targs.shape[0]
    nquad = int(iquad[-1] - 1)
    ipid = None if ipatch_id is None else _f(ipatch_id, np.int64)
    uvt = None if uvs_targ is None else _f(uvs_targ)
    pr = _params(kind, params)
    w = np.zeros(max(nquad, 1), float if kind == 0 else complex)
    wv = w if kind == 0 else w.view(float)
    stats = np.zeros(1, np.int64)
    ier = L.oracle_getnearquad(kind, *_sargs(s), _p(_f(s.srccoefs)), _p(_f(s.srcvals)),
                               targs.shape[1], nt, _p(targs), _p(ipid), _p(uvt), eps, _p(pr),
                               col_ind.shape[0], _p(_f(row_ptr, np.int64)),
                               _p(_f(col_ind, np.int64)), _p(_f(iquad, np.int64)), nquad, _p(wv),
                               _p(stats))
    if ier:
        raise RuntimeError(f"oracle_getnearquad failed ({ier})")
    return w[:nquad], int(stats[0])


def setup(s, kind, eps, params, targs=None, ipatch_id=None, uvs_targ=None) -> OSetup:
    """The setup sequence of helm_comb_dir_solver / lap_comb_dir_eval
    (helm_comb_dir.f:1957-2051, lap_comb_dir.f90:526-601), every step by the
    oracle: rfacs, centroids, brute-force near list, iquad, far orders,
    oversampled geometry and weights, near quadrature."""
    if targs is None:
        targs = s.srcvals
        ipatch_id, uvs_targ = patch_id_uvs(s)
    targs = _f(targs)
    iptype_avg = int(math.floor(int(np.sum(s.iptype)) / s.npatches))
    norder_avg = int(math.floor(int(np.sum(s.norders)) / s.npatches))
    rfac, rfac0 = rfacs(norder_avg, iptype_avg)
    cms, rads = centroid_rads(s)
    row_ptr, col_ind = findnear(cms, rads * rfac, targs)
    iquad = iquad_rsc(s, row_ptr, col_ind)
    beta = params[1] if kind == 0 else params[2]
    ikerorder = 0 if abs(beta) > 1e-16 else -1
    zk = 0.0 if kind == 0 else params[0]
    novers, ixyzso = far_order(eps, s, cms, rads, targs, ikerorder, zk, row_ptr, col_ind, rfac)
    srcover = oversample_geom(s, novers, ixyzso)
    so = OSurface(novers, ixyzso, _f(s.iptype, np.int64), srcover, np.zeros((srcover.shape[0], 9)))
    wover = qwts(so)
    wnear, nev = getnearquad(s, kind, eps, params, targs, ipatch_id, uvs_targ, row_ptr, col_ind,
                             iquad)
    return OSetup(ONear(row_ptr, col_ind, iquad, wnear), OOver(novers, ixyzso, srcover, wover),
                  rfac, rfac0, cms, rads, nev)


class GmresSolver:
    """zgmres_guru / dgmres_guru (src/common/gmres_routs.f90:13-375) one
    Arnoldi step at a time, with the oracle's matvec: (zid I + K) x = rhs,
    unrestarted, modified Gram-Schmidt in the w-weighted inner product,
    Givens rotations (rotmat_gmres.f:15-100), stop when the recurrence
    residual |s_{m+1}|/||rhs|| <= eps_gmres; finish() back-substitutes and
    takes the true residual with one more matvec, as the reference does.
    The same algorithm as oracle_gmres in oracle.c, stepwise so that a
    caller can time its iterations."""

    def __init__(self, kind, surf, params, near, over, zid, rhs, numit=200, eps_gmres=1e-10,
                 wts=None):
        self.kind, self.surf, self.params, self.near, self.over = kind, surf, params, near, over
        self.zid = complex(zid)
        self.w = qwts(surf) if wts is None else wts
        self.rhs = np.asarray(rhs, complex)
        self.numit, self.eps = numit, eps_gmres
        self.rb = float(np.sqrt(np.sum(self.w * np.abs(self.rhs) ** 2)))
        self.V = [self.rhs / self.rb]
        self.H = np.zeros((numit + 1, numit), complex)
        self.cs = np.zeros(numit, complex)
        self.sn = np.zeros(numit, complex)
        self.s = np.zeros(numit + 1, complex)
        self.s[0] = self.rb
        self.it = 0
        self.errs = []
        self.done = False

    def _apply(self, x):
        y = lpcomp(self.kind, self.surf, self.params, self.near, self.over,
                   x.real if self.kind == 0 else x)
        return np.asarray(y, complex)

    def step(self) -> bool:
        """One Arnoldi iteration; True once the residual test is met (or
        numit is reached)."""
        it = self.it
        wv = self._apply(self.V[it])
        for k in range(it + 1):
            z = np.sum(wv * np.conj(self.V[k]) * self.w)
            self.H[k, it] = z
            wv = wv - z * self.V[k]
        self.H[it, it] += self.zid
        wn = float(np.sqrt(np.sum(self.w * np.abs(wv) ** 2)))
        self.V.append(wv / wn)
        for k in range(it):
            t = self.cs[k] * self.H[k, it] + np.conj(self.sn[k]) * self.H[k + 1, it]
            self.H[k + 1, it] = -self.sn[k] * self.H[k, it] + self.cs[k] * self.H[k + 1, it]
            self.H[k, it] = t
        a, b = self.H[it, it], wn
        if a == 0:
            c, sgiv = 0.0, 1.0
        else:
            t = b / a
            c = 1.0 / np.sqrt(1.0 + abs(t) ** 2)
            sgiv = t * c
        self.cs[it], self.sn[it] = c, sgiv
        self.H[it, it] = c * self.H[it, it] + np.conj(sgiv) * wn
        self.s[it + 1] = -sgiv * self.s[it]
        self.s[it] = c * self.s[it]
        err = abs(self.s[it + 1]) / self.rb
        self.errs.append(err)
        self.it += 1
        self.done = err <= self.eps or self.it == self.numit
        return self.done

    def finish(self):
        """Back-substitution, solution and true relative residual (one
        matvec).  Returns (soln, niter, errs, rres)."""
        m = self.it
        y = np.zeros(m, complex)
        for j in range(m - 1, -1, -1):
            y[j] = (self.s[j] - np.dot(self.H[j, j + 1:m], y[j + 1:m])) / self.H[j, j]
        x = sum(y[i] * self.V[i] for i in range(m))
        r = self.zid * x + self._apply(x) - self.rhs
        rres = float(np.sqrt(np.sum(self.w * np.abs(r) ** 2)) / self.rb)
        soln = x.real if self.kind == 0 else x
        return soln, m, np.array(self.errs), rres
