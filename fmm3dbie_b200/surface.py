"""Surfaces and setup for the layer-potential path, in the reference's layout.

A ``Surface`` holds the reference's discretisation arrays: ``norders``,
``ixyzs`` (1-based), ``iptype``, ``srcvals`` (npts x 12 in memory, i.e. the
Fortran ``srcvals(12,npts)``) and ``srccoefs`` (npts x 9).  The setup
functions follow the sequence of ``helm_comb_dir_solver``
(src/helm_wrappers/helm_comb_dir.f:1957-2051) and ``lap_comb_dir_eval``
(src/lap_wrappers/lap_comb_dir.f90:526-601).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


def _init():
    lib = L.lib()
    L.check(lib.bie_init(None), "bie_init")
    return lib


@dataclass
class Surface:
    norders: np.ndarray
    ixyzs: np.ndarray
    iptype: np.ndarray
    srcvals: np.ndarray
    srccoefs: np.ndarray

    @property
    def npatches(self) -> int:
        return int(self.norders.shape[0])

    @property
    def npts(self) -> int:
        return int(self.srcvals.shape[0])

    def args(self):
        """(npatches, norders, ixyzs, iptype, npts, srccoefs, srcvals) pointers."""
        return (self.npatches, L.ptr(self.norders), L.ptr(self.ixyzs), L.ptr(self.iptype),
                self.npts, L.ptr(self.srccoefs), L.ptr(self.srcvals))

    def qwts(self) -> np.ndarray:
        lib = _init()
        w = np.zeros(self.npts)
        L.check(lib.bie_get_qwts(self.npatches, L.ptr(self.norders), L.ptr(self.ixyzs),
                                 L.ptr(self.iptype), self.npts, L.ptr(self.srcvals), L.ptr(w)),
                "get_qwts")
        return w

    def patch_id_uvs(self):
        lib = _init()
        ip = np.zeros(self.npts, dtype=np.int64)
        uv = np.zeros((self.npts, 2))
        L.check(lib.bie_get_patch_id_uvs(self.npatches, L.ptr(self.norders), L.ptr(self.ixyzs),
                                         L.ptr(self.iptype), self.npts, L.ptr(ip), L.ptr(uv)),
                "get_patch_id_uvs")
        return ip, uv

    @property
    def xyz(self):
        return self.srcvals[:, 0:3]

    @property
    def normals(self):
        return self.srcvals[:, 9:12]


def disc_exps(iptype: int, norder: int):
    """(uvs, umat, vmat, wts) of a patch type/order (get_disc_exps); umat maps
    nodal values to basis coefficients (coefs = umat @ vals)."""
    lib = _init()
    npols = (norder + 1) * (norder + 2) // 2 if iptype == 1 else (norder + 1) ** 2
    uvs = np.zeros((npols, 2))
    um = np.zeros((npols, npols), order="F")
    vm = np.zeros((npols, npols), order="F")
    w = np.zeros(npols)
    L.check(lib.bie_get_disc_exps(norder, npols, iptype, L.ptr(uvs), um.ctypes.data_as(L.PDBL),
                                  vm.ctypes.data_as(L.PDBL), L.ptr(w)), "get_disc_exps")
    return uvs, np.ascontiguousarray(um), np.ascontiguousarray(vm), w


def from_srcvals(norders, iptype, srcvals) -> "Surface":
    """Surface from nodal values only: srccoefs = umat * srcvals(1:9) per
    patch (as getgeominfo / open_gov3_geometry do)."""
    norders = np.ascontiguousarray(norders, np.int64)
    iptype = np.ascontiguousarray(iptype, np.int64)
    srcvals = np.ascontiguousarray(srcvals, float)
    npols = np.array([(n + 1) * (n + 2) // 2 if t == 1 else (n + 1) ** 2
                      for n, t in zip(norders, iptype)], np.int64)
    ixyzs = np.concatenate([[1], 1 + np.cumsum(npols)]).astype(np.int64)
    srccoefs = np.zeros((srcvals.shape[0], 9))
    for key in set(zip(iptype.tolist(), norders.tolist())):
        _, um, _, _ = disc_exps(*key)
        sel = np.nonzero((iptype == key[0]) & (norders == key[1]))[0]
        np_ = um.shape[0]
        idx = (ixyzs[sel] - 1)[:, None] + np.arange(np_)[None, :]
        vals = srcvals[idx, :9]                     # (npatch, npols, 9)
        srccoefs[idx] = np.einsum("lj,pjk->plk", um, vals)
    return Surface(norders, ixyzs, iptype, srcvals, srccoefs)


def read_go3(path) -> "Surface":
    """.go3 triangle mesh (open_gov3_geometry, src/surface_routs/in_go3.f90:1):
    order, number of patches, then x, y, z, dx/du, dy/du, dz/du, dx/dv, dy/dv,
    dz/dv, nx, ny, nz, each as npts consecutive values; RV nodes."""
    with open(path) as f:
        norder = int(f.readline().split()[0])
        npatches = int(f.readline().split()[0])
        vals = np.array(f.read().split(), dtype=float)
    npols = (norder + 1) * (norder + 2) // 2
    npts = npatches * npols
    if vals.size < 12 * npts:
        raise ValueError(f"{path}: expected {12 * npts} values, found {vals.size}")
    srcvals = np.ascontiguousarray(vals[: 12 * npts].reshape(12, npts).T)
    return from_srcvals(np.full(npatches, norder, np.int64), np.ones(npatches, np.int64), srcvals)


def write_go3(surf: "Surface", path) -> None:
    """Write a single-order triangle surface in .go3 layout."""
    if len(set(surf.norders.tolist())) != 1 or np.any(surf.iptype != 1):
        raise ValueError(".go3 holds triangles of one order")
    with open(path, "w") as f:
        f.write(f"{int(surf.norders[0])}\n{surf.npatches}\n")
        np.savetxt(f, surf.srcvals.T.reshape(-1), fmt="%.17g")


def icosa_ellipsoid(nref: int, norder: int, axes=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0)):
    """Icosahedron refined nref times, projected radially onto the ellipsoid
    center + axes * x/|x|, order-norder Vioreanu-Rokhlin nodes."""
    lib = _init()
    npat = int(lib.bie_icosa_npatches(nref))
    npols = (norder + 1) * (norder + 2) // 2
    npts = npat * npols
    no = np.zeros(npat, np.int64)
    ix = np.zeros(npat + 1, np.int64)
    ip = np.zeros(npat, np.int64)
    sv = np.zeros((npts, 12))
    sc = np.zeros((npts, 9))
    ax = np.asarray(axes, float)
    ce = np.asarray(center, float)
    L.check(lib.bie_surf_icosa_ellipsoid(nref, norder, L.ptr(ax), L.ptr(ce), L.ptr(no), L.ptr(ix),
                                         L.ptr(ip), L.ptr(sv), L.ptr(sc)), "surf_icosa_ellipsoid")
    return Surface(no, ix, ip, sv, sc)


def icosa_sphere(nref: int, norder: int):
    return icosa_ellipsoid(nref, norder)


def torus_quad(nu: int, nv: int, norder: int, R=2.0, r0=0.6, r1=0.15, m=3):
    """Torus with minor radius r0 + r1 cos(m p), nu x nv quad patches, tensor
    Gauss-Legendre nodes (iptype 11)."""
    lib = _init()
    npat = nu * nv
    npols = (norder + 1) ** 2
    npts = npat * npols
    no = np.zeros(npat, np.int64)
    ix = np.zeros(npat + 1, np.int64)
    ip = np.zeros(npat, np.int64)
    sv = np.zeros((npts, 12))
    sc = np.zeros((npts, 9))
    L.check(lib.bie_surf_torus_quad(nu, nv, norder, R, r0, r1, m, L.ptr(no), L.ptr(ix), L.ptr(ip),
                                    L.ptr(sv), L.ptr(sc)), "surf_torus_quad")
    return Surface(no, ix, ip, sv, sc)


# ---- setup pieces (names follow the reference routines) ---------------------
def get_rfacs(norder: int, iptype: int):
    lib = _init()
    a, b = L.DBL(), L.DBL()
    lib.bie_get_rfacs(norder, iptype, L.C.byref(a), L.C.byref(b))
    return a.value, b.value


def get_centroid_rads(s: Surface):
    lib = _init()
    cms = np.zeros((s.npatches, 3))
    rads = np.zeros(s.npatches)
    L.check(lib.bie_get_centroid_rads(s.npatches, L.ptr(s.norders), L.ptr(s.ixyzs),
                                      L.ptr(s.iptype), s.npts, L.ptr(s.srccoefs), L.ptr(cms),
                                      L.ptr(rads)), "get_centroid_rads")
    return cms, rads


def findnear(cms, rad_near, targs, engine: str = "cpu"):
    """Row-sparse near list (1-based row_ptr, col_ind); engine "gpu" builds it
    on the device (the same lists), "auto" there when a device is visible."""
    lib = _init()
    cms = np.ascontiguousarray(cms, float)
    rad_near = np.ascontiguousarray(rad_near, float)
    targs = np.ascontiguousarray(targs, float)
    ndt = targs.shape[1]
    nt = targs.shape[0]
    if _engine(engine) == "gpu":
        row_ptr = np.zeros(nt + 1, np.int64)
        cap = 32 * nt + 64
        while True:
            col_ind = np.zeros(cap, np.int64)
            st = lib.bie_findnear_gpu(L.ptr(cms), cms.shape[0], L.ptr(rad_near), ndt, L.ptr(targs),
                                      nt, L.ptr(row_ptr), L.ptr(col_ind), cap)
            nnz = int(row_ptr[-1] - 1)
            if st == 0 or nnz <= cap:
                L.check(st, "findnear_gpu")
                return row_ptr, col_ind[:nnz]
            cap = nnz
    nnz = L.I64()
    L.check(lib.bie_findnearmem(L.ptr(cms), cms.shape[0], L.ptr(rad_near), ndt, L.ptr(targs), nt,
                                L.C.byref(nnz)), "findnearmem")
    row_ptr = np.zeros(nt + 1, np.int64)
    col_ind = np.zeros(max(nnz.value, 1), np.int64)
    L.check(lib.bie_findnear(L.ptr(cms), cms.shape[0], L.ptr(rad_near), ndt, L.ptr(targs), nt,
                             L.ptr(row_ptr), L.ptr(col_ind)), "findnear")
    return row_ptr, col_ind[:nnz.value]


def get_iquad_rsc(s: Surface, row_ptr, col_ind):
    lib = _init()
    nnz = col_ind.shape[0]
    iquad = np.zeros(nnz + 1, np.int64)
    L.check(lib.bie_get_iquad_rsc(s.npatches, L.ptr(s.ixyzs), row_ptr.shape[0] - 1, nnz,
                                  L.ptr(row_ptr), L.ptr(col_ind), L.ptr(iquad)), "get_iquad_rsc")
    return iquad


def get_far_order(eps, s: Surface, cms, rads, targs, ikerorder, zk, row_ptr, col_ind, rfac,
                  engine: str = "cpu"):
    """Far-field oversampling order per patch and ixyzso; engine as findnear."""
    lib = _init()
    targs = np.ascontiguousarray(targs, float)
    nf = np.zeros(s.npatches, np.int64)
    ixo = np.zeros(s.npatches + 1, np.int64)
    z = np.array([complex(zk).real, complex(zk).imag])
    fn = lib.bie_get_far_order_gpu if _engine(engine) == "gpu" else lib.bie_get_far_order
    L.check(fn(eps, s.npatches, L.ptr(s.norders), L.ptr(s.ixyzs),
                                  L.ptr(s.iptype), L.ptr(cms), L.ptr(rads), s.npts,
                                  L.ptr(s.srccoefs), targs.shape[1], targs.shape[0], L.ptr(targs),
                                  ikerorder, L.ptr(z), col_ind.shape[0], L.ptr(row_ptr),
                                  L.ptr(col_ind), rfac, L.ptr(nf), L.ptr(ixo)), "get_far_order")
    return nf, ixo


def oversample_geom(s: Surface, novers, ixyzso, engine: str = "cpu"):
    """Oversampled geometry srcover (nptso x 12); engine as findnear."""
    lib = _init()
    nptso = int(ixyzso[-1] - 1)
    so = np.zeros((nptso, 12))
    fn = lib.bie_oversample_geom_gpu if _engine(engine) == "gpu" else lib.bie_oversample_geom
    L.check(fn(s.npatches, L.ptr(s.norders), L.ptr(s.ixyzs), L.ptr(s.iptype),
                                    s.npts, L.ptr(s.srccoefs), L.ptr(s.srcvals), L.ptr(novers),
                                    L.ptr(ixyzso), nptso, L.ptr(so)), "oversample_geom")
    return so


def oversample_fun_surf(s: Surface, u, novers, ixyzso):
    """Oversample nd real functions u (npts x nd) to (nptso x nd)."""
    lib = _init()
    u = np.ascontiguousarray(u, float)
    nd = 1 if u.ndim == 1 else u.shape[1]
    nptso = int(ixyzso[-1] - 1)
    uo = np.zeros((nptso, nd)) if u.ndim > 1 else np.zeros(nptso)
    L.check(lib.bie_oversample_fun_surf(nd, s.npatches, L.ptr(s.norders), L.ptr(s.ixyzs),
                                        L.ptr(s.iptype), s.npts, L.ptr(u), L.ptr(novers),
                                        L.ptr(ixyzso), nptso, L.ptr(uo)), "oversample_fun_surf")
    return uo


def get_fmm_thresh(src, trg):
    lib = _init()
    src = np.ascontiguousarray(src, float)
    trg = np.ascontiguousarray(trg, float)
    t = L.DBL()
    lib.bie_get_fmm_thresh(src.shape[1], src.shape[0], L.ptr(src), trg.shape[1], trg.shape[0],
                           L.ptr(trg), L.C.byref(t))
    return t.value


def hkrand(iseed: int) -> float:
    return float(_init().bie_hkrand(iseed))


@dataclass
class NearField:
    """Row-sparse near interactions and their quadrature (getnearquad_*)."""
    row_ptr: np.ndarray
    col_ind: np.ndarray
    iquad: np.ndarray
    wnear: np.ndarray  # float64 (Laplace) or complex128 (Helmholtz)

    @property
    def nnz(self):
        return int(self.col_ind.shape[0])

    @property
    def nquad(self):
        return int(self.iquad[-1] - 1)


@dataclass
class Oversampled:
    novers: np.ndarray
    ixyzso: np.ndarray
    srcover: np.ndarray
    wover: np.ndarray

    @property
    def nptso(self):
        return int(self.srcover.shape[0])


@dataclass
class Setup:
    near: NearField
    over: Oversampled
    rfac: float
    rfac0: float
    cms: np.ndarray = field(repr=False)
    rads: np.ndarray = field(repr=False)


def _engine(engine: str) -> str:
    if engine not in ("auto", "cpu", "gpu"):
        raise ValueError(f"engine must be 'auto', 'cpu' or 'gpu', not {engine!r}")
    if engine == "auto":
        import torch
        return "gpu" if torch.cuda.is_available() else "cpu"
    return engine


def getnearquad(s: Surface, kind: int, eps: float, params, targs, ipatch_id, uvs_targ,
                row_ptr, col_ind, iquad, rfac0, engine: str = "auto", stats=None):
    """getnearquad_{lap,helm}_comb_dir_eval; params = (alpha, beta) for
    Laplace, (k, alpha, beta) for Helmholtz.  engine "cpu" runs the host
    generator, "gpu" the device one (same rules and tolerance), "auto" the
    device one when a CUDA device is visible.  stats (engine "gpu"): an int64
    array of 4 that receives kernel evaluations, self pairs, near pairs and
    the device time of the pair kernel in microseconds."""
    engine = _engine(engine)
    if engine == "gpu":
        return _getnearquad_gpu(s, kind, eps, params, targs, ipatch_id, uvs_targ, row_ptr,
                                col_ind, iquad, rfac0, stats)
    lib = _init()
    targs = np.ascontiguousarray(targs, float)
    nt = targs.shape[0]
    nquad = int(iquad[-1] - 1)
    ipatch_id = np.ascontiguousarray(ipatch_id, np.int64)
    uvs_targ = np.ascontiguousarray(uvs_targ, float)
    args = (s.npatches, L.ptr(s.norders), L.ptr(s.ixyzs), L.ptr(s.iptype), s.npts,
            L.ptr(s.srccoefs), L.ptr(s.srcvals), targs.shape[1], nt, L.ptr(targs),
            L.ptr(ipatch_id), L.ptr(uvs_targ), eps)
    if kind == 0:
        dp = np.asarray(params, float)
        w = np.zeros(max(nquad, 1))
        L.check(lib.bie_getnearquad_lap_comb_dir_eval(*args, L.ptr(dp), 1, col_ind.shape[0],
                                                       L.ptr(row_ptr), L.ptr(col_ind),
                                                       L.ptr(iquad), rfac0, nquad, L.ptr(w)),
                "getnearquad_lap_comb_dir_eval")
        return w[:nquad]
    zp = np.ascontiguousarray(np.asarray(params, complex)).view(float)
    w = np.zeros(max(nquad, 1), complex)
    L.check(lib.bie_getnearquad_helm_comb_dir_eval(*args, L.ptr(zp), 1, col_ind.shape[0],
                                                    L.ptr(row_ptr), L.ptr(col_ind), L.ptr(iquad),
                                                    rfac0, nquad, w.view(float).ctypes.data_as(L.PDBL)),
            "getnearquad_helm_comb_dir_eval")
    return w[:nquad]


def _getnearquad_gpu(s, kind, eps, params, targs, ipatch_id, uvs_targ, row_ptr, col_ind, iquad,
                     rfac0, stats):
    lib = _init()
    targs = np.ascontiguousarray(targs, float)
    nt = targs.shape[0]
    nquad = int(iquad[-1] - 1)
    ipatch_id = np.ascontiguousarray(ipatch_id, np.int64)
    uvs_targ = np.ascontiguousarray(uvs_targ, float)
    st = np.zeros(4, np.int64)
    args = (s.npatches, L.ptr(s.norders), L.ptr(s.ixyzs), L.ptr(s.iptype), s.npts,
            L.ptr(s.srccoefs), L.ptr(s.srcvals), targs.shape[1], nt, L.ptr(targs),
            L.ptr(ipatch_id), L.ptr(uvs_targ), eps)
    tail = (1, col_ind.shape[0], L.ptr(row_ptr), L.ptr(col_ind), L.ptr(iquad), rfac0, nquad)
    if kind == 0:
        dp = np.asarray(params, float)
        w = np.zeros(max(nquad, 1))
        L.check(lib.bie_getnearquad_lap_comb_dir_eval_gpu(*args, L.ptr(dp), *tail, L.ptr(w),
                                                           L.ptr(st)),
                "getnearquad_lap_comb_dir_eval_gpu")
    else:
        zp = np.ascontiguousarray(np.asarray(params, complex)).view(float)
        w = np.zeros(max(nquad, 1), complex)
        L.check(lib.bie_getnearquad_helm_comb_dir_eval_gpu(*args, L.ptr(zp), *tail,
                                                            w.view(float).ctypes.data_as(L.PDBL),
                                                            L.ptr(st)),
                "getnearquad_helm_comb_dir_eval_gpu")
    if stats is not None:
        stats[:len(stats)] = st[:len(stats)]
    return w[:nquad]


def setup(s: Surface, kind: int, eps: float, params, targs=None, ipatch_id=None, uvs_targ=None,
          engine: str = "auto", stats=None):
    """The setup of lap_comb_dir_eval / helm_comb_dir_solver: near list, far
    order, oversampled geometry and near quadrature.  targs defaults to the
    surface nodes (on-surface, with self interactions).  engine: where the
    steps run ("gpu": near list, far orders, oversampled geometry and near
    quadrature on the device; "cpu": on the host; "auto": the device when one
    is visible); stats: the near quadrature generator's counters (see
    getnearquad)."""
    if targs is None:
        targs = s.srcvals
        ipatch_id, uvs_targ = s.patch_id_uvs()
    targs = np.ascontiguousarray(targs, float)
    nt = targs.shape[0]
    if ipatch_id is None:
        ipatch_id = -np.ones(nt, np.int64)
        uvs_targ = np.zeros((nt, 2))
    iptype_avg = int(math.floor(s.iptype.sum() / s.npatches))
    norder_avg = int(math.floor(s.norders.sum() / s.npatches))
    rfac, rfac0 = get_rfacs(norder_avg, iptype_avg)
    cms, rads = get_centroid_rads(s)
    engine = _engine(engine)
    row_ptr, col_ind = findnear(cms, rads * rfac, targs, engine=engine)
    iquad = get_iquad_rsc(s, row_ptr, col_ind)
    beta = params[1] if kind == 0 else params[2]
    ikerorder = 0 if abs(beta) > 1e-16 else -1
    zk = 0.0 if kind == 0 else params[0]
    novers, ixyzso = get_far_order(eps, s, cms, rads, targs, ikerorder, zk, row_ptr, col_ind, rfac,
                                   engine=engine)
    srcover = oversample_geom(s, novers, ixyzso, engine=engine)
    so = Surface(novers, ixyzso, s.iptype, srcover, np.zeros((srcover.shape[0], 9)))
    wover = so.qwts()
    wnear = getnearquad(s, kind, eps, params, targs, ipatch_id, uvs_targ, row_ptr, col_ind, iquad,
                        rfac0, engine=engine, stats=stats)
    return Setup(NearField(row_ptr, col_ind, iquad, wnear), Oversampled(novers, ixyzso, srcover, wover),
                 rfac, rfac0, cms, rads)
