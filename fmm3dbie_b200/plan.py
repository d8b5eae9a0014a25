"""Device-resident operator plans (torch tensors as device buffers).

``Plan`` wraps ``bie_plan_*``: geometry, near quadrature (folded into
W_eff) and oversampling are uploaded once; ``matvec`` and ``solve`` then work
on CUDA tensors on the caller's current torch stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .surface import NearField, Oversampled, Surface


def _stream_ptr(torch, device):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _dptr(t):
    return C.c_void_p(t.data_ptr())


class Plan:
    """Operator K of lpcomp_{lap,helm}_comb_dir_addsub on the current CUDA device.

    kind 0 (Laplace): params = (alpha, beta); kind 1 (Helmholtz): params =
    (k, alpha, beta).  targs=None: targets are the surface nodes (lpcomp and
    solver case); otherwise targs is (ntarg, ndtarg) on the host.
    """

    def __init__(self, kind: int, params, surf: Surface, near: NearField, over: Oversampled,
                 targs=None):
        import torch
        self.torch = torch
        if not torch.cuda.is_available():
            raise RuntimeError("fmm3dbie_b200.Plan needs a CUDA device")
        self.kind = kind
        self.cplx = kind == 1
        self.device = torch.device("cuda", torch.cuda.current_device())
        lib = L.lib()
        L.check(lib.bie_init(None), "bie_init")
        if kind == 0:
            pr = np.asarray(params, float)
        else:
            pr = np.ascontiguousarray(np.asarray(params, complex)).view(float)
        if targs is None:
            ndt, nt, tp = 12, 0, None
        else:
            targs = np.ascontiguousarray(targs, float)
            ndt, nt, tp = targs.shape[1], targs.shape[0], L.ptr(targs)
        w = np.ascontiguousarray(near.wnear, float if kind == 0 else complex)
        wv = w if kind == 0 else w.view(float)
        h = C.c_void_p()
        L.check(lib.bie_plan_create(kind, L.ptr(pr), *surf.args(), ndt, nt, tp, near.nnz,
                                    L.ptr(near.row_ptr), L.ptr(near.col_ind), L.ptr(near.iquad),
                                    near.nquad, L.ptr(wv), L.ptr(over.novers), over.nptso,
                                    L.ptr(over.ixyzso), L.ptr(over.srcover), L.ptr(over.wover),
                                    C.byref(h)), "bie_plan_create")
        self._h = h
        info = self.info()
        self.npts, self.ntarg, self.nptso, self.nnz, self.nquad = (int(x) for x in info[:5])
        self.nchunks = (int(info[5]), int(info[6]))

    def info(self):
        """npts, ntarg, nptso, nnz, nquad, far chunks (f64, f32), kind, far
        variant (f64, f32)."""
        info = np.zeros(10, np.int64)
        L.lib().bie_plan_info(self._h, L.ptr(info))
        return info

    def set_far(self, iprec: int, nd: int, variant: int, nchunks: int):
        """Pin the far-field shape of (iprec, nd) (variants 0-2 CUDA cores,
        3-4 tensor cores for FP32 Helmholtz with nd >= 4)."""
        L.check(L.lib().bie_plan_set_far(self._h, iprec, nd, variant, nchunks), "bie_plan_set_far")

    def get_far(self, iprec: int, nd: int):
        """(variant, nchunks, tensor-core timeout flag) of (iprec, nd)."""
        out = np.zeros(3, np.int64)
        L.check(L.lib().bie_plan_get_far(self._h, iprec, nd, L.ptr(out)), "bie_plan_get_far")
        return tuple(int(v) for v in out)

    def set_far_method(self, iprec: int, method: int, theta: float = 0.0, p: int = 0,
                       leaf_t: int = 0, leaf_s: int = 0):
        """Far field of precision iprec: 0 direct sum, 1 hierarchical
        (dual-tree barycentric Lagrange interpolation; theta, p, leaf_t,
        leaf_s: opening angle, grid points per side, targets / sources per
        leaf; 0 = defaults)."""
        L.check(L.lib().bie_plan_set_far_method(self._h, iprec, method, float(theta), int(p),
                                                int(leaf_t), int(leaf_s), None),
                "bie_plan_set_far_method")

    def get_far_method(self, iprec: int) -> dict:
        """Method and tree statistics of precision iprec."""
        out = np.zeros(16)
        L.check(L.lib().bie_plan_get_far_method(self._h, iprec, L.ptr(out)),
                "bie_plan_get_far_method")
        keys = ["method", "p", "theta", "target_nodes", "source_nodes", "leaves", "pp_check",
                "pp", "pc", "cp", "cc", "source_proxies", "target_proxies", "kernel_evals",
                "build_ms", "updown_terms"]
        return {k: float(v) for k, v in zip(keys, out)}

    def close(self):
        if getattr(self, "_h", None):
            L.lib().bie_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def dtype(self):
        return self.torch.complex128 if self.cplx else self.torch.float64

    def _check(self, t, n, nd):
        if t.device != self.device or t.dtype != self.dtype or not t.is_contiguous():
            raise ValueError(f"expected a contiguous {self.dtype} tensor on {self.device}")
        if t.numel() != n * nd:
            raise ValueError(f"expected {n}*{nd} values, got {t.numel()}")

    def matvec(self, sigma, iprec: int = 0, out=None):
        """pot = K sigma for sigma of shape (npts,) or (npts, nd)."""
        torch = self.torch
        nd = 1 if sigma.dim() == 1 else sigma.shape[1]
        self._check(sigma, self.npts, nd)
        if out is None:
            shape = (self.ntarg,) if sigma.dim() == 1 else (self.ntarg, nd)
            out = torch.empty(shape, dtype=self.dtype, device=self.device)
        self._check(out, self.ntarg, nd)
        L.check(L.lib().bie_plan_matvec(self._h, iprec, nd, _dptr(sigma), _dptr(out),
                                        _stream_ptr(torch, self.device)), "bie_plan_matvec")
        return out

    def solve(self, rhs, zid, mode: int = 0, numit: int = 200, eps_gmres: float = 1e-6, x0=None,
              out=None):
        """Solve (zid I + K) x = rhs; rhs (npts,) or (npts, nd) independent systems.

        mode 0: FP64 GMRES (the reference method); 1: FP32-matvec GMRES inside
        FP64 iterative refinement.  x0: initial guess; the stopping test stays
        relative to ||rhs||, and in mode 1 a guess whose residual is not
        below ||rhs|| is replaced by zero (info["x0_dropped"]).  Returns (x,
        info dict)."""
        torch = self.torch
        nd = 1 if rhs.dim() == 1 else rhs.shape[1]
        self._check(rhs, self.npts, nd)
        if out is None:
            out = torch.empty_like(rhs)
        if x0 is not None:
            self._check(x0, self.npts, nd)
        z = np.array([complex(zid).real, complex(zid).imag])
        niter = np.zeros(nd, np.int64)
        rres = np.zeros(nd)
        errs = np.zeros((numit + 1) * nd)
        st = L.lib().bie_plan_solve(self._h, mode, nd, L.ptr(z), _dptr(rhs),
                                    _dptr(x0) if x0 is not None else None, numit, eps_gmres,
                                    _dptr(out), L.ptr(niter), L.ptr(errs), L.ptr(rres),
                                    _stream_ptr(torch, self.device))
        if st not in (0, 3, 4):
            L.check(st, "bie_plan_solve")
        info = {"status": int(st), "niter": niter, "rres": rres}
        if mode == 0:
            info["errs"] = errs.reshape(nd, numit + 1)
        else:
            info["fp64_matvecs"] = int(errs[0])
            info["fp32_matvecs"] = int(errs[1])
            ms = np.zeros(4)
            L.lib().bie_last_mixed_stats(L.ptr(ms))
            info["increment_matvecs"] = int(ms[2])
            info["max_increment_ratio"] = float(ms[3])
            if x0 is not None:
                info["x0_dropped"] = errs[2:2 + nd].astype(bool)
        return out, info

    @staticmethod
    def set_mixed_residual(mode: str) -> None:
        """Refinement residual of the mixed solvers, process wide: "increment"
        (default: FP32 operator on small corrections, FP64 on the first
        step) or "full" (FP64 operator on x after every inner solve)."""
        L.check(L.lib().bie_set_mixed_residual({"full": 0, "increment": 1}[mode]),
                "bie_set_mixed_residual")

    def timing(self, enable: bool | None = None):
        t = np.zeros(8)
        L.lib().bie_plan_timing(self._h, -1 if enable is None else int(enable), L.ptr(t))
        out = {}
        for p, tag in ((0, "f64"), (1, "f32")):
            out[tag] = {"strengths_ms": t[4 * p], "far_ms": t[4 * p + 1],
                        "combine_ms": t[4 * p + 2], "calls": int(t[4 * p + 3])}
        return out
