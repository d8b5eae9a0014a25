"""Batches of independent surfaces (uneven sizes, orders and wavenumbers).

``SurfaceBatch`` solves many surfaces together.  With ``engine="graph"``
(default) the surfaces form one device operator (``bie_batch_*``): every
matvec stage -- strengths or oversampling, far field, near correction -- is
one persistent launch walking a work list that spans all surfaces, the three
launches are captured once in a CUDA graph, and GMRES runs all (surface,
density) systems in the same launches.  With ``engine="streams"`` each surface
keeps its own plan and solves on its own CUDA stream from its own host thread
(the ctypes calls release the GIL).  Each surface may carry several
right-hand sides.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .plan import Plan
from .surface import Surface, setup


@dataclass
class BatchItem:
    surf: Surface
    kind: int          # 0 Laplace, 1 Helmholtz
    params: tuple      # (alpha, beta) or (k, alpha, beta)
    zid: complex       # identity term of the second-kind equation


class SurfaceBatch:
    def __init__(self, items, eps: float, engine: str = "graph", setups=None):
        import torch
        if engine not in ("graph", "streams"):
            raise ValueError("engine must be 'graph' or 'streams'")
        self.torch = torch
        self.engine = engine
        self.items = list(items)
        if engine == "graph" and len({it.kind for it in self.items}) != 1:
            raise ValueError("a graph batch needs one kernel kind for all surfaces")
        self.setups = (list(setups) if setups is not None else
                       [setup(it.surf, it.kind, eps, it.params) for it in self.items])
        self.plans = [Plan(it.kind, it.params, it.surf, st.near, st.over)
                      for it, st in zip(self.items, self.setups)]
        dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.npts = [it.surf.npts for it in self.items]
        self.offsets = np.concatenate([[0], np.cumsum(self.npts)]).astype(np.int64)
        self._b = None
        if engine == "graph":
            lib = L.lib()
            h = C.c_void_p()
            L.check(lib.bie_batch_create(C.byref(h)), "bie_batch_create")
            self._b = h
            for p in self.plans:
                L.check(lib.bie_batch_add(h, p._h), "bie_batch_add")
                p._h = None  # the batch owns it now
            L.check(lib.bie_batch_finalize(h, self._stream()), "bie_batch_finalize")
            self.plans = []
        else:
            self.streams = [torch.cuda.Stream(dev) for _ in self.items]

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def close(self):
        if self._b is not None:
            L.lib().bie_batch_destroy(self._b)
            self._b = None
        for p in self.plans:
            p.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        """surfaces, nodes, kind, reduction chunks, far variant and chunk
        length kept for (f32, nd = 1)."""
        out = np.zeros(6, np.int64)
        L.check(L.lib().bie_batch_info(self._b, L.ptr(out)), "bie_batch_info")
        return out

    def set_graph(self, enable: bool):
        L.check(L.lib().bie_batch_set_graph(self._b, int(enable)), "bie_batch_set_graph")

    def concat(self, parts):
        """Per-surface (npts_q, nd) tensors -> one (nodes, nd) batch vector."""
        return self.torch.cat([p.reshape(p.shape[0], -1) for p in parts], 0).contiguous()

    def split(self, x):
        return [x[self.offsets[q]:self.offsets[q + 1]] for q in range(len(self.items))]

    def matvec(self, x, iprec: int = 0, out=None):
        """K x for the batch vector x (nodes, nd) (graph engine)."""
        if self._b is None:
            raise RuntimeError("matvec is available with engine='graph'")
        nd = 1 if x.dim() == 1 else x.shape[1]
        if out is None:
            out = self.torch.empty_like(x)
        L.check(L.lib().bie_batch_matvec(self._b, iprec, nd, C.c_void_p(x.data_ptr()),
                                         C.c_void_p(out.data_ptr()), self._stream()),
                "bie_batch_matvec")
        return out

    def solve(self, rhs, mode: int = 1, numit: int = 200, eps_gmres: float = 1e-7,
              concurrent: bool = True, x0=None):
        """rhs[q]: (npts_q, nrhs) device tensors.  Returns (solutions, infos,
        device milliseconds from the first launch to the last completion)."""
        if self.engine == "graph":
            return self._solve_graph(rhs, mode, numit, eps_gmres, x0)
        return self._solve_streams(rhs, mode, numit, eps_gmres, concurrent)

    def _solve_graph(self, rhs, mode, numit, eps_gmres, x0):
        torch = self.torch
        nd = {r.shape[1] if r.dim() == 2 else 1 for r in rhs}
        if len(nd) != 1:
            raise ValueError("a graph batch needs the same number of right-hand sides per surface")
        nd = nd.pop()
        b = self.concat(rhs)
        xb = torch.empty_like(b)
        x0b = self.concat(x0) if x0 is not None else None
        ns = len(self.items)
        z = np.zeros(2 * ns)
        for q, it in enumerate(self.items):
            z[2 * q], z[2 * q + 1] = complex(it.zid).real, complex(it.zid).imag
        niter = np.zeros(ns * nd, np.int64)
        rres = np.zeros(ns * nd)
        stats = np.zeros(2)
        main = torch.cuda.current_stream(self.device)
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(main)
        st = L.lib().bie_batch_solve(self._b, mode, nd, L.ptr(z), C.c_void_p(b.data_ptr()),
                                     C.c_void_p(x0b.data_ptr()) if x0b is not None else None,
                                     numit, eps_gmres, C.c_void_p(xb.data_ptr()), L.ptr(niter),
                                     L.ptr(rres), L.ptr(stats), self._stream())
        stop.record(main)
        stop.synchronize()
        if st not in (0, 3, 4):
            L.check(st, "bie_batch_solve")
        sols = [x.reshape(r.shape) for x, r in zip(self.split(xb), rhs)]
        infos = []
        for q in range(ns):
            info = {"status": int(st), "niter": niter[q * nd:(q + 1) * nd],
                    "rres": rres[q * nd:(q + 1) * nd]}
            if mode == 1:
                info["fp64_matvecs"] = int(stats[0])
                info["fp32_matvecs"] = int(stats[1])
            infos.append(info)
        return sols, infos, start.elapsed_time(stop)

    def _solve_streams(self, rhs, mode, numit, eps_gmres, concurrent):
        torch = self.torch
        main = torch.cuda.current_stream(self.device)
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        ends = [torch.cuda.Event() for _ in self.items]
        out = [None] * len(self.items)
        errors = []
        start.record(main)

        def run(q):
            try:
                s = self.streams[q] if concurrent else main
                with torch.cuda.stream(s):
                    s.wait_event(start)
                    out[q] = self.plans[q].solve(rhs[q], self.items[q].zid, mode=mode,
                                                 numit=numit, eps_gmres=eps_gmres)
                    ends[q].record(s)
            except Exception as e:  # reported after the join
                errors.append((q, e))

        if concurrent:
            th = [threading.Thread(target=run, args=(q,)) for q in range(len(self.items))]
            for t in th:
                t.start()
            for t in th:
                t.join()
        else:
            for q in range(len(self.items)):
                run(q)
        if errors:
            raise errors[0][1]
        for e in ends:
            main.wait_event(e)
        stop.record(main)
        stop.synchronize()
        sols = [o[0] for o in out]
        infos = [o[1] for o in out]
        return sols, infos, start.elapsed_time(stop)


def uneven_ellipsoids(kind: int, nsurf: int = 32, nrhs: int = 4, seed: int = 4):
    """Uneven batch: 32 ellipsoids with semi-axes U(0.5,3), 80/320/1280 patches,
    orders {4,6,8}, zk U(1,6) (Helmholtz, zpars = (k, -ik, 1)) or alpha =
    beta = 1 (Laplace), and nrhs interior point sources inside 0.3 x the
    semi-axes.  Returns (items, rhs arrays, source points)."""
    from .surface import icosa_ellipsoid
    rng = np.random.default_rng(seed)
    axes = rng.uniform(0.5, 3.0, (nsurf, 3))
    nrefs = rng.choice([1, 2, 3], nsurf)
    orders = rng.choice([4, 6, 8], nsurf)
    zks = rng.uniform(1.0, 6.0, nsurf)
    items, rhs, srcs = [], [], []
    for q in range(nsurf):
        s = icosa_ellipsoid(int(nrefs[q]), int(orders[q]), tuple(axes[q]))
        u = rng.normal(size=(nrhs, 3))
        u *= (rng.uniform(0, 1, (nrhs, 1)) ** (1 / 3)) / np.linalg.norm(u, axis=1)[:, None]
        x0 = 0.3 * axes[q] * u
        r = np.linalg.norm(s.xyz[:, None, :] - x0[None, :, :], axis=2)
        if kind == 0:
            items.append(BatchItem(s, 0, (1.0, 1.0), 0.5))
            rhs.append(1.0 / (4 * np.pi * r))
        else:
            k = float(zks[q])
            items.append(BatchItem(s, 1, (k, -1j * k, 1.0), 0.5))
            rhs.append(np.exp(1j * k * r) / (4 * np.pi * r))
        srcs.append(x0)
    return items, rhs, srcs
