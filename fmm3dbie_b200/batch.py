"""Batches of independent surfaces (uneven sizes, orders and wavenumbers).

``SurfaceBatch`` keeps one device plan per surface and solves all of them
together: every surface's GMRES runs on its own CUDA stream from its own host
thread (the ctypes calls release the GIL), so small and large surfaces share
the GPU concurrently instead of queueing behind each other.  Each surface may
carry several right-hand sides, which its plan solves as one multi-density
batch.  After the first solve of a plan no call allocates device memory, so
the streams never serialise on a cudaFree.
"""
from __future__ import annotations

import threading
from dataclasses import dataclass

import numpy as np

from .plan import Plan
from .surface import Surface, setup


@dataclass
class BatchItem:
    surf: Surface
    kind: int          # 0 Laplace, 1 Helmholtz
    params: tuple      # (alpha, beta) or (k, alpha, beta)
    zid: complex       # identity term of the second-kind equation


class SurfaceBatch:
    def __init__(self, items, eps: float):
        import torch
        self.torch = torch
        self.items = list(items)
        self.setups = [setup(it.surf, it.kind, eps, it.params) for it in self.items]
        self.plans = [Plan(it.kind, it.params, it.surf, st.near, st.over)
                      for it, st in zip(self.items, self.setups)]
        dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.streams = [torch.cuda.Stream(dev) for _ in self.items]

    def close(self):
        for p in self.plans:
            p.close()

    def solve(self, rhs, mode: int = 1, numit: int = 200, eps_gmres: float = 1e-7,
              concurrent: bool = True):
        """rhs[q]: (npts_q, nrhs_q) device tensors.  Returns (solutions,
        infos, device milliseconds from the first launch to the last
        completion)."""
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
