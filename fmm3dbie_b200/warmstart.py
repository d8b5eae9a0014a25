"""Learned warm start for plane-wave Helmholtz solves.

The reference solver starts GMRES from zero (helm_comb_dir_solver_guru,
src/helm_wrappers/helm_comb_dir.f:2071, calls zgmres_guru at :2222).  Here a
per-node MLP, trained on solves that the method itself produced, predicts the
density of the plane-wave problem

    (zid I + K_k) sigma = -exp(i k d.x)          (zid = 1/2, zpars = (k, -ik, 1))

and the prediction is handed to the solver as its initial guess.  GMRES from
zero stays the fallback and the arbiter: the solve runs to the same relative
residual either way, and a guess whose residual is not below ||rhs|| is
dropped.

The network (csrc/cuda/mlp.cu) maps one row (d, (k - kc)/ks, x/xs, n) to the
demodulated density tau = sigma exp(-i k d.x), which varies on the scale of
the geometry rather than of the wavelength; the guess is tau_hat exp(i k d.x).
Training, inference, the feature gather and the (de)modulation all run in the
library's own kernels; torch only holds the device buffers.

The torus workload: x = (R + r(p) cos t) cos p, y = (R + r(p) cos t) sin p,
z = r(p) sin t, R = 2, r(p) = 0.6 + 0.15 cos 3p, 64 x 32 quad patches with
6 x 6 Gauss-Legendre nodes (iptype 11, norder 5, 73,728 nodes), k on a grid
in [1, 8] so that one near quadrature serves every direction at that k.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import _lib as L
from .plan import Plan
from .surface import Surface, setup, torus_quad

NPARAMS = 200706
N_IN, WIDTH, N_OUT = 10, 256, 2
_OFF_W = [0, 2560, 2560 + 65536, 2560 + 2 * 65536, 2560 + 3 * 65536]
_SHAPE_W = [(WIDTH, N_IN), (WIDTH, WIDTH), (WIDTH, WIDTH), (WIDTH, WIDTH), (N_OUT, WIDTH)]
ZID = 0.5
# feature scaling: x / 2.75 (torus extent), (k - 4.5) / 3.5 (k in [1, 8])
DEFAULT_NORM = (2.75, 4.5, 3.5)


def init_params(seed: int = 0) -> np.ndarray:
    """Glorot-uniform weights, zero biases, float32 in the flat layout."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, np.float32)
    for off, (fo, fi) in zip(_OFF_W, _SHAPE_W):
        a = math.sqrt(6.0 / (fi + fo))
        p[off:off + fo * fi] = rng.uniform(-a, a, fo * fi).astype(np.float32)
    return p


def _stream(torch, device):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _p(t):
    return C.c_void_p(t.data_ptr())


class WarmStartMLP:
    """The network on the current CUDA device (bie_mlp_* entry points)."""

    def __init__(self, params=None, seed: int = 0, max_rows: int = 65536, norm=DEFAULT_NORM):
        import torch
        self.torch = torch
        if not torch.cuda.is_available():
            raise RuntimeError("WarmStartMLP needs a CUDA device")
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.norm = np.array(norm, float)
        h = C.c_void_p()
        L.check(L.lib().bie_mlp_create(int(max_rows), C.byref(h)), "bie_mlp_create")
        self._h = h
        self.max_rows = int(max_rows)
        self.set_params(init_params(seed) if params is None else params)

    def close(self):
        if getattr(self, "_h", None):
            L.lib().bie_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _s(self):
        return _stream(self.torch, self.device)

    def info(self):
        """nparams, max_rows, inputs, width, hidden layers, outputs, Adam steps,
        weight count, engine, tcgen05 timeout flag."""
        out = np.zeros(10, np.int64)
        L.check(L.lib().bie_mlp_info(self._h, L.ptr(out)), "bie_mlp_info")
        return out

    def set_engine(self, engine: int):
        """0: mma.sync hidden-layer forward GEMMs; 1: tcgen05 (tensor memory)."""
        L.check(L.lib().bie_mlp_set_engine(self._h, int(engine)), "bie_mlp_set_engine")

    def set_params(self, params):
        t = self.torch.as_tensor(np.asarray(params, np.float32) if not
                                 isinstance(params, self.torch.Tensor) else params,
                                 dtype=self.torch.float32, device=self.device).contiguous()
        if t.numel() != NPARAMS:
            raise ValueError(f"expected {NPARAMS} parameters, got {t.numel()}")
        L.check(L.lib().bie_mlp_set_params(self._h, _p(t), self._s()), "bie_mlp_set_params")
        self.torch.cuda.current_stream(self.device).synchronize()

    def params(self):
        t = self.torch.empty(NPARAMS, dtype=self.torch.float32, device=self.device)
        L.check(L.lib().bie_mlp_get_params(self._h, _p(t), self._s()), "bie_mlp_get_params")
        return t

    def _rows(self, X):
        if X.dtype != self.torch.float32 or not X.is_contiguous() or X.shape[-1] != N_IN:
            raise ValueError("X must be a contiguous float32 (m, 10) tensor")
        return X.shape[0]

    def forward(self, X):
        m = self._rows(X)
        Y = self.torch.empty((m, N_OUT), dtype=self.torch.float32, device=self.device)
        L.check(L.lib().bie_mlp_forward(self._h, _p(X), m, _p(Y), self._s()), "bie_mlp_forward")
        return Y

    def grad(self, X, T):
        m = self._rows(X)
        G = self.torch.empty(NPARAMS, dtype=self.torch.float32, device=self.device)
        loss = self.torch.empty(1, dtype=self.torch.float32, device=self.device)
        L.check(L.lib().bie_mlp_grad(self._h, _p(X), _p(T), m, _p(G), _p(loss), self._s()),
                "bie_mlp_grad")
        return G, loss

    def train_step(self, X, T, lr: float, loss_out=None):
        m = self._rows(X)
        L.check(L.lib().bie_mlp_train_step(self._h, _p(X), _p(T), m, float(lr),
                                           _p(loss_out) if loss_out is not None else None,
                                           self._s()), "bie_mlp_train_step")

    def predict_density(self, srcvals_dev, dirk, out=None):
        """Initial guesses (npts, nd) complex128 for plane waves dirk[q] =
        (dx, dy, dz, k); srcvals_dev is the (npts, 12) srcvals on the device."""
        torch = self.torch
        npts = srcvals_dev.shape[0]
        dk = torch.as_tensor(np.asarray(dirk, float).reshape(-1, 4), device=self.device).contiguous()
        nd = dk.shape[0]
        if out is None:
            out = torch.empty((npts, nd), dtype=torch.complex128, device=self.device)
        L.check(L.lib().bie_mlp_predict_density(self._h, _p(srcvals_dev), npts, _p(dk), nd,
                                                L.ptr(self.norm), _p(out), self._s()),
                "bie_mlp_predict_density")
        return out

    def save(self, path: str, meta: dict | None = None):
        p = self.params().cpu().numpy()
        np.savez(path, params=p, norm=self.norm, meta=json.dumps(meta or {}))

    @classmethod
    def load(cls, path: str, max_rows: int = 65536):
        z = np.load(path, allow_pickle=False)
        return cls(params=z["params"], norm=tuple(z["norm"]), max_rows=max_rows)


# ---- the plane-wave problem on one surface ------------------------------------
def torus_surface(nu: int = 64, nv: int = 32, norder: int = 5) -> Surface:
    return torus_quad(nu, nv, norder, R=2.0, r0=0.6, r1=0.15, m=3)


def k_grid(nk: int, lo: float = 1.0, hi: float = 8.0) -> np.ndarray:
    """Wavenumbers at which near quadratures are generated (cell centres of
    [lo, hi], so the grid covers the interval evenly)."""
    return lo + (hi - lo) * (np.arange(nk) + 0.5) / nk


def random_directions(n: int, rng) -> np.ndarray:
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1)[:, None]


class PlaneWaveProblem:
    """Plans for (zid I + K_k) sigma = -exp(i k d.x) on one surface, one per k."""

    def __init__(self, surf: Surface, ks, eps: float = 1e-7):
        import torch
        self.torch = torch
        self.surf = surf
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.srcvals = torch.as_tensor(np.ascontiguousarray(surf.srcvals),
                                       device=self.device).contiguous()
        self.ks = [float(k) for k in ks]
        self.plans = {}
        self.setups = {}      # host copies of each wavenumber's setup arrays
        self.setup_s = 0.0
        for k in self.ks:
            t = time.perf_counter()
            zp = (k, -1j * k, 1.0)
            st = setup(surf, 1, eps, zp)
            self.setup_s += time.perf_counter() - t
            self.plans[k] = Plan(1, zp, surf, st.near, st.over)
            self.setups[k] = st

    def close(self):
        for p in self.plans.values():
            p.close()

    def rhs(self, k: float, dirs):
        torch = self.torch
        d = torch.as_tensor(np.asarray(dirs, float).reshape(-1, 3), device=self.device)
        ph = float(k) * (self.srcvals[:, 0:3] @ d.T)
        return (-torch.exp(1j * ph)).contiguous()

    @staticmethod
    def dirk(k: float, dirs):
        dirs = np.asarray(dirs, float).reshape(-1, 3)
        return np.concatenate([dirs, np.full((dirs.shape[0], 1), float(k))], axis=1)

    def solve(self, k: float, dirs, mode: int = 1, eps: float = 1e-6, x0=None, numit: int = 300):
        rhs = self.rhs(k, dirs)
        return self.plans[float(k)].solve(rhs, ZID, mode=mode, numit=numit, eps_gmres=eps, x0=x0)


def demodulate(srcvals_dev, dirk, sigma, tau_out):
    """tau_out[q, i] = sigma[i, q] exp(-i k_q d_q.x_i) (complex64 rows)."""
    import torch
    dk = torch.as_tensor(np.asarray(dirk, float).reshape(-1, 4), device=sigma.device).contiguous()
    nd = dk.shape[0]
    L.check(L.lib().bie_mlp_demodulate(_p(srcvals_dev), srcvals_dev.shape[0], _p(dk), nd,
                                       _p(sigma), _p(tau_out), _stream(torch, sigma.device)),
            "bie_mlp_demodulate")


def collect(problem: PlaneWaveProblem, dirs_per_k: dict, eps: float = 1e-7, batch: int = 16,
            log=None):
    """Solve every (k, d) with the mixed-precision solver and return (dirk
    (N x 4), tau (N, npts) complex64 on the device, solver stats)."""
    torch = problem.torch
    npts = problem.surf.npts
    rows = []
    for k, dirs in dirs_per_k.items():
        rows.append(PlaneWaveProblem.dirk(k, dirs))
    dirk = np.concatenate(rows, axis=0)
    tau = torch.empty((dirk.shape[0], npts), dtype=torch.complex64, device=problem.device)
    j = 0
    iters = []
    t0 = time.perf_counter()
    for k, dirs in dirs_per_k.items():
        for b0 in range(0, len(dirs), batch):
            d = dirs[b0:b0 + batch]
            x, info = problem.solve(k, d, mode=1, eps=eps)
            if info["status"] != 0:
                raise RuntimeError(f"training solve did not converge at k={k}: {info}")
            demodulate(problem.srcvals, dirk[j:j + len(d)], x, tau[j:j + len(d)])
            iters.append(int(info["fp32_matvecs"]))
            j += len(d)
            if log:
                log(f"k={k:.3f} solved {j}/{dirk.shape[0]} ({time.perf_counter() - t0:.1f} s)")
    return dirk, tau, {"fp32_matvecs_per_batch": iters, "seconds": time.perf_counter() - t0}


def train(mlp: WarmStartMLP, srcvals_dev, dirk, tau, steps: int, batch: int = 16384,
          lr: float = 2e-3, lr_final: float = 2e-5, seed: int = 1, log_every: int = 0, log=None):
    """Adam on the mean squared error of tau over random (solve, node) rows;
    cosine learning-rate decay from lr to lr_final.  Returns the per-step loss."""
    torch = mlp.torch
    dev = mlp.device
    npts = srcvals_dev.shape[0]
    dk = torch.as_tensor(np.asarray(dirk, float), device=dev).contiguous()
    nsol = dk.shape[0]
    X = torch.empty((batch, N_IN), dtype=torch.float32, device=dev)
    T = torch.empty((batch, N_OUT), dtype=torch.float32, device=dev)
    losses = torch.zeros(steps, dtype=torch.float32, device=dev)
    tau_f = tau.view(torch.float32)
    s = _stream(torch, dev)
    lib = L.lib()
    norm = L.ptr(mlp.norm)
    for it in range(steps):
        L.check(lib.bie_mlp_gather(_p(srcvals_dev), npts, _p(dk), nsol, _p(tau_f), norm,
                                   C.c_uint64((seed << 40) + it), batch, _p(X), _p(T), s),
                "bie_mlp_gather")
        c = 0.5 * (1 + math.cos(math.pi * it / max(steps - 1, 1)))
        mlp.train_step(X, T, lr_final + (lr - lr_final) * c, losses[it:it + 1])
        if log and log_every and (it + 1) % log_every == 0:
            log(f"step {it + 1}/{steps} loss {losses[it].item():.4e}")
    return losses.cpu().numpy()


def prediction_error(mlp: WarmStartMLP, srcvals_dev, dirk, tau):
    """Relative L2 error of the predicted tau per solve."""
    torch = mlp.torch
    npts = srcvals_dev.shape[0]
    out = []
    for q in range(len(dirk)):
        x0 = mlp.predict_density(srcvals_dev, dirk[q:q + 1])
        tt = torch.empty((1, npts), dtype=torch.complex64, device=mlp.device)
        demodulate(srcvals_dev, dirk[q:q + 1], x0.contiguous(), tt)
        ref = tau[q]
        out.append(float(torch.linalg.norm(tt[0] - ref) / torch.linalg.norm(ref)))
    return np.array(out)


def evaluate(problem: PlaneWaveProblem, mlp: WarmStartMLP, k: float, dirs, eps: float = 1e-6):
    """Solve the directions at k from zero and from the network's guess
    (mixed precision, one batch) and report iterations, device time and
    accuracy against an FP64 solution at 1e-11."""
    torch = problem.torch
    dirk = PlaneWaveProblem.dirk(k, dirs)
    w = torch.as_tensor(problem.surf.qwts(), device=problem.device)

    def wn(v):
        return torch.sqrt((w[:, None] * v.abs() ** 2).sum(0))

    xref, _ = problem.solve(k, dirs, mode=0, eps=1e-11)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    xz, iz = problem.solve(k, dirs, mode=1, eps=eps)
    ev[1].record()
    ev[2].record()
    x0 = mlp.predict_density(problem.srcvals, dirk)
    xw, iw = problem.solve(k, dirs, mode=1, eps=eps, x0=x0)
    ev[3].record()
    torch.cuda.synchronize()
    r = {"k": float(k), "nd": int(len(dirs)),
         "pred_err_median": float(torch.median(wn(x0 - xref) / wn(xref))),
         "iters_zero": float(iz["niter"].mean()), "iters_warm": float(iw["niter"].mean()),
         "fp64_matvecs_zero": iz["fp64_matvecs"], "fp64_matvecs_warm": iw["fp64_matvecs"],
         "ms_zero": ev[0].elapsed_time(ev[1]), "ms_warm": ev[2].elapsed_time(ev[3]),
         "err_zero": float(torch.max(wn(xz - xref) / wn(xref))),
         "err_warm": float(torch.max(wn(xw - xref) / wn(xref))),
         "rres_zero": float(iz["rres"].max()), "rres_warm": float(iw["rres"].max())}
    return r


def main(argv=None):
    ap = argparse.ArgumentParser(description="Train the warm-start MLP on the torus workload")
    ap.add_argument("--nu", type=int, default=64)
    ap.add_argument("--nv", type=int, default=32)
    ap.add_argument("--norder", type=int, default=5)
    ap.add_argument("--nk", type=int, default=8)
    ap.add_argument("--nsolves", type=int, default=2000)
    ap.add_argument("--steps", type=int, default=300000)
    ap.add_argument("--batch", type=int, default=32768)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--eps", type=float, default=1e-7)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    import torch
    log = lambda s: print(s, flush=True)  # noqa: E731
    surf = torus_surface(a.nu, a.nv, a.norder)
    ks = k_grid(a.nk)
    rng = np.random.default_rng(a.seed)
    per_k = a.nsolves // a.nk
    dirs = {float(k): random_directions(per_k, rng) for k in ks}
    t = time.perf_counter()
    prob = PlaneWaveProblem(surf, ks)
    log(f"setup of {len(ks)} wavenumbers: {time.perf_counter() - t:.1f} s")
    dirk, tau, stats = collect(prob, dirs, eps=a.eps, log=log)
    torch.cuda.synchronize()
    mlp = WarmStartMLP(seed=a.seed)
    t = time.perf_counter()
    losses = train(mlp, prob.srcvals, dirk, tau, a.steps, batch=a.batch, lr=a.lr,
                   log_every=max(a.steps // 20, 1), log=log)
    torch.cuda.synchronize()
    tt = time.perf_counter() - t
    err = prediction_error(mlp, prob.srcvals, dirk[::25], tau[::25])
    meta = {"surface": [a.nu, a.nv, a.norder], "ks": [float(k) for k in ks],
            "nsolves": int(dirk.shape[0]), "steps": a.steps, "batch": a.batch, "lr": a.lr,
            "seed": a.seed, "eps": a.eps, "train_seconds": tt,
            "final_loss": float(np.mean(losses[-100:])),
            "train_rel_err_median": float(np.median(err)), "collect": stats["seconds"]}
    log(json.dumps(meta))
    mlp.save(a.out, meta)
    # held-out directions at two of the grid wavenumbers
    hold = np.random.default_rng(a.seed + 1000)
    for k in (ks[len(ks) // 4], ks[(3 * len(ks)) // 4]):
        log(json.dumps(evaluate(prob, mlp, float(k), random_directions(16, hold))))
    prob.close()


if __name__ == "__main__":
    main()
