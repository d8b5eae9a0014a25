#!/usr/bin/env python
"""Benchmark: Helmholtz combined-field Dirichlet solves per second on one B200.

Workload (the headline configuration): exterior Helmholtz CFIE Dirichlet
problem on the ellipsoid with semi-axes (1,2,3), an icosahedron refined 3x
(1280 flat triangles radially projected) discretised with order-6
Vioreanu-Rokhlin nodes (npts = 35840), zk = 2, zpars = (zk, -i zk, 1),
eps = 1e-7, right-hand side the field of a unit point source at
(0.1,-0.2,0.3) inside the surface, solved to FP64 relative residual 1e-10.
One step = one full solve.

  ours (value)  : FP32/complex64 matvec GMRES inside FP64 iterative
                  refinement to FP64 relative residual <= 1e-10, inputs
                  resident on the device (plan built once);
  fp64 path     : the reference method (FP64 GMRES to the same residual) on
                  the same plan, reported beside it;
  e2e           : the same solve through the host-buffer C-ABI entry point
                  bie_helm_comb_dir_solver_guru_ext (all operator data, rhs and
                  solution copied between pinned host memory and the device
                  inside the timed region);
  legs          : 64 plane waves at zk 5 (batched), 32 uneven ellipsoids, the
                  quad torus with the learned warm start, each against plain
                  FP64 GMRES one right-hand side at a time, each with its
                  error against the FP64 oracle; the hierarchical far field;
  --impl reference : the oracle (oracle/: an FP64 C restatement of the
                  reference path, its own surface, setup and near quadrature,
                  and a CPU far field standing in for FMM3D) timed on the host
                  cores, one GMRES iteration per step.

Timing: per-step CUDA events on the launch stream, an L2 flush (write of a
256 MiB buffer) between timed steps, barrier + synchronize around the timed
region, max over ranks.  N > 1 runs independent replicas (the path has no
data exchange between solves): value = all ranks' solves / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/sec at 1e-6 rel err: mixed-prec+batched+warm-start vs plain FP64 GPU"
WORKLOAD = ("Helmholtz CFIE Dirichlet GMRES solve, ellipsoid (1,2,3), 1280 order-6 RV patches, "
            "npts 35840, zk=2, zpars=(2,-2i,1), eps=1e-7, interior point-source rhs, "
            "FP64 residual 1e-10")
ZK = 2.0
ZPARS = (ZK, -1j * ZK, 1.0)
EPS = 1e-7
X0 = np.array([0.1, -0.2, 0.3])
TOL_RES = 1e-10     # FP64 relative residual target of the timed solves (config 2)
TOL_LOOSE = 1e-7    # the same solves stopped at 1e-7, reported beside them
TOL_WARM = 3e-7     # residual target of the torus warm-start solves (error <= 1e-6)
# identical in both arms
CONFIG = {"workload": WORKLOAD, "residual": TOL_RES,
          "parallelism": "replicas, one process per GPU, no data exchange",
          "l2": "L2 flushed (256 MiB write) between timed steps; the FP32 near-correction "
                "matrix (140 MB) alone exceeds L2"}
ORACLE_TREE = (0.5, 9, 256)   # treecode theta, Chebyshev points per side, leaf size
FLOPS_PER_PAIR = {"helm": 26 + 16, "lap": 15 + 4}   # 1 density: geometry + per-density MACs


def flops_per_pair(kind: str, nd: int = 1) -> int:
    return (26 + 16 * nd) if kind == "helm" else (15 + 4 * nd)


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), \
        int(os.environ.get("LOCAL_RANK", 0))


def build_problem(nref=3, norder=6, nq_stats=None):
    """The ellipsoid, its setup (near quadrature on the device when one is
    visible; nq_stats receives the generator's counters) and the rhs."""
    from fmm3dbie_b200 import surface as S
    s = S.icosa_ellipsoid(nref, norder, (1.0, 2.0, 3.0))
    t = time.time()
    st = S.setup(s, 1, EPS, ZPARS, stats=nq_stats)
    r = np.linalg.norm(s.xyz - X0, axis=1)
    rhs = np.exp(1j * ZK * r) / (4 * np.pi * r)
    return s, st, rhs, time.time() - t


def nearquad_compare(s, st):
    """Near quadrature of the bench ellipsoid by the host generator (all host
    cores) and the device generator, on the same near list."""
    from fmm3dbie_b200 import surface as S
    targs = s.srcvals
    ipatch_id, uvs = s.patch_id_uvs()
    nf = st.near
    args = (s, 1, EPS, ZPARS, targs, ipatch_id, uvs, nf.row_ptr, nf.col_ind, nf.iquad, st.rfac0)
    t0 = time.time()
    wc = S.getnearquad(*args, engine="cpu")
    t_cpu = time.time() - t0
    gs = np.zeros(4, np.int64)
    t0 = time.time()
    wg = S.getnearquad(*args, engine="gpu", stats=gs)
    t_gpu = time.time() - t0
    diff = float(np.max(np.abs(wg - wc)) / np.max(np.abs(wc)))
    return {"host_generator_s": round(t_cpu, 3), "host_cores": len(os.sched_getaffinity(0)),
            "device_call_s": round(t_gpu, 3), "device_kernel_ms": gs[3] / 1e3,
            "kernel_evals": int(gs[0]), "pairs": int(gs[1] + gs[2]),
            "max_abs_diff_over_max": diff}


def exterior_field_error(s, soln, zp=ZPARS, x0=X0, n=100, radius=5.0, seed=2):
    """Max relative error of the smooth-rule field (alpha S + beta D) soln at
    n seeded points on the sphere of the given radius against the analytic
    field of the interior point source (helm_dir_iter_example.f)."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    targ = radius * v / np.linalg.norm(v, axis=1)[:, None]
    k = zp[0]
    w = s.qwts()
    u = np.zeros(n, complex)
    for i, t in enumerate(targ):
        dx = t[None, :] - s.xyz
        r = np.linalg.norm(dx, axis=1)
        dn = np.sum(dx * s.normals, 1)
        ker = (zp[1] / r + zp[2] * dn * (1 - 1j * k * r) / r ** 3) * np.exp(1j * k * r) / (4 * np.pi)
        u[i] = np.sum(ker * w * soln)
    d = np.linalg.norm(targ - x0, axis=1)
    uex = np.exp(1j * k * d) / (4 * np.pi * d)
    return float(np.max(np.abs(u - uex)) / np.max(np.abs(uex)))


def gpu_uuid(dev_index):
    """NVML/nvidia-smi identifier of a CUDA device (CUDA ordinals and NVML
    indices differ under CUDA_VISIBLE_DEVICES)."""
    try:
        import torch
        u = str(torch.cuda.get_device_properties(dev_index).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(dev_index)


class NvmlClockSampler:
    """Clocks and throttle reasons sampled every 20 ms through NVML from a
    background thread during the timed region."""
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40}

    def __init__(self, dev_index, period=0.02):
        import threading
        import pynvml
        self.nv = pynvml
        pynvml.nvmlInit()
        self.h = pynvml.nvmlDeviceGetHandleByUUID(gpu_uuid(dev_index).encode())
        self.period = period
        self.rows = []
        self.stop_ev = threading.Event()
        self.th = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        nv = self.nv
        while not self.stop_ev.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                smax = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
                try:
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except Exception:
                    rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                self.rows.append((sm, smax, rs))
            except Exception:
                pass
            self.stop_ev.wait(self.period)

    def start(self):
        self.th.start()

    def stop(self):
        self.stop_ev.set()
        self.th.join(timeout=5)
        sm = [r[0] for r in self.rows]
        reasons = sorted({k for r in self.rows for k, b in self.BITS.items() if r[2] & b})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(r[1] for r in self.rows) if self.rows else None,
                "reasons": reasons, "samples": len(self.rows), "sampler": "nvml"}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_uuid(gpu_index)
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [ln.strip().split(",") for ln in self.f.read().splitlines() if ln.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(rows)}


# ---- CPU legs: the oracle (test infrastructure) as baseline and checker -------
# Only the functions in this section import oracle/; none of them runs inside
# a GPU timed region, and the GPU path never calls the oracle.
def oracle_problem():
    """The headline problem built by the oracle alone: its own surface
    (the reference's icosahedron and ellipsoid chart), near list, far
    orders, oversampled geometry and near quadrature."""
    import oracle
    t0 = time.time()
    s = oracle.icosa_ellipsoid(3, 6, (1.0, 2.0, 3.0))
    st = oracle.setup(s, 1, EPS, ZPARS)
    r = np.linalg.norm(s.xyz - X0, axis=1)
    rhs = np.exp(1j * ZK * r) / (4 * np.pi * r)
    return s, st, rhs, time.time() - t0


def oracle_far_choice(s, st):
    """The faster of the oracle's two CPU far fields on this surface, timed
    in-run: the vectorised direct sum (exact) or the barycentric treecode
    (ORACLE_TREE; its difference from the direct sum is measured)."""
    import oracle
    rng = np.random.default_rng(0)
    sig = rng.normal(size=s.npts) + 1j * rng.normal(size=s.npts)
    w = oracle.qwts(s)
    out = {}
    for m in (1, 2):
        oracle.set_far_method(m, *ORACLE_TREE)
        t0 = time.perf_counter()
        y = oracle.lpcomp(1, s, ZPARS, st.near, st.over, sig)
        out[m] = (time.perf_counter() - t0, y)
    err = float(np.sqrt(np.sum(w * np.abs(out[2][1] - out[1][1]) ** 2) /
                        np.sum(w * np.abs(out[1][1]) ** 2)))
    m = 1 if out[1][0] <= out[2][0] else 2
    oracle.set_far_method(m, *ORACLE_TREE)
    names = {1: "vectorised direct sum (exact)",
             2: f"barycentric Lagrange treecode (theta {ORACLE_TREE[0]}, {ORACLE_TREE[1]} "
                f"Chebyshev points per side + k side/2, leaves {ORACLE_TREE[2]}; O(N log N))"}
    return m, {"method": names[m], "matvec_s_direct": round(out[1][0], 3),
               "matvec_s_treecode": round(out[2][0], 3), "treecode_vs_direct": err}


def reference_arm(args):
    """The reference's CPU path, timed: the oracle's FP64 GMRES
    (zgmres_guru) with its matvec (lpcomp_helm_comb_dir_addsub restated, the
    FMM replaced by the faster of the oracle's CPU far fields) on the
    headline surface, which the oracle also builds and sets up itself.  One
    step = one operator application of the solve: an Arnoldi iteration, or
    the closing true-residual evaluation; the steps run one continuous solve
    (a new one from zero after each completes), so the run executes at least
    one whole solve, whose iteration count converts steps to solves."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    import oracle
    cores = len(os.sched_getaffinity(0))
    s, st, rhs, t_setup = oracle_problem()
    method, far = oracle_far_choice(s, st)
    new = lambda: oracle.GmresSolver(1, s, ZPARS, st.near, st.over, 0.5, rhs, numit=300,  # noqa: E731
                                     eps_gmres=TOL_RES)
    g = new()
    solves = []
    cur = []           # step times of the solve in progress
    times = []
    step = 0
    while step < args.warmup + args.steps or not solves:
        t0 = time.perf_counter()
        if g.done:
            x, m, errs, rres = g.finish()
        else:
            g.step()
        dt = time.perf_counter() - t0
        cur.append(dt)
        if g.done and len(cur) == g.it + 1:
            solves.append({"niter": m, "rres": rres, "s": float(sum(cur))})
            g, cur = new(), []
        if args.warmup <= step < args.warmup + args.steps:
            times.append(dt)
        step += 1
    ops = solves[0]["niter"] + 1
    ms = 1000.0 * float(np.mean(times))
    value = 1000.0 / (ms * ops)
    sample = (f"oracle FP64 GMRES on the headline surface (oracle's own surface, setup and near "
              f"quadrature; far field: {far['method']}), {args.steps} timed operator "
              f"applications of {ops} per solve ({solves[0]['niter']} Arnoldi iterations + "
              f"the true residual); a whole solve measured in-run took {solves[0]['s']:.1f} s")
    base = {"value": value, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample}
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "impl": "reference", "data": "synthetic: seeded ellipsoid surface and point-source rhs",
            "config": CONFIG, "cpu_baseline": base,
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "reference": {"setup_s": round(t_setup, 1), "npts": s.npts, "nptso": st.over.nptso,
                          "far_field": far, "solves": solves, "steps_run": step,
                          "untimed_steps_after": step - args.warmup - args.steps}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_leg(x_mixed, x_fp64, niter64, sample_iters=6):
    """CPU baseline of the 'ours' line and the oracle checks of the headline
    solve.  Baseline: the oracle's FP64 GMRES on its own setup of the same
    surface, sample_iters Arnoldi iterations timed, scaled to one solve of
    niter64 + 1 operator applications (niter64 from the GPU's plain FP64
    GMRES on this surface).  Checks: the residual of the GPU solutions under
    the oracle's operator (independent setup and near quadrature; exact
    vectorised direct far field)."""
    import oracle
    cores = len(os.sched_getaffinity(0))
    s, st, rhs, t_setup = oracle_problem()
    method, far = oracle_far_choice(s, st)
    g = oracle.GmresSolver(1, s, ZPARS, st.near, st.over, 0.5, rhs, numit=300, eps_gmres=TOL_RES)
    g.step()   # warm-up
    t0 = time.perf_counter()
    for _ in range(sample_iters):
        g.step()
    t_it = (time.perf_counter() - t0) / sample_iters
    value = 1.0 / (t_it * (niter64 + 1))
    base = {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": (f"oracle FP64 GMRES iterations on the headline surface (oracle's own "
                       f"setup, {t_setup:.0f} s; far field: {far['method']}): {sample_iters} "
                       f"iterations at {t_it:.2f} s, scaled to {niter64}+1 operator "
                       f"applications per solve"),
            "far_field": far}
    oracle.set_far_method(1)
    w = oracle.qwts(s)
    checks = {}
    for tag, x in (("mixed", x_mixed), ("fp64", x_fp64)):
        y = oracle.lpcomp(1, s, ZPARS, st.near, st.over, x)
        res = rhs - (0.5 * x + y)
        checks[tag] = float(np.sqrt(np.sum(w * np.abs(res) ** 2) / np.sum(w * np.abs(rhs) ** 2)))
    oracle.set_far_method(0)
    return base, {"oracle_residual": checks,
                  "note": "relative residual of the GPU solution under the oracle's operator "
                          "(oracle's own surface, near list, far orders, oversampling and near "
                          "quadrature; exact far field)"}


def oracle_residual(kind, surf, params, near, over, rhs, x, zid=0.5):
    """Residual of a GPU solution under the oracle's matvec on the same
    inputs (exact vectorised direct far field)."""
    import oracle
    oracle.set_far_method(1)
    w = oracle.qwts(surf)
    y = oracle.lpcomp(kind, surf, params, near, over, x)
    oracle.set_far_method(0)
    r = rhs - (zid * x + y)
    return float(np.sqrt(np.sum(w * np.abs(r) ** 2) / np.sum(w * np.abs(rhs) ** 2)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--matvec-only", type=int, default=0,
                    help="build the workload, run this many matvecs (see --prec) and exit "
                         "(the command the ncu summaries in profiles/ use)")
    ap.add_argument("--prec", type=int, default=1, help="matvec precision for --matvec-only")
    ap.add_argument("--nd", type=int, default=1, help="densities per matvec for --matvec-only")
    ap.add_argument("--clock-sampler", default="nvml", choices=["nvml", "smi"])
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched leg (64 plane-wave right-hand sides)")
    ap.add_argument("--torus", action="store_true", help="(default) the torus warm-start leg")
    ap.add_argument("--no-torus", action="store_true", help="skip the torus warm-start leg")
    ap.add_argument("--nearquad-only", type=int, default=0, metavar="NREF",
                    help="only run the device near-quadrature generator (Helmholtz, eps 1e-7) on "
                         "the (1,2,3) ellipsoid refined NREF times, order 6, and print its counters")
    ap.add_argument("--no-nearquad", action="store_true",
                    help="skip the near-quadrature generator comparison (host vs device)")
    ap.add_argument("--tree-only", type=int, default=0, metavar="NREF",
                    help="only compare the hierarchical and direct far fields on the (1,2,3) "
                         "ellipsoid refined NREF times (order --tree-order)")
    ap.add_argument("--tree-order", type=int, default=6)
    ap.add_argument("--tree", type=int, default=4, metavar="NREF",
                    help="add the hierarchical far-field leg on the ellipsoid refined NREF times")
    ap.add_argument("--uneven", action="store_true", help="(default) the uneven batch leg")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven batch leg")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.matvec_only:
        return matvec_only(args)
    if args.nearquad_only:
        return nearquad_only(args.nearquad_only)
    if args.tree_only:
        print(json.dumps({"tree": tree_leg(args.tree_only, args.tree_order)}))
        return 0

    import torch
    import torch.distributed as dist
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from fmm3dbie_b200 import Plan, layer
    from fmm3dbie_b200 import _lib as L
    lib = L.lib()

    nq_stats = np.zeros(4, np.int64)
    s, st, rhs, t_setup = build_problem(nq_stats=nq_stats)
    P = Plan(1, ZPARS, s, st.near, st.over)
    stream = torch.cuda.current_stream(dev)
    r_d = torch.tensor(rhs, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2

    # accuracy reference: tight FP64 solution
    x_ref, info_ref = P.solve(r_d, 0.5, mode=0, numit=300, eps_gmres=1e-13)
    w = torch.tensor(s.qwts(), device=dev)

    def relerr(x):
        return float(torch.sqrt(torch.sum(w * (x - x_ref).abs() ** 2) /
                                torch.sum(w * x_ref.abs() ** 2)))

    def timed(fn, k, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ts = []
        for _ in range(k):
            flush.fill_(1.0)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            out = fn()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        return ts, out

    # ---- plain FP64 GPU path (the reference method) --------------------------
    f64 = lambda: P.solve(r_d, 0.5, mode=0, numit=300, eps_gmres=TOL_RES)  # noqa: E731
    ts64, (x64, info64) = timed(f64, max(1, args.steps // 2), 1)
    t64 = float(np.mean(ts64))
    # the same two paths stopped at residual 1e-7
    loose = {}
    for mode, tag in ((0, "fp64"), (1, "mixed")):
        fl = lambda: P.solve(r_d, 0.5, mode=mode, numit=300, eps_gmres=TOL_LOOSE)  # noqa: E731
        tl, (xl, il) = timed(fl, 3, 1)
        loose[tag] = {"solves_per_s": 1000.0 / float(np.mean(tl)), "ms_per_solve": float(np.mean(tl)),
                      "niter": int(il["niter"][0]), "rres": float(il["rres"][0]),
                      "rel_err_vs_fp64_1e-13": relerr(xl)}
    loose["speedup_vs_fp64"] = loose["fp64"]["ms_per_solve"] / loose["mixed"]["ms_per_solve"]

    # ---- ours: mixed precision, timed region with clocks + stage timing -------
    mixed = lambda: P.solve(r_d, 0.5, mode=1, numit=300, eps_gmres=TOL_RES)  # noqa: E731
    for _ in range(args.warmup):
        mixed()
    if args.clock_sampler == "nvml":
        try:
            clocks = NvmlClockSampler(local)
        except Exception:
            clocks = ClockSampler(local)
    else:
        clocks = ClockSampler(local)
    clocks.start()
    n0 = lib.bie_launch_count()
    tsm, (xm, infom) = timed(mixed, args.steps, 0)
    launches = int(lib.bie_launch_count() - n0)
    ck = clocks.stop()
    # stage times (CUDA events per matvec stage; the stage timing synchronises
    # after every matvec, so it runs after the timed region, on two more solves)
    P.timing(True)
    for _ in range(2):
        mixed()
    torch.cuda.synchronize()
    stages = P.timing(False)
    pinfo = P.info()
    tm = float(np.mean(tsm))
    tmax = float(np.sum(tsm))
    if world > 1:
        tt = torch.tensor([tmax], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        tmax = float(tt.item())
    value = world * args.steps / (tmax / 1000.0)

    # roofline of the dominant kernel: the f32 far-field N-body
    far32 = stages["f32"]
    far_ms = far32["far_ms"] / max(far32["calls"], 1)
    pairs = float(P.ntarg) * float(P.nptso)
    achieved = pairs * flops_per_pair("helm") / (far_ms * 1e-3) / 1e12
    peak_tf = ctypes_double_pair(lib)
    mufu_pk = mufu_peak(lib)
    mufu_ach = pairs * MUFU_PER_PAIR["helm"] / (far_ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "far_kernel_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get("bytes_per_launch")
        except Exception:
            traffic = None
    far64 = stages["f64"]
    far64_ms = far64["far_ms"] / max(far64["calls"], 1) if far64["calls"] else None

    # ---- e2e through the host-buffer C-ABI (pinned host memory) ---------------
    e2e = None
    if args.e2e_steps > 0:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
        hs = {k: pin(getattr(s, k)) for k in ("norders", "ixyzs", "iptype", "srcvals", "srccoefs")}
        from fmm3dbie_b200.surface import Surface, NearField, Oversampled
        s_p = Surface(**hs)
        n_p = NearField(pin(st.near.row_ptr), pin(st.near.col_ind), pin(st.near.iquad),
                        pin(st.near.wnear))
        o_p = Oversampled(pin(st.over.novers), pin(st.over.ixyzso), pin(st.over.srcover),
                          pin(st.over.wover))
        rhs_p = pin(rhs[:, None])
        h2d = sum(a.nbytes for a in list(hs.values()) + [n_p.row_ptr, n_p.col_ind, n_p.iquad,
                                                          n_p.wnear, o_p.novers, o_p.ixyzso,
                                                          o_p.srcover, o_p.wover, rhs_p])
        d2h = rhs_p.nbytes
        run = lambda: layer.helm_comb_dir_solver_guru_ext(s_p, EPS, ZPARS, 300, 1, rhs_p, n_p, o_p,  # noqa: E731
                                                          TOL_RES, iprec=1)
        run()
        torch.cuda.synchronize()
        te = []
        for _ in range(args.e2e_steps):
            t0 = time.perf_counter()
            out = run()
            te.append(time.perf_counter() - t0)
        e2e = {"value": 1.0 / float(np.mean(te)), "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "path": "bie_helm_comb_dir_solver_guru_ext (host buffers)",
               "rres": float(out[1][0])}

    # ---- cold solve through the reference's simple interface -------------------
    # helm_comb_dir_solver: setup (near list, far orders, oversampled geometry,
    # near quadrature) + plan + FP64 GMRES, host buffers in and out
    e2e_cold = None
    if args.e2e_steps > 0 and rank == 0:
        lib_ = L.lib()
        cold = {}
        for eng, reps in ((1, 2), (0, 1)):
            lib_.bie_set_nearquad_engine(eng)
            for _ in range(reps):
                t0 = time.perf_counter()
                niter_c, _, rres_c, _, st_c = layer.helm_comb_dir_solver(s, EPS, ZPARS, 300, 1, rhs,
                                                                        TOL_RES)
                cold[eng] = time.perf_counter() - t0
        lib_.bie_set_nearquad_engine(1)
        e2e_cold = {"value": 1.0 / cold[1], "unit": "solves/s",
                    "path": "bie_helm_comb_dir_solver (setup + plan + FP64 GMRES, host buffers)",
                    "s_per_solve_device_setup": round(cold[1], 3),
                    "s_per_solve_host_setup": round(cold[0], 3), "niter": niter_c,
                    "rres": rres_c}

    # second oracle: the analytic exterior field of the interior point source
    # at 100 seeded targets on the radius-5 sphere, from the timed solution
    xm_h = xm.cpu().numpy()
    ext = exterior_field_error(s, xm_h)

    base = None
    checks = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base, checks = cpu_baseline_leg(xm_h, x64.cpu().numpy(), int(info64["niter"][0]))
    nearquad = None
    if rank == 0 and world == 1 and not args.no_nearquad:
        nearquad = nearquad_compare(s, st)
    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        P.close()
        batched = batched_leg(dev)
    uneven = None
    if rank == 0 and world == 1 and not args.no_uneven:
        P.close()
        uneven = uneven_leg(dev)
    torus = None
    if rank == 0 and world == 1 and not args.no_torus:
        P.close()
        torus = torus_leg(dev)
    tree = None
    if rank == 0 and world == 1 and args.tree:
        P.close()
        tree = tree_leg(args.tree)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tmax / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64 matvec + c128 refinement/Krylov",
            "data": "synthetic: seeded ellipsoid surface and point-source rhs",
            "config": CONFIG,
            "fp64_path": {"solves_per_s": 1000.0 / t64, "ms_per_solve": t64,
                          "niter": int(info64["niter"][0]), "rres": float(info64["rres"][0]),
                          "rel_err_vs_fp64_1e-13": relerr(x64)},
            "speedup_vs_fp64": t64 / tm,
            "mixed": {"inner_iters": int(infom["niter"][0]), "rres": float(infom["rres"][0]),
                      "rel_err_vs_fp64_1e-13": relerr(xm), "fp64_matvecs": infom["fp64_matvecs"],
                      "fp32_matvecs": infom["fp32_matvecs"]},
            "accuracy": {"exterior_field_max_rel_err": ext,
                         "exterior_field_note": "100 seeded points on the radius-5 sphere, "
                                                "against the analytic point-source field",
                         "oracle": checks},
            "residual_1e-7": loose,
            "problem": {"npts": P.npts, "nptso": P.nptso, "nnz": P.nnz, "nquad": P.nquad,
                        "setup_s": round(t_setup, 2),
                        "nearquad_device_kernel_ms": nq_stats[3] / 1e3,
                        "nearquad_kernel_evals": int(nq_stats[0]),
                        "far_shape_variant_chunks": {"f64": [int(pinfo[8]), int(pinfo[5])],
                                                     "f32": [int(pinfo[9]), int(pinfo[6])]}},
            "roofline": {"kernel": "far_kernel<helm,f32>", "bound": "fp32", "achieved": achieved,
                         "peak": peak_tf, "unit": "TFLOP/s", "frac": achieved / peak_tf,
                         "traffic": traffic,
                         "peak_source": "FP32 FFMA loop measured in this run "
                                        "(MEASURED_PEAKS.json has no FP32 SIMT figure)",
                         "flops_per_pair": flops_per_pair("helm"), "pairs_per_launch": pairs,
                         "avg_launch_ms": far_ms,
                         "mufu": {"ops_per_pair": MUFU_PER_PAIR["helm"], "achieved_gops": mufu_ach,
                                  "peak_gops": mufu_pk, "frac": mufu_ach / mufu_pk,
                                  "peak_source": "rsqrt.approx loop measured in this run"}},
            "stage_ms_per_matvec": {
                "f32": {k: far32[k] / max(far32["calls"], 1) for k in ("strengths_ms", "far_ms", "combine_ms")},
                "f64": {k: far64[k] / max(far64["calls"], 1) for k in ("strengths_ms", "far_ms", "combine_ms")}},
            "gpu_launches": launches,
            "clocks": ck,
            "e2e": e2e,
            "e2e_cold": e2e_cold,
            "cpu_baseline": base,
            "nearquad": nearquad,
            "batched": batched,
            "uneven": uneven,
            "torus_warm_start": torus,
            "tree": tree,
        }
        print(json.dumps(line), flush=True)
    P.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def batched_leg(dev, steps=1):
    """64 incident plane waves on the same (1,2,3) ellipsoid at
    zk = 5, zpars = (5, -5i, 1); rhs = -incident field at the nodes.  All 64
    systems share every launch.  Reports solves/s (64 per batch) for the
    mixed-precision and the plain FP64 paths (residual 1e-7) and their error
    against a tight FP64 solution; plain FP64 GMRES one right-hand side at a
    time; the oracle residual of two mixed solutions."""
    import torch
    from fmm3dbie_b200 import Plan
    from fmm3dbie_b200 import surface as S
    zk = 5.0
    zp = (zk, -1j * zk, 1.0)
    s = S.icosa_ellipsoid(3, 6, (1.0, 2.0, 3.0))
    t0 = time.time()
    st = S.setup(s, 1, EPS, zp)
    t_setup = time.time() - t0
    rng = np.random.default_rng(3)
    d = rng.normal(size=(64, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    rhs = -np.exp(1j * zk * (s.xyz @ d.T))
    P = Plan(1, zp, s, st.near, st.over)
    R = torch.tensor(np.ascontiguousarray(rhs), device=dev)
    w = torch.tensor(s.qwts(), device=dev)[:, None]
    xref, _ = P.solve(R, 0.5, mode=0, numit=300, eps_gmres=1e-12)
    xsol = {}

    def relerr(x):
        num = torch.sum(w * (x - xref).abs() ** 2, 0)
        den = torch.sum(w * xref.abs() ** 2, 0)
        return float(torch.max(torch.sqrt(num / den)))

    out = {"workload": "64 plane waves, ellipsoid (1,2,3), 1280 order-6 patches, "
                       "zk=5, zpars=(5,-5i,1), eps=1e-7", "nrhs": 64, "setup_s": round(t_setup, 2),
           "nptso": P.nptso}
    for mode, tag in ((1, "mixed"), (0, "fp64")):
        P.solve(R, 0.5, mode=mode, numit=300, eps_gmres=TOL_LOOSE)  # warm-up (tunes the kernels)
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            x, info = P.solve(R, 0.5, mode=mode, numit=300, eps_gmres=TOL_LOOSE)
            b.record()
            b.synchronize()
            ts.append(a.elapsed_time(b))
        t = float(np.mean(ts))
        xsol[tag] = x
        out[tag] = {"solves_per_s": 64 * 1000.0 / t, "ms_per_batch": t,
                    "max_niter": int(np.max(info["niter"])), "max_rel_err": relerr(x)}
    out["speedup_vs_fp64"] = out["fp64"]["ms_per_batch"] / out["mixed"]["ms_per_batch"]
    # the reference method proper: plain FP64 GMRES, one right-hand side at a time
    P.solve(R[:, 0].contiguous(), 0.5, mode=0, numit=300, eps_gmres=TOL_LOOSE)  # warm-up / tuning
    torch.cuda.synchronize()
    ts, its = [], []
    for q in range(2):
        r1 = R[:, q].contiguous()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        _, info = P.solve(r1, 0.5, mode=0, numit=300, eps_gmres=TOL_LOOSE)
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
        its.append(int(info["niter"][0]))
    out["fp64_single"] = {"solves_per_s": 1000.0 / float(np.mean(ts)), "ms_per_solve": float(np.mean(ts)),
                          "niter": its, "sample": "2 of the 64 systems, one at a time"}
    out["speedup_vs_fp64_single"] = out["mixed"]["solves_per_s"] / out["fp64_single"]["solves_per_s"]
    # stage times of one FP32 matvec of the 64 densities (CUDA events); the
    # oversampling stage against its bytes: sigma read (c128) and the
    # oversampled densities written (c64)
    P.matvec(R, 1)
    torch.cuda.synchronize()
    P.timing(True)
    P.matvec(R, 1)
    torch.cuda.synchronize()
    tm = P.timing(False)["f32"]
    ob = float(s.npts) * 64 * 16 + float(P.nptso) * 64 * 8
    out["fp32_matvec_nd64_ms"] = {"strengths": tm["strengths_ms"], "far": tm["far_ms"],
                                  "combine": tm["combine_ms"],
                                  "strengths_gbs": ob / (tm["strengths_ms"] * 1e-3) / 1e9,
                                  "strengths_bytes": ob}
    # the oversampling alone on each engine (CUDA cores, tensor cores), 64
    # densities, mean of 10 launches by CUDA events
    import ctypes as C
    from fmm3dbie_b200 import _lib as L
    osv = torch.empty((P.nptso, 64), dtype=torch.complex64, device=dev)
    eng = {}
    for e in (0, 1):
        args = (P._h, e, 64, C.c_void_p(R.data_ptr()), C.c_void_p(osv.data_ptr()), C.c_void_p(0))
        L.check(L.lib().bie_plan_oversample(*args), "bie_plan_oversample")
        a_ = torch.cuda.Event(enable_timing=True)
        b_ = torch.cuda.Event(enable_timing=True)
        a_.record()
        for _ in range(10):
            L.lib().bie_plan_oversample(*args)
        b_.record()
        b_.synchronize()
        ms = a_.elapsed_time(b_) / 10
        eng["cuda_cores" if e == 0 else "tensor_cores"] = {"ms": ms, "gbs": ob / (ms * 1e-3) / 1e9}
    out["oversample_nd64"] = eng
    # error against the oracle: residual of two mixed solutions under the
    # oracle's matvec on the same inputs
    xs = xsol["mixed"].cpu().numpy()
    out["oracle_residual_mixed"] = {str(q): oracle_residual(1, s, zp, st.near, st.over, rhs[:, q],
                                                            xs[:, q]) for q in (0, 63)}
    P.close()
    return out


WARMSTART_WEIGHTS = os.path.join(ROOT, "fmm3dbie_b200", "weights", "warmstart_torus.npz")


def torus_leg(dev, nd=16, weights=WARMSTART_WEIGHTS):
    """Plane-wave Helmholtz solves on the 64 x 32 quad torus
    (73,728 nodes) at two of the training grid's wavenumbers, 16 held-out
    directions each.  Times the plain FP64 GMRES path one right-hand side at
    a time (the reference method), the mixed-precision path on the batch of
    16 from zero, and the same from the trained network's guess."""
    import torch
    from fmm3dbie_b200.warmstart import (PlaneWaveProblem, WarmStartMLP, random_directions,
                                         torus_surface)
    if not os.path.exists(weights):
        return {"skipped": f"no trained network at {os.path.relpath(weights, ROOT)}"}
    z = np.load(weights)
    meta = json.loads(str(z["meta"]))
    ks_grid = meta["ks"]
    ks = [ks_grid[len(ks_grid) // 4], ks_grid[(3 * len(ks_grid)) // 4]]
    surf = torus_surface(*meta["surface"])
    t0 = time.time()
    prob = PlaneWaveProblem(surf, ks)
    t_setup = time.time() - t0
    mlp = WarmStartMLP.load(weights)
    hold = np.random.default_rng(int(meta["seed"]) + 1000)
    out = {"workload": "torus R=2, r=0.6+0.15cos3p, 64x32 quads, 6x6 nodes "
                       f"(npts {surf.npts}), plane waves, zpars=(k,-ik,1), eps=1e-7, "
                       f"{nd} held-out directions per k, tolerance {TOL_WARM:g}",
           "setup_s": round(t_setup, 1), "network": meta, "per_k": []}
    w = torch.tensor(surf.qwts(), device=dev)[:, None]
    tot = {"mixed_zero": 0.0, "mixed_warm": 0.0, "fp64_single": 0.0}
    n_single = 0
    for k in ks:
        dirs = random_directions(nd, hold)
        dirk = PlaneWaveProblem.dirk(k, dirs)
        xref, _ = prob.solve(k, dirs, mode=0, eps=1e-11)

        def relerr(x):
            return float(torch.max(torch.sqrt(torch.sum(w * (x - xref).abs() ** 2, 0) /
                                              torch.sum(w * xref.abs() ** 2, 0))))

        def timed(fn):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            r = fn()
            b.record()
            b.synchronize()
            return r, a.elapsed_time(b)

        prob.solve(k, dirs, mode=1, eps=TOL_WARM)  # warm-up (tunes the kernels)
        (xz, iz), mz = timed(lambda: prob.solve(k, dirs, mode=1, eps=TOL_WARM))
        (xw, iw), mw = timed(lambda: prob.solve(k, dirs, mode=1, eps=TOL_WARM,
                                                x0=mlp.predict_density(prob.srcvals, dirk)))
        x0 = mlp.predict_density(prob.srcvals, dirk)
        prob.solve(k, dirs[:1], mode=0, eps=TOL_WARM)  # warm-up / tuning of the nd=1 FP64 path
        pe = torch.sqrt(torch.sum(w * (x0 - xref).abs() ** 2, 0) / torch.sum(w * xref.abs() ** 2, 0))
        (x1, i1), m1 = timed(lambda: prob.solve(k, dirs[:1], mode=0, eps=TOL_WARM))
        tot["mixed_zero"] += mz
        tot["mixed_warm"] += mw
        tot["fp64_single"] += m1
        n_single += 1
        out["per_k"].append({
            "k": k, "pred_err_median": float(torch.median(pe)),
            "mixed_zero": {"ms": mz, "inner_iters_mean": float(iz["niter"].mean()),
                           "fp64_matvecs": iz["fp64_matvecs"], "max_rel_err": relerr(xz),
                           "max_rres": float(iz["rres"].max())},
            "mixed_warm": {"ms": mw, "inner_iters_mean": float(iw["niter"].mean()),
                           "fp64_matvecs": iw["fp64_matvecs"], "max_rel_err": relerr(xw),
                           "max_rres": float(iw["rres"].max()),
                           "x0_dropped": int(iw["x0_dropped"].sum())},
            "fp64_single": {"ms_per_solve": m1, "niter": int(i1["niter"][0]),
                            "rres": float(i1["rres"][0])}})
        if k == ks[-1]:
            # error against the oracle: one warm-started mixed solution's
            # residual under the oracle's matvec on the same inputs
            stk = prob.setups[k]
            x1 = xw[:, 0].cpu().numpy()
            b1 = -np.exp(1j * k * (surf.xyz @ dirs[0]))
            out["per_k"][-1]["oracle_residual_mixed_warm"] = oracle_residual(
                1, surf, (k, -1j * k, 1.0), stk.near, stk.over, b1, x1)
    n = nd * len(ks)
    out["solves_per_s"] = {"mixed_batched_warm": n * 1000.0 / tot["mixed_warm"],
                           "mixed_batched_zero": n * 1000.0 / tot["mixed_zero"],
                           "fp64_single": n_single * 1000.0 / tot["fp64_single"]}
    sp = out["solves_per_s"]
    out["speedup_vs_fp64_single"] = sp["mixed_batched_warm"] / sp["fp64_single"]
    out["warm_gain"] = sp["mixed_batched_warm"] / sp["mixed_batched_zero"]
    mlp.close()
    prob.close()
    return out


def uneven_leg(dev, kinds=(0, 1)):
    """32 ellipsoids (semi-axes U(0.5,3), 80/320/1280 patches, orders {4,6,8},
    zk U(1,6)), 4 interior point sources each, Laplace and Helmholtz batches.
    The graph engine runs every matvec stage of all surfaces as one
    persistent launch replayed from a CUDA graph (each surface's 4 systems
    share the launches); the streams engine solves each surface on its own
    stream.  Reports systems solved per second."""
    import torch
    from fmm3dbie_b200.batch import SurfaceBatch, uneven_ellipsoids
    from fmm3dbie_b200.surface import setup
    out = {"workload": "32 ellipsoids, npts 1200-57600, 4 point-source rhs each"}
    for kind in kinds:
        t0 = time.time()
        items, rhs, _ = uneven_ellipsoids(kind)
        setups = [setup(it.surf, it.kind, EPS, it.params) for it in items]
        t_setup = time.time() - t0
        R = [torch.tensor(np.ascontiguousarray(r), device=dev) for r in rhs]
        nsys = sum(r.shape[1] for r in rhs)
        res = {"setup_s": round(t_setup, 1), "npts_total": int(sum(it.surf.npts for it in items)),
               "systems": nsys}
        G = SurfaceBatch(items, EPS, engine="graph", setups=setups)
        sols = {}
        for mode, tag in ((1, "mixed"), (0, "fp64")):
            G.solve(R, mode=mode, eps_gmres=TOL_LOOSE)  # warm-up / tuning / graph capture
            sols[tag], infos, ms = G.solve(R, mode=mode, eps_gmres=TOL_LOOSE)
            res[tag] = {"solves_per_s": nsys * 1000.0 / ms, "ms": ms,
                        "max_rres": float(max(np.max(i["rres"]) for i in infos)),
                        "max_niter": int(max(np.max(i["niter"]) for i in infos))}
            if mode == 1:
                res[tag]["batch_matvecs_fp32_fp64"] = [infos[0]["fp32_matvecs"],
                                                       infos[0]["fp64_matvecs"]]
        info = G.info()
        res["far_variant_chunk_f32_nd1"] = [int(info[4]), int(info[5])]
        G.close()
        S = SurfaceBatch(items, EPS, engine="streams", setups=setups)
        S.solve(R, mode=1, eps_gmres=TOL_LOOSE)
        _, infos, ms = S.solve(R, mode=1, eps_gmres=TOL_LOOSE)
        res["mixed_streams"] = {"solves_per_s": nsys * 1000.0 / ms, "ms": ms,
                                "max_rres": float(max(np.max(i["rres"]) for i in infos))}
        S.close()
        res["speedup_vs_fp64"] = res["fp64"]["ms"] / res["mixed"]["ms"]
        # the reference method proper: plain FP64 GMRES one right-hand side
        # at a time (the first right-hand side of every surface)
        from fmm3dbie_b200 import Plan
        t_single, its = 0.0, []
        for q, it in enumerate(items):
            Pq = Plan(it.kind, it.params, it.surf, setups[q].near, setups[q].over)
            r1 = R[q][:, 0].contiguous()
            Pq.solve(r1, it.zid, mode=0, numit=300, eps_gmres=TOL_LOOSE)  # warm-up / tuning
            a_ = torch.cuda.Event(enable_timing=True)
            b_ = torch.cuda.Event(enable_timing=True)
            a_.record()
            _, i1 = Pq.solve(r1, it.zid, mode=0, numit=300, eps_gmres=TOL_LOOSE)
            b_.record()
            b_.synchronize()
            t_single += a_.elapsed_time(b_)
            its.append(int(i1["niter"][0]))
            Pq.close()
        res["fp64_single"] = {"solves_per_s": len(items) * 1000.0 / t_single,
                              "ms_total": t_single, "max_niter": max(its),
                              "sample": f"the first right-hand side of each of the {len(items)} "
                                        "surfaces, one at a time"}
        best = max(res["mixed"]["solves_per_s"], res["mixed_streams"]["solves_per_s"])
        res["speedup_vs_fp64_single"] = best / res["fp64_single"]["solves_per_s"]
        # error against the oracle on the largest surface (first system)
        qbig = int(np.argmax([it.surf.npts for it in items]))
        it = items[qbig]
        res["oracle_residual_mixed_largest_surface"] = oracle_residual(
            kind, it.surf, it.params, setups[qbig].near, setups[qbig].over,
            rhs[qbig][:, 0], sols["mixed"][qbig][:, 0].cpu().numpy(), zid=it.zid)
        out["laplace" if kind == 0 else "helmholtz"] = res
    return out


def nearquad_only(nref):
    """Device near-quadrature generator alone (two calls; the second is
    reported), for profiling."""
    from fmm3dbie_b200 import surface as S
    s = S.icosa_ellipsoid(nref, 6, (1.0, 2.0, 3.0))
    targs = s.srcvals
    ipatch_id, uvs = s.patch_id_uvs()
    rfac, rfac0 = S.get_rfacs(6, 1)
    cms, rads = S.get_centroid_rads(s)
    row_ptr, col_ind = S.findnear(cms, rads * rfac, targs)
    iquad = S.get_iquad_rsc(s, row_ptr, col_ind)
    gs = np.zeros(4, np.int64)
    for _ in range(2):
        t0 = time.time()
        S.getnearquad(s, 1, EPS, ZPARS, targs, ipatch_id, uvs, row_ptr, col_ind, iquad, rfac0,
                      engine="gpu", stats=gs)
        dt = time.time() - t0
    print(json.dumps({"nearquad": {"npts": s.npts, "pairs": int(gs[1] + gs[2]),
                                   "self_pairs": int(gs[1]), "kernel_evals": int(gs[0]),
                                   "device_kernel_ms": gs[3] / 1e3, "call_s": round(dt, 4),
                                   "gevals_per_s": float(gs[0]) / (gs[3] * 1e3)}}))
    return 0


def matvec_only(args):
    import torch
    from fmm3dbie_b200 import Plan
    s, st, rhs, _ = build_problem()
    P = Plan(1, ZPARS, s, st.near, st.over)
    r = torch.tensor(rhs, device="cuda")
    if args.nd > 1:
        r = r[:, None].repeat(1, args.nd).contiguous()
    for _ in range(args.matvec_only):
        P.matvec(r, args.prec)
    torch.cuda.synchronize()
    t = P.timing(True)
    P.matvec(r, args.prec)
    torch.cuda.synchronize()
    t = P.timing(False)
    print(json.dumps({"matvec_prec": args.prec, "stage_ms": t}))
    return 0


def tree_leg(nref, norder=6, solve=True):
    """Hierarchical against direct far field on a large ellipsoid (1,2,3):
    icosahedron refined nref times, order norder, Helmholtz k = 2 (zpars
    (2, -2i, 1)), eps 1e-7, device setup.  Per precision: far-stage time of
    one matvec (CUDA events) with each method, the tree's kernel
    evaluations, and the tree matvec's weighted relative L2 difference from
    the direct FP64 matvec; then the mixed-precision solve with each method
    (the FP32 inner and FP64 outer matvecs both on the tree) and the
    difference of the two solutions."""
    import torch
    from fmm3dbie_b200 import Plan
    from fmm3dbie_b200 import surface as S
    s = S.icosa_ellipsoid(nref, norder, (1.0, 2.0, 3.0))
    t0 = time.time()
    st = S.setup(s, 1, EPS, ZPARS)
    t_setup = time.time() - t0
    r = np.linalg.norm(s.xyz - X0, axis=1)
    rhs = torch.tensor(np.exp(1j * ZK * r) / (4 * np.pi * r), device="cuda")
    t0 = time.time()
    P = Plan(1, ZPARS, s, st.near, st.over)
    t_plan = time.time() - t0
    w = torch.tensor(s.qwts(), device="cuda")

    def rel(a, b):
        ww = w if a.dim() == 1 else w[:, None]
        return float(torch.sqrt((ww * (a - b).abs() ** 2).sum() / (ww * b.abs() ** 2).sum()))

    def far_ms(prec, reps=3):
        P.matvec(rhs, prec)
        torch.cuda.synchronize()
        P.timing(True)
        for _ in range(reps):
            P.matvec(rhs, prec)
        torch.cuda.synchronize()
        t = P.timing(False)
        k = "f32" if prec == 1 else "f64"
        return t[k]["far_ms"] / reps, (t[k]["strengths_ms"] + t[k]["combine_ms"]) / reps

    out = {"workload": f"ellipsoid (1,2,3), {20 * 4 ** nref} order-{norder} patches, zk=2, "
                       f"zpars=(2,-2i,1), eps=1e-7",
           "npts": s.npts, "nptso": P.nptso, "pairs": float(s.npts) * P.nptso,
           "setup_s": round(t_setup, 2), "plan_s": round(t_plan, 2)}
    P.set_far_method(0, 0)
    y_ref = P.matvec(rhs, 0)
    for prec in (0, 1):
        k = "f32" if prec == 1 else "f64"
        P.set_far_method(prec, 0)
        d_far, d_rest = far_ms(prec)
        yd = P.matvec(rhs, prec)
        t0 = time.time()
        P.set_far_method(prec, 1)
        t_build = time.time() - t0
        info = P.get_far_method(prec)
        t_far, t_rest = far_ms(prec)
        yt = P.matvec(rhs, prec)
        out[k] = {"direct_far_ms": d_far, "tree_far_ms": t_far, "other_stages_ms": t_rest,
                  "speedup": d_far / t_far, "tree_build_s": round(t_build, 3),
                  "tree_p": info["p"], "tree_theta": info["theta"],
                  "tree_kernel_evals": info["kernel_evals"],
                  "tree_updown_terms": info["updown_terms"],
                  "evals_frac_of_direct": info["kernel_evals"] / (float(s.npts) * P.nptso),
                  "forms_pp_pc_cp_cc": [int(info["pp"] + info["pp_check"]), int(info["pc"]),
                                        int(info["cp"]), int(info["cc"])],
                  "tree_vs_direct_f64": rel(yt, y_ref), "direct_vs_direct_f64": rel(yd, y_ref)}
    # 16 densities at once (FP32): the direct multi-density kernels (their
    # autotuned shape) against the multi-density tree kernel
    nd = 16
    xm = (rhs[:, None] * torch.arange(1, nd + 1, device="cuda")).contiguous()
    md = {}
    for method in (0, 1):
        P.set_far_method(1, method)
        ym = P.matvec(xm, 1)
        torch.cuda.synchronize()
        P.timing(True)
        P.matvec(xm, 1)
        torch.cuda.synchronize()
        md[method] = (P.timing(False)["f32"]["far_ms"], ym)
    out["f32_nd16"] = {"direct_far_ms": md[0][0], "tree_far_ms": md[1][0],
                       "speedup": md[0][0] / md[1][0],
                       "tree_vs_direct": rel(md[1][1], md[0][1])}
    if solve:
        res = {}
        for method in (0, 1):
            P.set_far_method(0, method)
            P.set_far_method(1, method)
            P.solve(rhs, 0.5, mode=1, numit=200, eps_gmres=1e-7)  # warm (autotune)
            torch.cuda.synchronize()
            t0 = time.time()
            x, inf = P.solve(rhs, 0.5, mode=1, numit=200, eps_gmres=1e-7)
            torch.cuda.synchronize()
            res[method] = (time.time() - t0, x, inf)
        out["mixed_solve"] = {"direct_s": res[0][0], "tree_s": res[1][0],
                              "speedup": res[0][0] / res[1][0],
                              "tree_vs_direct_solution": rel(res[1][1], res[0][1]),
                              "rres_direct": float(res[0][2]["rres"][0]),
                              "rres_tree": float(res[1][2]["rres"][0])}
    P.close()
    return out


def ctypes_double_pair(lib):
    import ctypes as C
    tf, ms = C.c_double(), C.c_double()
    lib.bie_measure_fp32_peak(C.byref(tf), C.byref(ms))
    return tf.value


def mufu_peak(lib):
    """Measured MUFU throughput in G ops/s (rsqrt.approx loop)."""
    import ctypes as C
    g, ms = C.c_double(), C.c_double()
    lib.bie_measure_mufu_peak(C.byref(g), C.byref(ms))
    return g.value


MUFU_PER_PAIR = {"helm": 3, "lap": 1}   # rsqrt, sin, cos (Helmholtz); rsqrt (Laplace)


if __name__ == "__main__":
    sys.exit(main())
