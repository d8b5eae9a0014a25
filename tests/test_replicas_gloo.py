"""bench.py --gpus N runs N independent replicas: each rank solves its own
copy, the timed region is closed by a barrier, and rank 0 reports
N * steps / max_rank_time.  This exercises that host logic with the gloo
backend on CPU (world_size 2): every rank applies the FP64 oracle operator to
its own density (the CPU stand-in for a replica's solve) and the ranks
reduce the maximum time."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import time

    import torch

    import bench
    import oracle
    from fmm3dbie_b200 import surface as S

    dist.init_process_group("gloo", rank=rank, world_size=world)
    s = S.icosa_sphere(1, 3)
    st = S.setup(s, 0, 1e-6, (1.0, 1.0))
    rng = np.random.default_rng(rank)
    dist.barrier()
    t0 = time.perf_counter()
    steps = 2
    for _ in range(steps):
        pot = oracle.lpcomp(0, s, (1.0, 1.0), st.near, st.over, rng.normal(size=s.npts))
    t = torch.tensor([time.perf_counter() - t0], dtype=torch.float64)
    dist.barrier()
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    assert bench.env_rank() == (rank, world, 0)
    out[rank] = (float(t.item()), float(tmax.item()), world * steps / float(tmax.item()),
                 bool(np.all(np.isfinite(pot))))
    dist.destroy_process_group()


def test_two_replicas_gloo(built):
    mp_ctx = mp.get_context("spawn")
    with mp_ctx.Manager() as m:
        out = m.dict()
        port = 29500 + (os.getpid() % 2000)
        procs = [mp_ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        res = dict(out)
    assert set(res) == {0, 1}
    tmax = max(res[0][0], res[1][0])
    for r in (0, 1):
        assert res[r][1] == pytest.approx(tmax)
        assert res[r][2] == pytest.approx(2 * 2 / tmax)
        assert res[r][3]
