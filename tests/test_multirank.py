"""The N > 1 path of bench.py on CPU: two gloo ranks, each advancing its own
replica (the reference path does not shard one simulation), a barrier
around the timed region, and the whole-job rate from the slowest rank.

Each rank steps the oracle on the same inputs, so the replicas must agree
bit for bit; rank 1 is made slower on purpose and the aggregate must follow
it.
"""
import os
import sys
import time

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "grasph.jl_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import datetime
    import bench
    import grasph_b200 as G
    from grasph_b200 import scenarios
    from pyoracle import OracleBackend
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        lf, meta = scenarios.dambreak_2d(nx=10, ny=20, dx=0.1, tank=(2.0, 2.5))
        s = G.Session([lf], backend=OracleBackend(threads=1))
        s.push()
        dist.barrier()
        t0 = time.perf_counter()
        s.step(3, meta["cfl"])
        if rank == 1:
            time.sleep(0.3)
        local = time.perf_counter() - t0
        dist.barrier()
        slowest = bench.max_over_ranks(local, dist, device="cpu")
        s.pull()
        out[rank] = (local, slowest, bench.job_rate(meta["n_fluid"], 3, slowest, world),
                     np.asarray(lf.systems[0].x).tobytes())
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_and_aggregate():
    world = 2
    port = 29500 + (os.getpid() % 1000)
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    (l0, s0, r0, x0), (l1, s1, r1, x1) = res[0], res[1]
    assert x0 == x1, "replicas on identical inputs must agree"
    assert s0 == s1 == pytest.approx(max(l0, l1))
    assert l1 >= 0.3 and s0 >= l1
    assert r0 == r1
    assert r0 == pytest.approx(200 * 3 * world / s0)
