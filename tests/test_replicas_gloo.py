"""The bench's multi-GPU path (replicas: no data-path collective, one barrier-bracketed timing
reduced to the slowest rank) exercised with world_size 2 on the gloo backend, on the CPU."""
from __future__ import annotations

import os
import socket

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank: int, world: int, port: int, out):
    import sys

    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    import bench
    from pbrt_b200 import workloads as W

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each rank's own replica input
        v, f = W.displaced_icosphere(2, seed=1)
        rays = W.incoherent_rays(1024, v.min(0), v.max(0), seed=bench.rank_ray_seed(rank))
        dist.barrier()
        local_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        slowest = bench.max_over_ranks(local_ms, dist, torch.device("cpu"))
        rate = bench.whole_job_rate(world, rays.shape[1], slowest * 1e-3)
        dist.barrier()
        out[rank] = (slowest, rate, float(rays[0, :8].sum()))
    finally:
        dist.destroy_process_group()


def test_replica_timing_reduces_to_the_slowest_rank():
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0  # max over ranks
    assert res[0][1] == res[1][1] == 2 * 1024 / 0.015  # whole-job rays/s at the slowest time
    assert res[0][2] != res[1][2]  # the ranks trace different rays


def test_single_process_helpers():
    import sys

    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, None) == 3.5
    assert bench.whole_job_rate(1, 100, 0.5) == 200.0
    assert bench.rank_ray_seed(0) != bench.rank_ray_seed(1)
    assert np.isfinite(bench.whole_job_rate(8, 1 << 24, 1e-3))
