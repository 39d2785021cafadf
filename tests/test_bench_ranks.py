"""The multi-rank path of bench.py on the CPU (gloo, world size 2): every
rank draws its own seeded points, the job time is the maximum over ranks,
and the job throughput counts all ranks' points over that time."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        import bench
        _, f = bench.make_inputs(rank)
        ms = bench.max_over_ranks(torch, dist, 10.0 + 5.0 * rank, world, 'cpu')
        out[rank] = (float(np.sum(f[:, :64])), ms,
                     bench.job_rate(24, world, ms))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_points_and_take_the_slowest_time():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    (s0, ms0, r0), (s1, ms1, r1) = res[0], res[1]
    assert s0 != s1                       # different seeded points per rank
    assert ms0 == ms1 == 15.0             # the slowest rank's time
    assert r0 == r1 == pytest.approx(48 / 15e-3)
