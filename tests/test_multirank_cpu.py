"""The several-GPU form of bench.py runs independent replicas (the path has no
data exchange between solves) and reports the slowest rank.  This exercises
that host logic with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = [10.0 + rank, 20.0 - rank]  # rank 1 is slower in the first timing
        t, e = bench.max_over_ranks(local, dist)
        out[rank] = (t, e, bench.job_throughput(1000, 5, world, t))
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_is_max_over_ranks():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1]
    t, e, v = res[0]
    assert t == 11.0 and e == 20.0
    assert v == pytest.approx(2 * 1000 * 5 / 0.011)
