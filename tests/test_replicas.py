"""Multi-GPU replicas (no data-path collective): the timing reduction every rank
runs and the whole-job throughput, exercised with world_size 2 over gloo on CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    try:
        ms = bench.max_over_ranks(times[rank], world, torch.device("cpu"))
        out[rank] = (ms, bench.replica_throughput(world, 160, ms))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("times", [(12.5, 20.0), (30.0, 7.0)])
def test_max_over_ranks_and_throughput_gloo(times):
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), times, out), nprocs=world, join=True)
        res = dict(out)
    slowest = max(times)
    for r in range(world):
        ms, thr = res[r]
        assert ms == slowest
        assert thr == pytest.approx(world * 160 / (slowest / 1e3))


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, 1, None) == 3.5
    assert bench.replica_throughput(1, 10, 1000.0) == pytest.approx(10.0)
