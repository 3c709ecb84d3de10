"""The replica path of bench.py on CPU with the gloo backend, world size 2:
every rank runs its own lattice, the timed region is the slowest rank's, and
the whole-job value counts every rank's node updates."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank                  # rank 1 is the slowest
        slowest = bench.max_over_ranks(ms, world, "cpu")
        value = bench.replica_value(1_000_000, 20, world, slowest)
        out[rank] = (slowest, value)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_slowest_rank_and_total_updates():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    slowest, value = res[0]
    assert slowest == pytest.approx(15.0)
    # 2 replicas x 1e6 nodes x 20 steps in 15 ms
    assert value == pytest.approx(2 * 1e6 * 20 / 15e-3 / 1e6)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.0, 1) == 3.0
    assert bench.replica_value(100, 10, 1, 1.0) == pytest.approx(100 * 10 / 1e-3 / 1e6)
