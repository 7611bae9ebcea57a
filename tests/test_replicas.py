"""Replica (multi-GPU) bookkeeping of bench.py on CPU: two gloo ranks, each with
its own solve time, agree on the slowest rank's time and on the whole-job rate
(converged states x world size / slowest time per solve)."""
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
        tsum = 3.0 + rank  # rank 1 is the slower replica: 4 s for 2 solves
        rate, per_solve = bench.replica_rate(288, tsum, 2, world, dist, "cpu")
        out[rank] = (rate, per_solve, bench.max_over_ranks(10.0 * rank, dist, "cpu"))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_slowest_replica():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        rate, per_solve, mx = res[rank]
        assert per_solve == pytest.approx(2.0)
        assert rate == pytest.approx(288 * 2 / 2.0)
        assert mx == pytest.approx(10.0)


def test_single_process_rate():
    import bench
    rate, per_solve = bench.replica_rate(288, 1.5, 3, 1, None, "cpu")
    assert per_solve == pytest.approx(0.5) and rate == pytest.approx(576.0)
