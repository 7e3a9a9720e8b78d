"""Multi-GPU is replicas only: each rank runs its own simulation and bench.py
reduces the ranks' times (max) and work (sum) into one whole-job
throughput.  This checks that reduction with two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r: (r + 1) * 10 ms for (r + 1) * 1000 particle-steps
        value, ms_max = bench.reduce_replicas(10.0 * (rank + 1), 1000.0 * (rank + 1), world, "cpu")
        out[rank] = (value, ms_max)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_is_summed_work_over_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    for value, ms_max in res.values():
        assert ms_max == pytest.approx(20.0)
        assert value == pytest.approx(3000.0 / 0.020)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    value, ms_max = bench.reduce_replicas(4.0, 2000.0, 1, "cpu")
    assert ms_max == 4.0 and value == pytest.approx(5e5)
