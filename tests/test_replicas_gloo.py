"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): replicas get
distinct seeds, the timed region is the maximum over ranks, and the reported
throughput is the whole job's."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    elapsed = 2.0 + rank  # the second replica is slower
    dist.barrier()
    t, value = bench.aggregate_over_ranks(elapsed, trajectories_per_rank=4, world=world, dist=dist)
    out[rank] = (t, value, bench.replica_seed(1234, rank))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_gloo():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    t0, v0, s0 = out[0]
    t1, v1, s1 = out[1]
    assert t0 == t1 == 3.0                      # max over ranks
    assert v0 == v1 == pytest.approx(3600.0 * 4 * 2 / 3.0)
    assert s0 != s1                             # independent chains


def test_single_rank_needs_no_process_group():
    import bench
    t, v = bench.aggregate_over_ranks(2.0, 3, 1)
    assert t == 2.0 and v == pytest.approx(3600.0 * 3 / 2.0)
