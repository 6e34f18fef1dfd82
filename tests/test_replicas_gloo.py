"""The N>1 path of bench.py (independent replicas, no collective in the step) with
world_size 2 over gloo on the CPU: the job time is the max over ranks, the throughput
counts every rank's cells, and every replica gets its own seed."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms_local = 10.0 + 5.0 * rank             # rank 1 is the slow one
    ms, value = bench.aggregate(ms_local, cells=1000, steps=4, world=world, dist=dist, device="cpu")
    out[rank] = (ms, value, bench.replica_seed(rank))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregation_world2():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert out[0][0] == pytest.approx(15.0) and out[1][0] == pytest.approx(15.0)
    assert out[0][1] == pytest.approx(1000 * 4 * 2 / 0.015)
    assert out[0][2] != out[1][2]


def _failing_worker(rank, world, port):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        raise RuntimeError("replica 1 fails before its step")
    bench.aggregate(10.0, cells=1000, steps=4, world=world, dist=dist, device="cpu")
    dist.destroy_process_group()


def test_failing_replica_is_reported():
    """A rank that raises between steps ends the job with an error on the host: the
    launcher reports it and stops the other rank, which would otherwise wait in its
    collective until the process-group timeout."""
    world = 2
    port = _free_port()
    with pytest.raises(mp.ProcessRaisedException, match="replica 1 fails"):
        mp.start_processes(_failing_worker, args=(world, port), nprocs=world, start_method="spawn", join=True)
