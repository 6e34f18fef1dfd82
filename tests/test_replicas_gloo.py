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


def _shard_worker(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "2_b200"))
    import datetime
    import numpy as np
    import torch.distributed as dist
    from mumax2 import workloads as W
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    classes, (lo, hi) = W.ensemble_shard(2048, seed=0, rank=rank, world=world)
    ids = np.concatenate([c["ids"] for c in classes])
    cells = sum(len(c["ids"]) * int(np.prod(c["n"])) for c in classes)
    # a stand-in per-simulation result: <m> of its initial direction
    rows = np.concatenate([np.asarray(c["m0"]) for c in classes])
    g = W.gather_per_sim(dist, ids, rows, 2048)
    out[rank] = (lo, hi, int(cells), None if g is None else g.tolist())
    dist.barrier()
    dist.destroy_process_group()


def test_ensemble_sharded_over_ranks_and_gathered_world2():
    """N > 1 ensemble: each rank takes a contiguous, cell-balanced block of the same 2048
    simulations (no collective while stepping), and the per-simulation results come
    back to rank 0 in simulation order with one all-gather."""
    import sys
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "2_b200"))
    from mumax2 import workloads as W
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_shard_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    (lo0, hi0, c0, g0), (lo1, hi1, c1, g1) = out[0], out[1]
    assert lo0 == 0 and hi0 == lo1 and hi1 == 2048
    assert abs(c0 - c1) / (c0 + c1) < 0.05            # balanced by cells
    assert g1 is None
    full = W.ensemble(2048, seed=0)
    want = np.zeros((2048, 3))
    for c in full:
        want[c["ids"]] = np.asarray(c["m0"])
    assert np.array_equal(np.asarray(g0), want)


def test_partition_is_contiguous_and_balanced():
    from mumax2 import workloads as W
    w = [1, 1, 1, 10, 1, 1, 1, 1, 10, 1]
    parts = W.partition(w, 3)
    assert parts[0][0] == 0 and parts[-1][1] == len(w)
    assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
    assert W.partition(w, 1) == [(0, len(w))]
