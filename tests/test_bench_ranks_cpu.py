"""bench.py's multi-GPU arithmetic on two gloo ranks (CPU): N independent replicas,
the whole-job value is the units of all ranks over the slowest rank's time, and
every rank computes the same numbers (rank 0 prints them)."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, ws, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        ms_local = 1.0 + rank          # rank 1 is the slow one
        value, ms = bench.replica_throughput(3.0e9, ms_local, ws, device="cpu")
        mx = bench.reduce_max(10.0 * rank, ws, device="cpu")
        bench.barrier(ws)
        out[rank] = (value, ms, mx)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_ranks():
    ws, port = 2, 29000 + os.getpid() % 1000
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    for r in range(ws):
        value, ms, mx = res[r]
        assert ms == 2.0                                  # the slowest rank's time
        assert value == pytest.approx(3.0e9 * ws / 2.0e-3)  # all ranks' units over it
        assert mx == 10.0
