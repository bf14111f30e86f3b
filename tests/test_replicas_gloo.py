"""The multi-GPU arm of bench.py runs N independent replicas (the path does
not shard): each rank times its own steps, the job time is the slowest
rank's, and the value is all ranks' cell updates over that time. This
checks that logic with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms_local = 100.0 + 50.0 * rank  # rank 1 is the slow one
    ms = bench.max_over_ranks(ms_local, dist, "cpu")
    out[rank] = (ms, bench.replica_value(1000, world, 10, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_takes_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ms, value = res[r]
        assert ms == 150.0
        assert value == pytest.approx(2 * 1000 * 10 / 0.150)
