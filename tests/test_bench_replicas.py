"""The replicas path of bench.py (N > 1: independent routes, one per GPU) on CPU:
two gloo ranks with different step times agree on the slowest time and on the
whole-job throughput."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 100.0 * (rank + 1)  # rank 1 is the slow replica
    t = bench.max_over_ranks(ms, dist, "cpu")
    out[rank] = (t, bench.replica_throughput(1000, 2, world, t))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1] == (200.0, 1000 * 2 * 2 / 0.2)


def test_single_rank_needs_no_collective():
    assert bench.max_over_ranks(12.5, None) == 12.5
    assert bench.replica_throughput(130000, 3, 1, 30.0) == 130000 * 3 / 0.03
