"""The multi-rank plumbing of bench.py, on CPU with two gloo ranks: the path
runs as independent replicas (no collective on the data path), and timings
are reduced to the slowest rank's before rank 0 reports."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    w, r, local = bench.dist_setup()
    dist.init_process_group("gloo", rank=r, world_size=w)
    out[rank] = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 3.0], "cpu") + [w, r, local]
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_report_the_slowest():
    world = 2
    with mp.get_context("spawn").Manager() as m:  # a forked manager could inherit held locks
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        assert res[rank][:3] == [2.0, 10.0, 3.0]
        assert res[rank][3:] == [world, rank, rank]
