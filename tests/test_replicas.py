"""The multi-GPU form is replicas only: each rank verifies its own batch and
the only collectives are the timing barrier and the max-over-ranks of the
elapsed time.  That host logic runs here on CPU with the gloo backend,
world size 2."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = 1.5 if rank == 0 else 4.0  # rank 1 is the slow one
        dist.barrier()
        t = bench.max_over_ranks(local, world, "cpu")
        out[rank] = (t, bench.replica_rate(4096, world, 10, t))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 4.0
    assert res[0][1] == pytest.approx(4096 * 2 * 10 / 4.0)


def test_single_rank_is_local():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(2.5, 1, "cpu") == 2.5
    assert bench.replica_rate(100, 1, 4, 2.0) == 200
