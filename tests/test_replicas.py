"""Replica plumbing of bench.py on CPU: two ranks over gloo (world size 2) agree on the maximum
of their timings (the job's time is the slowest rank's) and pass the barrier; no GPU and no data
path collective are involved (the path runs as independent replicas)."""
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
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    r, w, _ = bench.dist_init(world)
    assert (r, w) == (rank, world)
    bench.dist_barrier(w)
    out[rank] = bench.dist_max(1.5 + rank, w)
    bench.dist_barrier(w)
    import torch.distributed as dist
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_ranks_max_over_ranks():
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        assert dict(out) == {0: 2.5, 1: 2.5}
