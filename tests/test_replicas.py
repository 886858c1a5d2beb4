"""Multi-process plumbing of bench.py --gpus N (replicas: no data-path collective;
the only exchange is the maximum of the timings over the ranks), run as two
gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        vals = [1.0 + rank, 5.0 - rank, 2.5, 7.0 * (rank + 1)]
        out[rank] = bench.max_over_ranks(vals, world, "cpu")
    finally:
        dist.destroy_process_group()


def test_timings_are_the_maximum_over_two_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        assert out[0] == out[1] == [2.0, 5.0, 2.5, 14.0]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3, 4.5], 1, "cpu") == [3.0, 4.5]
