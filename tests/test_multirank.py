"""Multi-process path of bench.py on CPU: two gloo ranks reduce their
per-rank timings and work counts the way the GPU ranks do (max of the
device time, sums of the edge steps), and every rank checks its own seeded
replica of the workload."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        mx, sm = bench.reduce_over_ranks([1.5 + rank, -rank], [10.0 * (rank + 1), 1.0])
        (only,), empty = bench.reduce_over_ranks([0.25 * rank], [])
        out.put((rank, mx, sm, only, empty, bench.replica_seed(3, rank)))
    finally:
        dist.destroy_process_group()


def test_reduce_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, mx, sm, only, empty, seed in res:
        assert mx == [2.5, 0.0]
        assert sm == [30.0, 2.0]
        assert only == 0.25
        assert empty == []
    assert res[0][5] != res[1][5]


def test_reduce_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks([3.0], [4, 5]) == ([3.0], [4.0, 5.0])
