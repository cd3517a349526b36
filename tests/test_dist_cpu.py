"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): the
max-over-ranks timing, the sums of whole-job counts, the barrier, the
partition of independent candidates across ranks, and that only rank 0 runs
the reference arm."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = {}
        bench.barrier(dist)
        out["max"] = bench.allmax(dist, 1.5 + rank)
        out["sum"] = bench.allsum(dist, 1.5 + rank)
        mine = bench.shard(list(range(11)), rank, world)
        parts = [None] * world
        dist.all_gather_object(parts, mine)
        out["parts"] = parts
        out["ref"] = bench.run_reference(None, world, rank, dist) if rank != 0 else "skipped"
        bench.barrier(dist)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_and_partition():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        assert res[r]["max"] == 2.5
        assert res[r]["sum"] == 4.0
        parts = res[r]["parts"]
        assert sorted(parts[0] + parts[1]) == list(range(11))
        assert not set(parts[0]) & set(parts[1])
    assert res[1]["ref"] is None          # only rank 0 runs the reference arm
