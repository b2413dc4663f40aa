"""Replica mode of bench.py on CPU with the gloo backend, world size 2:
max-over-ranks timing, summed throughput, one barrier pair per timed region,
distinct seeds per rank."""
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


def _worker(rank, ws, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    from pic_b200 import deck
    dist, r, w = bench._dist()
    try:
        t = 10.0 + rank               # per-rank "device time"
        mx = bench._max_over_ranks(dist, t)
        tot = bench._sum_over_ranks(dist, 100.0 * (rank + 1))
        seed = deck.config("tiny").seed + 1000 * r
        bench._barrier(dist)
        q.put((r, w, mx, tot, seed))
    finally:
        dist.destroy_process_group()


def test_replica_reductions_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2, 2]
    assert all(o[2] == 11.0 for o in out)       # slowest rank's time
    assert all(o[3] == 300.0 for o in out)      # whole-job work
    assert out[0][4] != out[1][4]               # independent replicas
