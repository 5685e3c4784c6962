"""Replica plumbing of bench.py on CPU ranks (gloo, world size 2): the
replica assignment covers every item exactly once and the timing reduction
takes the maximum over ranks.  No GPU is involved."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        mine = bench.shard(list(range(11)), ws, rank)
        bench.barrier(ws)
        t = bench.max_over_ranks(1.5 + rank, ws)
        q.put((rank, mine, t, bench._dist()))
    finally:
        dist.destroy_process_group()


def test_replicas_and_max_over_ranks_gloo():
    import torch.multiprocessing as mp

    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    items = sorted(x for _, mine, _, _ in out for x in mine)
    assert items == list(range(11))
    assert all(t == 2.5 for _, _, t, _ in out)
    assert [d for _, _, _, d in out] == [(2, 0, 0), (2, 1, 1)]


def test_single_rank_defaults(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench._dist() == (1, 0, 0)
    assert bench.max_over_ranks(3.25, 1) == 3.25
    assert bench.shard([1, 2, 3], 1, 0) == [1, 2, 3]
