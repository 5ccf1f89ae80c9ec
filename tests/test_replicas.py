"""Multi-process plumbing of the replica / instance-shard runs, on CPU ranks.

Two gloo ranks deal a problem set round robin and reduce timings and counts
exactly as bench.py does on GPUs (max of times, sum of counts).
"""

from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from curved_lbm import replicas

    w, r, _ = replicas.init(backend="gloo", timeout_s=60.0)
    mine = replicas.deal(range(10), r, w)
    times, counts = replicas.reduce_times_and_counts([1.0 + r, 5.0 - r], [len(mine), sum(mine)])
    out[rank] = (mine, times, counts)
    replicas.finalize()


def test_deal_is_a_partition():
    from curved_lbm import replicas

    parts = [replicas.deal(range(11), r, 3) for r in range(3)]
    assert sorted(x for p in parts for x in p) == list(range(11))
    assert [len(p) for p in parts] == [4, 4, 3]


def test_two_gloo_ranks_reduce_like_the_bench():
    import torch.multiprocessing as mp

    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0][0] == [0, 2, 4, 6, 8] and res[1][0] == [1, 3, 5, 7, 9]
    for r in (0, 1):
        assert res[r][1] == [2.0, 5.0]           # max over ranks
        assert res[r][2] == [10.0, 45.0]         # sum over ranks
