"""Multi-process plumbing of the replica / instance-shard runs, on CPU ranks.

Two gloo ranks deal a problem set round robin and reduce timings and counts
exactly as bench.py does on GPUs (max of times, sum of counts); the
surrogate's data-parallel training pieces (flat all-reduce of several
tensors, the output statistics of the sharded training set, equal batch
counts per rank) give what one process gives on the whole set.
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


def _dataset(n=7, C=12, G=40, seed=5):
    import numpy as np

    rng = np.random.default_rng(seed)
    t = rng.normal(0.0, 1.0, (n, C, G)) * rng.uniform(0.1, 3.0, (1, C, 1))
    m = (rng.random((n, G)) > 0.3).astype(float)
    return t, m


def _worker_train(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import numpy as np
    import torch

    from curved_lbm import replicas, warmstart

    w, r, _ = replicas.init(backend="gloo", timeout_s=60.0)
    a = torch.tensor([r + 1.0, 2.0], dtype=torch.float32)
    b = torch.full((2, 2), 10.0 * r, dtype=torch.float32)
    replicas.allreduce_([a, b])
    c = torch.tensor([float(r), 7.0 - r], dtype=torch.float64)
    replicas.allreduce_([c], op="max")
    t, m = _dataset()
    idx = replicas.deal(range(len(t)), r, w)
    scale = warmstart.output_scale(t[idx], m[idx], "cpu")

    class _Net:
        B = 4

    sur = warmstart.Surrogate.__new__(warmstart.Surrogate)
    sur.net = _Net()
    n_max = torch.tensor([float(len(idx))], dtype=torch.float64)
    replicas.allreduce_([n_max], op="max")
    nb = len(sur._batches(list(idx), np.random.default_rng(r), int(n_max.item())))
    out[rank] = (a.tolist(), b.tolist(), c.tolist(), scale.tolist(), nb)
    replicas.finalize()


def test_two_gloo_ranks_train_pieces_match_one_process():
    import numpy as np
    import torch.multiprocessing as mp

    from curved_lbm import warmstart

    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker_train, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    t, m = _dataset()
    whole = warmstart.output_scale(t, m, "cpu")
    for r in (0, 1):
        a, b, c, scale, nb = res[r]
        assert a == [3.0, 4.0] and b == [[10.0, 10.0], [10.0, 10.0]]
        assert c == [1.0, 7.0]
        np.testing.assert_allclose(scale, whole, rtol=1e-6)
        assert nb == 1  # 4 and 3 cases: both ranks draw one batch of 4

