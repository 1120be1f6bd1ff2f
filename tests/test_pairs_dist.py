"""Pair-parallel scheduling on CPU: assignment properties and a world_size-2 gloo run."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from skmimageregistration_b200.pairs import assign_pairs, imbalance, pair_cost, run_pairs


def _sizes(n=64, seed=0):
    rng = np.random.default_rng(seed)
    lo, hi = np.array([64, 64, 64]), np.array([160, 160, 128])
    return [tuple(int(v) for v in rng.integers(lo, hi + 1)) for _ in range(n)]


def test_assignment_covers_every_pair_once_and_balances():
    costs = [pair_cost(s) for s in _sizes()]
    for world in (1, 2, 4, 8):
        a = assign_pairs(costs, world)
        flat = sorted(i for part in a for i in part)
        assert flat == list(range(len(costs)))
        assert imbalance(costs, a) < 1.15
        assert a == assign_pairs(costs, world)          # deterministic


def test_assignment_more_ranks_than_pairs():
    a = assign_pairs([5.0, 3.0], 4)
    assert sorted(i for p in a for i in p) == [0, 1]
    assert sum(1 for p in a if not p) == 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        def register(i):
            # stand-in for a registration: deterministic per pair, independent of the rank
            return {"value": -1.0 / (1.0 + i), "iterations": 10 + i}
        out = run_pairs(costs, register, rank, world)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_gathers_all_results():
    costs = [pair_cost(s) for s in _sizes(10, seed=3)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a = assign_pairs(costs, 2)
    for rank in (0, 1):
        out = res[rank]
        assert [r["pair"] for r in out] == list(range(len(costs)))
        for r in out:
            assert r["value"] == pytest.approx(-1.0 / (1.0 + r["pair"]))
            assert r["pair"] in a[r["rank"]]
    assert res[0] == res[1]
