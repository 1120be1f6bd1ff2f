"""Pair-parallel scheduling on CPU: assignment properties and a world_size-2 gloo run in which
each rank registers its pairs for real (FP64 oracle evaluator and optimizer)."""
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


# small 2-D pairs of uneven sizes, registered for real on the CPU by the FP64 restatement of the
# evaluator and of the adaptive-step optimizer (the oracle), so that each rank does actual work
PAIR_SHAPES = [(22, 24), (30, 26), (24, 34), (28, 28), (20, 36), (34, 30)]
PAIR_ITERS = 6


def _register_pair(i):
    """One pair: NCC + RD, control spacing 2, PAIR_ITERS optimizer iterations (FP64 oracle)."""
    from helpers import make_problem
    from oracle import oracle as O
    from skmimageregistration_b200.abi import MetricDesc, OptimizerDesc
    pb, _, _ = make_problem(2, shape=PAIR_SHAPES[i], seed=100 + i, sigma_c4=4.0, sigma_c0=8.0, cp_spacing=2.0,
                            spacing=(1.0, 1.0), origin=(0.0, 0.0))
    orc = O.Oracle(pb)
    m = MetricDesc.make("ncc", rd=1e-3)
    o = OptimizerDesc.make(a=200.0, number_of_iterations=PAIR_ITERS)
    opt = O.OracleOptimizer(orc, o, m, np.zeros(pb.num_parameters), np.ones(pb.C))
    vals = opt.run(PAIR_ITERS)
    out = {"first_value": float(vals[0]), "best_value": float(opt.state.best_value), "iterations": PAIR_ITERS,
           "best_checksum": float(np.sum(opt.best * np.arange(1, opt.best.size + 1)))}
    orc.close()
    return out


def _worker(rank, world, port, costs, q):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = run_pairs(costs, _register_pair, rank, world)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_registers_pairs_and_gathers_all_results():
    costs = [pair_cost(s + (1,), cp_spacing_voxels=2.0, support_voxels=4.0, D=2) for s in PAIR_SHAPES]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a = assign_pairs(costs, 2)
    assert all(a)                                          # both ranks registered pairs
    # the same registrations run in this process, one after the other
    single = {i: _register_pair(i) for i in range(len(PAIR_SHAPES))}
    for rank in (0, 1):
        out = res[rank]
        assert [r["pair"] for r in out] == list(range(len(PAIR_SHAPES)))
        for r in out:
            assert r["pair"] in a[r["rank"]]
            ref = single[r["pair"]]
            assert r["best_value"] < r["first_value"]      # the optimizer made progress on every pair
            for k in ("first_value", "best_value", "best_checksum"):
                assert r[k] == ref[k], (r, ref)          # deterministic: bitwise the single-process run
    assert res[0] == res[1]
