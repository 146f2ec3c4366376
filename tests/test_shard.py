"""Sharding independent bodies over ranks (nnkifmm.shard): the partition and
the final gather, with two gloo ranks on the CPU and a stand-in for the GPU
forest batch."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from nnkifmm.shard import partition, solve_modes_sharded


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = list(rng.integers(1000, 50000, 37))
    for world in (1, 2, 3, 8):
        parts = partition(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    assert partition([5, 5], 4) == [[0], [1], [], []]


def _fake_solver(bodies, kernelPar, tol, maxIter, **kw):
    # a 6 x 6 "mobility matrix" that identifies the body, and its info
    mats = [np.full((6, 6), float(len(c)) + kernelPar[0]) for c, _ in bodies]
    infos = [[(0, tol, len(f))] * 6 for _, f in bodies]
    return mats, infos


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(1)
        bodies = [(np.zeros((n, 3)), np.zeros((16 * n, 3))) for n in rng.integers(10, 200, 9)]
        mats, infos = solve_modes_sharded(bodies, [0.5, 1.0], tol=1e-7, solver=_fake_solver)
        ok = all(np.array_equal(m, np.full((6, 6), len(c) + 0.5)) for m, (c, _) in zip(mats, bodies))
        ok = ok and all(inf == [(0, 1e-7, len(f))] * 6 for inf, (_, f) in zip(infos, bodies))
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_in_body_order():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res == [(0, True), (1, True)]
