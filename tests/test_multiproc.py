"""Two-rank (gloo, CPU) tests of the multi-GPU host logic: max-over-ranks
timing and the sharding of independent problems across ranks, exercised on
oracle FMM runs of a small batch (each rank evaluates its shard; the
gathered results equal a single-rank evaluation)."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from sumpy_b200.distributed import max_over_ranks, shard_problems


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(i):
    rng = np.random.default_rng(1000 + i)
    n = int(np.exp(rng.uniform(np.log(200), np.log(800))))
    return rng.random((3, n)), rng.standard_normal(n)


def _worker(rank, world, port, out_q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle as O
        from sumpy_b200.tree import build_all
        costs = [_problem(i)[0].shape[1] for i in range(6)]
        mine = shard_problems(costs, world)[rank]
        res = {}
        for i in mine:
            pts, q = _problem(i)
            tree, trav, tcls = build_all(pts, None, 16)
            res[i] = O.run_fmm(tree, trav, tcls, 4, q, exclude_self=True)
        gathered = [None] * world
        dist.all_gather_object(gathered, res)
        tmax = max_over_ranks(10.0 + rank)
        if rank == 0:
            merged = {}
            for g in gathered:
                merged.update(g)
            out_q.put((tmax, merged))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_batch_matches_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    tmax, merged = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert tmax == 11.0
    assert sorted(merged) == list(range(6))
    from oracle import oracle as O
    from sumpy_b200.tree import build_all
    for i, pot in merged.items():
        pts, qq = _problem(i)
        tree, trav, tcls = build_all(pts, None, 16)
        ref = O.run_fmm(tree, trav, tcls, 4, qq, exclude_self=True)
        assert np.array_equal(pot, ref)


def test_shard_problems_partitions_and_balances():
    costs = [5, 1, 9, 3, 3, 7, 2]
    shards = shard_problems(costs, 3)
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= max(costs)
    assert max_over_ranks(4.5) == 4.5  # single process: identity
