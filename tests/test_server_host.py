"""Host-side logic of the screening server (CPU): slicing, FIFO admission under the pair
and HBM budgets, retirement accounting, top-K merging, shard ranges and hit merging, and a
2-rank gloo run of the sharded top-K merge."""
import collections
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fast_shepherd_score_b200.screen import Hit
from fast_shepherd_score_b200.server import (Planner, Request, merge_hits, merge_topk,
                                             shard_ranges)


def _req(rid, n, k=5):
    return Request(rid, {}, np.arange(n, dtype=np.int32), k, 0.0)


def test_planner_fifo_slices_and_pair_budget():
    pl = Planner(max_pairs_per_launch=10_000, hbm_budget_bytes=10 ** 12, bytes_per_pair=100,
                 slice_pairs=4096)
    pend = collections.deque([_req(0, 9000), _req(1, 3000)])
    s1 = pl.plan(pend)
    assert [(s.req.rid, s.start, s.stop) for s in s1] == [(0, 0, 4096), (0, 4096, 8192),
                                                          (0, 8192, 9000), (1, 0, 1000)]
    assert sum(s.n for s in s1) == 10_000
    s2 = pl.plan(pend)
    assert [(s.req.rid, s.start, s.stop) for s in s2] == [(1, 1000, 3000)]
    assert pl.plan(pend) == []


def test_planner_hbm_budget_admission_and_retirement():
    pl = Planner(max_pairs_per_launch=10 ** 6, hbm_budget_bytes=5000 * 100, bytes_per_pair=100,
                 slice_pairs=2000)
    pend = collections.deque([_req(0, 8000)])
    s1 = pl.plan(pend)
    assert sum(s.n for s in s1) == 4000            # 3 slices of 2000 would exceed 5000 pairs
    b = pl.admit(s1)
    assert pl.plan(pend) == []                      # budget held by the in-flight launch
    pl.retire(b)
    s2 = pl.plan(pend)
    assert sum(s.n for s in s2) == 4000 and pend[0].next == 8000


def test_merge_topk_matches_global_topk():
    rng = np.random.default_rng(0)
    r = _req(0, 1000, k=7)
    s = rng.random(1000)
    for a in range(0, 1000, 130):
        b = min(a + 130, 1000)
        merge_topk(r, s[a:b], np.arange(a, b), np.zeros((b - a, 4)), np.zeros((b - a, 3)))
    assert set(r.best_i.tolist()) == set(np.argsort(-s)[:7].tolist())


def test_shard_ranges_and_merge_hits():
    rs = shard_ranges(10, 3)
    assert rs[0][0] == 0 and rs[-1][1] == 10
    assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
    h = merge_hits([[Hit(0.9, 1, None), Hit(0.5, 2, None)], [Hit(0.7, 8, None)]], 2)
    assert [x.id for x in h] == [1, 8]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    n, k = 1000, 10
    lo, hi = shard_ranges(n, world)[rank]
    scores = np.random.default_rng(1).random(n)     # every rank sees the same "library"
    mine = [Hit(float(scores[i]), i, None) for i in range(lo, hi)]
    mine = sorted(mine, key=lambda h: -h.score)[:k]
    gathered = [None] * world
    dist.all_gather_object(gathered, [(h.score, h.id) for h in mine])
    if rank == 0:
        top = merge_hits([[Hit(s, i, None) for s, i in g] for g in gathered], k)
        out.put([h.id for h in top] == np.argsort(-scores)[:k].tolist())
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_topk_merge_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ok = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
    assert ok
