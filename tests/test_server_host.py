"""Host-side logic of the screening server (CPU only): slicing, admission order (FIFO and
shortest-remaining-first with ageing) under the pair and HBM budgets, retirement accounting,
top-K merging, cancellation and deadlines with launches in flight, and the sharded
multi-rank server over gloo (2 ranks) against a single server.

The device is replaced by a host engine (``FakeEngine``) whose launches can be held open; a
pair's score is a fixed function of the query and the global library index, as a real pair's
result depends only on the pair."""
import collections
import os
import threading
import time

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fast_shepherd_score_b200.screen import Hit
from fast_shepherd_score_b200.server import (Planner, Request, ServeLoop, latency_by_decade,
                                             merge_hits, merge_topk, shard_ranges, slowdown)


def _req(rid, n, k=5, arrival=0.0):
    return Request(rid, {}, np.arange(n, dtype=np.int32), k, arrival)


def pair_scores(seed, j):
    """The host engine's 'alignment score' of library molecule j against query `seed`."""
    j = np.asarray(j, np.float64)
    return (np.abs(np.sin(seed * 12.9898 + j * 78.233)) * 0.999).astype(np.float32)


class FakeEngine:
    """launch(slices) computes every pair's row at once; wait() returns it after `gate` is
    set (None: at once).  ``offset`` maps shard-local indices to global ones."""

    def __init__(self, offset=0, gate=None):
        self.offset, self.gate = offset, gate
        self.launches = []

    def launch(self, slices):
        self.launches.append([(s.req.rid, s.start, s.stop) for s in slices])
        rows = []
        for s in slices:
            j = s.req.lib_idx[s.start:s.stop].astype(np.int64) + self.offset
            r = np.zeros((s.n, 8), np.float32)
            r[:, 0] = pair_scores(s.req.query["seed"], j)
            r[:, 1] = 1.0
            rows.append(r)
        return np.concatenate(rows)

    def wait(self, h):
        if self.gate is not None:
            assert self.gate.wait(30)
        return h


def _loop(engine, n_lib=10_000, max_pairs=4000, slice_pairs=1000, budget=10 ** 12, **kw):
    return ServeLoop(engine, n_lib, Planner(max_pairs, budget, 100, slice_pairs,
                                            kw.pop("policy", "srpt")), **kw)


def test_planner_fifo_slices_and_pair_budget():
    pl = Planner(max_pairs_per_launch=10_000, hbm_budget_bytes=10 ** 12, bytes_per_pair=100,
                 slice_pairs=4096, policy="fifo")
    pend = collections.deque([_req(0, 9000), _req(1, 3000)])
    s1 = pl.plan(pend)
    assert [(s.req.rid, s.start, s.stop) for s in s1] == [(0, 0, 4096), (0, 4096, 8192),
                                                          (0, 8192, 9000), (1, 0, 1000)]
    assert sum(s.n for s in s1) == 10_000
    s2 = pl.plan(pend)
    assert [(s.req.rid, s.start, s.stop) for s in s2] == [(1, 1000, 3000)]
    assert pl.plan(pend) == []


def test_planner_shortest_remaining_first_with_ageing():
    pl = Planner(max_pairs_per_launch=3000, hbm_budget_bytes=10 ** 12, bytes_per_pair=100,
                 slice_pairs=1000, policy="srpt", aging_s=1.0)
    big, small = _req(0, 50_000, arrival=0.0), _req(1, 1500, arrival=0.5)
    pend = collections.deque([big, small])
    s1 = pl.plan(pend, now=0.5)                     # the small request goes first
    assert [(s.req.rid, s.n) for s in s1] == [(1, 1000), (1, 500), (0, 1000), (0, 500)]
    # ageing: a request waiting long enough overtakes a newer, smaller one
    late = _req(2, 2000, arrival=100.0)
    pend = collections.deque([big, late])
    assert pl.order(pend, now=100.0)[0] is big      # 48500 / 101 < 2000
    assert pl.order(collections.deque([big, _req(3, 400, arrival=100.0)]), 100.0)[0].rid == 3


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


def test_serve_loop_results_and_stats():
    eng = FakeEngine()
    with _loop(eng) as srv:
        idx = np.arange(200, 7300, dtype=np.int32)
        hits = srv.submit({"seed": 3}, idx, top_k=9).result(timeout=30)
        small = srv.submit({"seed": 4}, np.arange(50), top_k=3).result(timeout=30)
        st = srv.stats()
    want = idx[np.argsort(-pair_scores(3, idx), kind="stable")[:9]]
    assert [h.id for h in hits] == want.tolist()
    assert len(small) == 3
    assert st["completed"] == 2 and st["in_flight_bytes"] == 0
    assert set(st["by_request_size"]) == {"1e1-1e2", "1e3-1e4"}


def test_cancel_with_slices_in_flight():
    """A request cancelled while its first launch is in flight: the launch's HBM budget is
    returned when it retires, nothing more of it is launched, its future never resolves with
    hits, and a request queued behind it still completes."""
    gate = threading.Event()
    eng = FakeEngine(gate=gate)
    srv = _loop(eng, max_pairs=2000, slice_pairs=1000, max_in_flight=1)
    try:
        big = srv.submit({"seed": 1}, np.arange(9000), top_k=5)
        t0 = time.time()
        while not eng.launches and time.time() - t0 < 10:
            time.sleep(0.005)
        assert eng.launches[0] == [(0, 0, 1000), (0, 1000, 2000)]
        assert srv.stats()["in_flight_bytes"] == 2000 * 100
        assert srv.cancel(big)
        other = srv.submit({"seed": 2}, np.arange(500), top_k=5)
        gate.set()
        assert len(other.result(timeout=30)) == 5
        st = srv.stats()
        assert big.cancelled() and st["cancelled"] == 1 and st["completed"] == 1
        assert st["in_flight_bytes"] == 0 and st["queue_depth"] == 0
        launched = [r for L in eng.launches for r in L]
        assert [x for x in launched if x[0] == 0] == [(0, 0, 1000), (0, 1000, 2000)]
    finally:
        gate.set()
        srv.close()


def test_deadline_expiry():
    gate = threading.Event()
    eng = FakeEngine(gate=gate)
    srv = _loop(eng, max_pairs=1000, slice_pairs=1000, max_in_flight=1)
    try:
        fut = srv.submit({"seed": 5}, np.arange(5000), top_k=5, timeout=0.05)
        time.sleep(0.2)
        gate.set()
        with pytest.raises(TimeoutError):
            fut.result(timeout=30)
        assert srv.submit({"seed": 6}, np.arange(10), top_k=2).result(timeout=30)
        st = srv.stats()
        assert st["expired"] == 1 and st["in_flight_bytes"] == 0
        assert sum(x[0] == 0 for L in eng.launches for x in L) == 1   # only the first slice
    finally:
        gate.set()
        srv.close()


def test_latency_by_decade():
    rec = [(1500, 0.01), (2000, 0.03), (50_000, 0.2), (99_999, 0.4)]
    d = latency_by_decade(rec)
    assert d["1e3-1e4"]["requests"] == 2 and d["1e4-1e5"]["requests"] == 2


def test_slowdown_normalises_by_service_time():
    # capacity 1000 pairs/s: a 2000-pair request served alone takes 2 s (slowdown 1)
    rec = [(2000, 2.0), (2000, 4.0), (50_000, 50.0), (50_000, 150.0)]
    d = slowdown(rec, 1000.0)
    assert d["by_request_size"]["1e3-1e4"]["p50"] == pytest.approx(1.5)
    assert d["by_request_size"]["1e4-1e5"]["p99"] == pytest.approx(2.98, abs=0.01)
    assert slowdown([], 1000.0) == {} and slowdown(rec, 0.0) == {}


def test_shard_ranges_and_merge_hits():
    rs = shard_ranges(10, 3)
    assert rs[0][0] == 0 and rs[-1][1] == 10
    assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
    h = merge_hits([[Hit(0.9, 1, None), Hit(0.5, 2, None)], [Hit(0.7, 8, None)]], 2)
    assert [x.id for x in h] == [1, 8]


REQUESTS = [(11, (0, 3000), 7), (12, (1200, 1900), 4), (13, (2500, 2510), 3),
            (14, (0, 3000), 50), (15, (100, 140), 100)]


def _sharded_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from fast_shepherd_score_b200.sharded import ShardedScreenServer
    n_lib = 3000
    lo, hi = shard_ranges(n_lib, world)[rank]
    local = ServeLoop(FakeEngine(offset=lo), hi - lo, Planner(1500, 10 ** 12, 100, 500),
                      ids=np.arange(lo, hi))
    srv = ShardedScreenServer(local, lo, hi, n_lib)
    if rank == 0:
        futs = [srv.submit({"seed": s}, np.arange(a, b), top_k=k) for s, (a, b), k in REQUESTS]
        got = [[(h.id, h.score) for h in f.result(timeout=60)] for f in futs]
        # the same requests on one server holding the whole library
        with ServeLoop(FakeEngine(), n_lib, Planner(1500, 10 ** 12, 100, 500),
                       ids=np.arange(n_lib)) as one:
            want = [[(h.id, h.score) for h in one.submit({"seed": s}, np.arange(a, b),
                                                          top_k=k).result(timeout=60)]
                    for s, (a, b), k in REQUESTS]
        out.put((got == want, got[0][:3], want[0][:3], srv.ticks > 0))
    srv.close()
    dist.destroy_process_group()


def test_sharded_server_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_sharded_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    same, g, w, ticked = q.get(timeout=180)
    for p in procs:
        p.join(timeout=120)
    assert same, (g, w)
    assert ticked and all(p.exitcode == 0 for p in procs)
